"""Seeded synthetic scenes standing in for the reference's procedural cloth demos.

No dataset is read. Each generator takes a seed (numpy PCG64) and returns a Mesh.

* two_sheets(n): two n x n vertex sheets of 1 m. Sheet B sits 2 mm above sheet A and
  carries a sinusoidal bump of amplitude U[0.05, 0.2] m with 1-3 periods pushed down
  through A (closed intersection contours). n = 64 is the small CPU-runnable scene,
  n = 32 / 128 the differentiation-form sizes.
* folded_sheet(n): one n x n sheet (n = 256: 130,050 triangles) folded flat about a
  seeded line, then Gaussian vertex noise of 0.3 x edge length on every axis, so that
  the two layers cross each other in figure-eight and boundary-ending contours.
* layered_sheets(n, layers): stacked n x n sheets 1 mm apart with seeded multi-octave
  value-noise displacement of 2-20 mm so that layers pass through their neighbours.
"""
import numpy as np

from .mesh import Mesh


def grid(n, size=1.0):
    """n x n vertices on [0, size]^2 at z = 0 with a fixed diagonal split."""
    u = np.linspace(0.0, size, n, dtype=np.float64)
    xx, yy = np.meshgrid(u, u, indexing="ij")
    x = np.stack([xx.reshape(-1), yy.reshape(-1), np.zeros(n * n)], 1)
    i, j = np.meshgrid(np.arange(n - 1), np.arange(n - 1), indexing="ij")
    v00 = (i * n + j).reshape(-1)
    v10 = ((i + 1) * n + j).reshape(-1)
    v01 = (i * n + j + 1).reshape(-1)
    v11 = ((i + 1) * n + j + 1).reshape(-1)
    f = np.concatenate([np.stack([v00, v10, v11], 1), np.stack([v00, v11, v01], 1)], 0)
    # interleave the two triangles of each cell so face ids follow the cells
    f = f.reshape(2, -1, 3).transpose(1, 0, 2).reshape(-1, 3)
    return x, f.astype(np.uint32)


def two_sheets(n=64, seed=0):
    rng = np.random.default_rng(seed)
    amp = rng.uniform(0.05, 0.2)
    periods = int(rng.integers(1, 4))
    xa, f = grid(n)
    xb = xa.copy()
    # a seeded sub-cell xy shift keeps B's edges off A's edges (coincident grids would
    # put every crossing on a triangle boundary, which the EF filters reject)
    h = 1.0 / (n - 1)
    xb[:, :2] += rng.uniform(0.2, 0.45, 2) * h
    u, v = xa[:, 0], xa[:, 1]
    bump = (np.sin(np.pi * periods * u) ** 2) * (np.sin(np.pi * periods * v) ** 2)
    xb[:, 2] = 0.002 - amp * bump
    x = np.concatenate([xa, xb], 0)
    faces = np.concatenate([f, f + n * n], 0)
    obj = np.concatenate([np.zeros(n * n, np.uint32), np.ones(n * n, np.uint32)])
    m = Mesh(x.astype(np.float32), faces, object_of_vert=obj, rest_x=np.concatenate([xa, xb * [1, 1, 0] + [0, 0, 0.002]], 0))
    m.meta = {"kind": "two_sheets", "n": n, "seed": seed, "amplitude": amp, "periods": periods}
    return m


def folded_sheet(n=256, seed=1, noise=0.3):
    rng = np.random.default_rng(seed)
    x, f = grid(n)
    rest = x.copy()
    h = 1.0 / (n - 1)
    # fold line through a point near the centre with a seeded direction
    p = np.array([0.5, 0.5]) + rng.uniform(-0.1, 0.1, 2)
    ang = rng.uniform(0.0, np.pi)
    d = np.array([np.cos(ang), np.sin(ang)])
    nrm = np.array([-d[1], d[0]])
    s = (x[:, :2] - p) @ nrm
    side = s > 0
    # rotate the positive side by pi about the fold line: a flat fold onto the other half
    x[side, :2] -= 2.0 * s[side, None] * nrm[None, :]
    x += rng.normal(0.0, noise * h, x.shape)
    m = Mesh(x.astype(np.float32), f, rest_x=rest.astype(np.float32))
    m.meta = {"kind": "folded_sheet", "n": n, "seed": seed, "fold_point": p.tolist(), "fold_angle": ang,
              "noise_sigma": noise * h}
    return m


def _value_noise(rng, u, v, octaves=4):
    out = np.zeros_like(u)
    amp, freq, total = 1.0, 2, 0.0
    for _ in range(octaves):
        g = rng.uniform(-1.0, 1.0, (freq + 1, freq + 1))
        gu, gv = u * freq, v * freq
        i0 = np.clip(np.floor(gu).astype(int), 0, freq - 1)
        j0 = np.clip(np.floor(gv).astype(int), 0, freq - 1)
        fu, fv = gu - i0, gv - j0
        su, sv = fu * fu * (3 - 2 * fu), fv * fv * (3 - 2 * fv)
        a = g[i0, j0] * (1 - su) + g[i0 + 1, j0] * su
        b = g[i0, j0 + 1] * (1 - su) + g[i0 + 1, j0 + 1] * su
        out += amp * (a * (1 - sv) + b * sv)
        total += amp
        amp *= 0.5
        freq *= 2
    return out / total


def layered_sheets(n=512, layers=5, seed=4):
    rng = np.random.default_rng(seed)
    xg, f = grid(n)
    xs, fs, obj, rests = [], [], [], []
    for k in range(layers):
        x = xg.copy()
        amp = rng.uniform(0.002, 0.020)
        x[:, 2] = 0.001 * k + amp * _value_noise(rng, x[:, 0], x[:, 1])
        xs.append(x)
        rest = xg.copy()
        rest[:, 2] = 0.001 * k
        rests.append(rest)
        fs.append(f + k * n * n)
        obj.append(np.full(n * n, k, np.uint32))
    m = Mesh(np.concatenate(xs).astype(np.float32), np.concatenate(fs), object_of_vert=np.concatenate(obj),
             rest_x=np.concatenate(rests).astype(np.float32))
    m.meta = {"kind": "layered_sheets", "n": n, "layers": layers, "seed": seed}
    return m
