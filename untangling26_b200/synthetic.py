"""Seeded synthetic scenes standing in for the reference's procedural cloth demos.

No dataset is read. Each generator takes a seed (numpy PCG64) and returns a Mesh.

* two_sheets(n): two n x n vertex sheets of 1 m. Sheet B sits 2 mm above sheet A and
  carries a sinusoidal bump of amplitude U[0.05, 0.2] m with 1-3 periods pushed down
  through A (closed intersection contours). n = 64 is the small CPU-runnable scene,
  n = 32 / 128 the differentiation-form sizes.
* folded_sheet(n): one n x n sheet (n = 256: 130,050 triangles) folded flat about a
  seeded line, then Gaussian vertex noise of 0.3 x edge length on every axis, so that
  the two layers cross each other in figure-eight and boundary-ending contours.
* sheets_in_contact(n): two_sheets(n) with a third sheet lying exactly on sheet A (zero-distance
  proximity pairs, for the near-zero-distance EF conversion).
* layered_sheets(n, layers): stacked n x n sheets 1 mm apart with seeded multi-octave
  value-noise displacement of 2-20 mm so that layers pass through their neighbours.
* batch_scenes(num): independent two-body scenes (icosphere-derived shells or bumped
  sheets, 2k-60k triangles each) laid out apart, for the batched-vs-per-scene comparison.
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


def sheets_in_contact(n=32, seed=0):
    """two_sheets(n) plus a third sheet lying exactly on sheet A (the same vertex positions,
    its own object): every vertex and edge of it is at zero distance from A, the
    near-zero-distance proximity pairs that the reference turns into EF pairs when
    ignore_near_zero_dist_pairs is off."""
    m2 = two_sheets(n, seed)
    nn = n * n
    xa = m2.x[:nn]
    x = np.concatenate([m2.x, xa], 0)
    faces = np.concatenate([m2.faces, m2.faces[: len(m2.faces) // 2] + 2 * nn], 0)
    obj = np.concatenate([np.zeros(nn, np.uint32), np.ones(nn, np.uint32), np.full(nn, 2, np.uint32)])
    rest = np.concatenate([m2.rest_x, m2.rest_x[:nn]], 0)
    m = Mesh(x.astype(np.float32), faces, object_of_vert=obj, rest_x=rest)
    m.meta = dict(m2.meta, kind="sheets_in_contact")
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
    h = 1.0 / (n - 1)
    for k in range(layers):
        x = xg.copy()
        # a seeded sub-cell xy shift per layer keeps the layers' edges off each other's edges
        # (coincident grids put every crossing on a triangle boundary)
        x[:, :2] += rng.uniform(0.2, 0.45, 2) * h * (k > 0)
        amp = rng.uniform(0.002, 0.020)
        x[:, 2] = 0.001 * k + amp * _value_noise(rng, x[:, 0], x[:, 1])
        xs.append(x)
        rest = x.copy()
        rest[:, 2] = 0.001 * k
        rests.append(rest)
        fs.append(f + k * n * n)
        obj.append(np.full(n * n, k, np.uint32))
    m = Mesh(np.concatenate(xs).astype(np.float32), np.concatenate(fs), object_of_vert=np.concatenate(obj),
             rest_x=np.concatenate(rests).astype(np.float32))
    m.meta = {"kind": "layered_sheets", "n": n, "layers": layers, "seed": seed}
    return m


def icosphere(level):
    """Unit icosphere: the icosahedron with every triangle split in four `level` times (edge
    midpoints pushed to the sphere); outward winding. 20 * 4^level triangles."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1),
         (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
         (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, np.float64) / np.linalg.norm(p) for p in v]
    faces = f
    for _ in range(level):
        mid = {}

        def m(a, b):
            k = (min(a, b), max(a, b))
            if k not in mid:
                p = verts[a] + verts[b]
                verts.append(p / np.linalg.norm(p))
                mid[k] = len(verts) - 1
            return mid[k]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = m(a, b), m(b, c), m(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(verts), np.array(faces, np.uint32)


def _rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def _shell_pair(tris, rng):
    """Two closed shells derived from icospheres (radius U[0.1, 0.5] m, seeded low-order
    radial bumps), overlapped by U[5%, 60%] of the smaller radius."""
    level = int(np.clip(np.round(np.log(max(tris, 80) / 40.0) / np.log(4.0)), 2, 6))
    unit, f = icosphere(level)
    parts, rests = [], []
    radii = rng.uniform(0.1, 0.5, 2)
    depth = rng.uniform(0.05, 0.6) * radii.min()
    centers = [np.zeros(3), np.array([radii[0] + radii[1] - depth, 0.0, 0.0])]
    for k in range(2):
        R = _rotation(rng)
        d = unit @ R.T
        bump = np.zeros(len(d))
        for _ in range(3):
            a = _rotation(rng)[0]
            bump += rng.uniform(0.0, 0.06) * np.cos(rng.integers(2, 6) * np.arccos(np.clip(d @ a, -1.0, 1.0)))
        rests.append(centers[k] + radii[k] * d)
        parts.append(centers[k] + radii[k] * (1.0 + bump)[:, None] * d)
    return parts, rests, [f, f], {"kind": "shells", "level": level, "radii": radii.tolist(), "depth": float(depth)}


def _sheet_pair(tris, rng):
    n = int(np.clip(np.round(np.sqrt(tris / 4.0)) + 1, 8, 256))
    m = two_sheets(n, seed=int(rng.integers(0, 2 ** 31)))
    nv = n * n
    x = m.x.astype(np.float64)
    rest = m.rest_x.astype(np.float64)
    f = m.faces[: len(m.faces) // 2]
    return [x[:nv], x[nv:]], [rest[:nv], rest[nv:]], [f, f], {"kind": "sheets", "n": n, **{k: m.meta[k] for k in ("amplitude", "periods")}}


def batch_scenes(num=64, seed=2, tris_lo=2000, tris_hi=60000, spacing=3.0):
    """The batching workload: `num` independent two-body scenes, each with a seeded triangle
    count uniform in [tris_lo, tris_hi], made of a pair of icosphere-derived closed shells or
    a pair of bumped cloth sheets, laid out on a grid `spacing` m apart so that no two
    scenes touch. meta["scenes"] lists each scene's vertex / face ranges, so every scene can
    also be evaluated on its own (scene_mesh)."""
    rng = np.random.default_rng(seed)
    xs, rests, fs, obj, scenes = [], [], [], [], []
    nv = nf = 0
    cols = int(np.ceil(np.sqrt(num)))
    for s in range(num):
        tris = int(rng.integers(tris_lo, tris_hi + 1))
        parts, prest, pf, info = (_shell_pair if rng.uniform() < 0.5 else _sheet_pair)(tris, rng)
        off = np.array([spacing * (s % cols), spacing * (s // cols), 0.0])
        v0, f0 = nv, nf
        for k in range(2):
            xs.append(parts[k] + off)
            rests.append(prest[k] + off)
            fs.append(pf[k] + nv)
            obj.append(np.full(len(parts[k]), 2 * s + k, np.uint32))
            nv += len(parts[k])
            nf += len(pf[k])
        scenes.append(dict(info, verts=[v0, nv], faces=[f0, nf], tris=nf - f0))
    m = Mesh(np.concatenate(xs).astype(np.float32), np.concatenate(fs).astype(np.uint32), object_of_vert=np.concatenate(obj),
             rest_x=np.concatenate(rests).astype(np.float32))
    m.object_scene = np.repeat(np.arange(num, dtype=np.uint32), 2)
    m.meta = {"kind": "batch_scenes", "num": num, "seed": seed, "scenes": scenes}
    return m


def sub_batch(batch, scene_ids):
    """The listed scenes of a batch_scenes mesh as a batch of their own (same positions, in
    the listed order); meta["scenes"][j]["batch_scene"] names scene j's index in `batch`."""
    xs, rests, fs, obj, scenes = [], [], [], [], []
    nv = nf = 0
    for j, s in enumerate(scene_ids):
        sc = batch.meta["scenes"][s]
        v0, v1 = sc["verts"]
        f0, f1 = sc["faces"]
        xs.append(batch.x[v0:v1])
        rests.append(batch.rest_x[v0:v1])
        fs.append(batch.faces[f0:f1] - v0 + nv)
        obj.append(batch.object_of_vert[v0:v1] - batch.object_of_vert[v0] + 2 * j)
        scenes.append(dict(sc, verts=[nv, nv + v1 - v0], faces=[nf, nf + f1 - f0], batch_scene=int(s)))
        nv += v1 - v0
        nf += f1 - f0
    m = Mesh(np.concatenate(xs), np.concatenate(fs).astype(np.uint32), object_of_vert=np.concatenate(obj).astype(np.uint32),
             rest_x=np.concatenate(rests))
    m.object_scene = np.repeat(np.arange(len(scene_ids), dtype=np.uint32), 2)
    m.meta = {"kind": "batch_scenes", "num": len(scene_ids), "seed": batch.meta["seed"], "scenes": scenes,
              "of_batch": batch.meta["num"]}
    return m


def scene_mesh(batch, s):
    """Scene s of a batch_scenes mesh as a mesh of its own (same positions)."""
    sc = batch.meta["scenes"][s]
    v0, v1 = sc["verts"]
    f0, f1 = sc["faces"]
    x = batch.x[v0:v1]
    objv = batch.object_of_vert[v0:v1] - batch.object_of_vert[v0]
    m = Mesh(x, (batch.faces[f0:f1] - v0).astype(np.uint32), object_of_vert=objv.astype(np.uint32), rest_x=batch.rest_x[v0:v1])
    m.meta = {"kind": "scene_of_batch", "scene": s, **sc}
    return m
