"""The closed-form derivatives of the hit distance delta(x, r) = (w . n) / (r . n) and of the
objective J = (sum A) max(delta)^2 and displacement cost E = sum (delta + 3e-3)^2 / kappa,
checked against FP64 central differences (h = 1e-6 on x, 1e-7 on r) over 100 seeded trials.
CPU only: this pins the formulas the CUDA adjoint kernel evaluates."""
import numpy as np
import pytest

from oracle import adjoint as adj


def _hit(oracle, rng, t):
    """A hit of type t on vertices 0..3 (VF: p a b c, FV: q a b c, EE: p0 p1 q0 q1)."""
    if t == 0:
        sv = [0]
        dv = [1, 2, 3]
    elif t == 2:
        sv = [1, 2, 3]
        dv = [0]
    else:
        sv = [0, 1]
        dv = [2, 3]
    return oracle.hit(t, 0, 0, sv, dv, tuple(rng.uniform(0.1, 0.4, 2)), 0.0)[0]


def _grazing(h, P, r):
    """|r . n| / |n| of the hit's plane (small: the distance is ill-conditioned)."""
    Q = P[adj.hit_vertices(h)]
    n = np.cross(Q[1] - Q[0], Q[3] - Q[2]) if int(h["type"]) == 1 else np.cross(Q[2] - Q[1], Q[3] - Q[1])
    return abs(np.dot(r, n)) / np.linalg.norm(n)


def _random_case(oracle, rng):
    while True:
        h = _hit(oracle, rng, int(rng.integers(0, 3)))
        P = rng.normal(size=(4, 3))
        r = rng.normal(size=3)
        r /= np.linalg.norm(r)
        if _grazing(h, P, r) > 0.2:
            return h, P, r


def test_delta_gradient_central_differences(oracle):
    rng = np.random.default_rng(26)
    for _ in range(100):
        h, P, r = _random_case(oracle, rng)
        V = adj.hit_vertices(h)
        gP, gr = adj.delta_grads(h, P[V], r)
        for k in range(4):
            for a in range(3):
                hx = 1e-6
                Pp, Pm = P.copy(), P.copy()
                Pp[V[k], a] += hx
                Pm[V[k], a] -= hx
                fd = (adj.delta(h, Pp[V], r) - adj.delta(h, Pm[V], r)) / (2 * hx)
                assert abs(fd - gP[k, a]) <= 1e-6 * (1 + abs(gP[k, a])), (int(h["type"]), k, a, fd, gP[k, a])
        for a in range(3):
            hr = 1e-7
            rp, rm = r.copy(), r.copy()
            rp[a] += hr
            rm[a] -= hr
            fd = (adj.delta(h, P[V], rp) - adj.delta(h, P[V], rm)) / (2 * hr)
            assert abs(fd - gr[a]) <= 1e-5 * (1 + abs(gr[a]))
        # translation invariance: the vertex derivatives sum to zero
        assert np.abs(gP.sum(0)).max() <= 1e-9 * (1 + np.abs(gP).max())


def test_objective_gradient_central_differences(oracle):
    """J and E of a multi-hit support (distinct maxima, so J is smooth at the point)."""
    rng = np.random.default_rng(27)
    nv = 12
    checked = 0
    for _ in range(20):
        hits = []
        for k in range(3):
            t = int(rng.integers(0, 3))
            base = 4 * k
            if t == 0:
                hits.append(oracle.hit(0, base, 0, [base], [base + 1, base + 2, base + 3], tuple(rng.uniform(0.1, 0.4, 2)), 0.0)[0])
            elif t == 2:
                hits.append(oracle.hit(2, 0, base, [base + 1, base + 2, base + 3], [base], tuple(rng.uniform(0.1, 0.4, 2)), 0.0)[0])
            else:
                hits.append(oracle.hit(1, 0, 1, [base, base + 1], [base + 2, base + 3], tuple(rng.uniform(0.1, 0.9, 2)), 0.0)[0])
        x = rng.normal(size=(nv, 3))
        r = rng.normal(size=3)
        r /= np.linalg.norm(r)
        va, ea, fa = rng.uniform(0.5, 2.0, nv), rng.uniform(0.5, 2.0, 4), rng.uniform(0.5, 2.0, 4)
        vm = rng.uniform(0.5, 2.0, nv)
        if min(_grazing(h, x, r) for h in hits) < 0.2:
            continue
        ds = [adj.delta(h, x[adj.hit_vertices(h)], r) for h in hits]
        s = sorted(ds)
        if s[-1] - s[-2] < 1e-3 or max(abs(d) for d in ds) > 50:
            continue
        checked += 1
        gJx, gJr, gEx, gEr = adj.gradients(hits, x, r, va, ea, fa, vm)
        f = lambda xx, rr: adj.objective(hits, xx, rr, va, ea, fa, vm)[:2]
        for v in range(nv):
            for a in range(3):
                xp, xm = x.copy(), x.copy()
                xp[v, a] += 1e-6
                xm[v, a] -= 1e-6
                (Jp, Ep), (Jm, Em) = f(xp, r), f(xm, r)
                assert abs((Jp - Jm) / 2e-6 - gJx[v, a]) <= 1e-5 * (1 + abs(gJx[v, a]))
                assert abs((Ep - Em) / 2e-6 - gEx[v, a]) <= 1e-5 * (1 + abs(gEx[v, a]))
        for a in range(3):
            rp, rm = r.copy(), r.copy()
            rp[a] += 1e-7
            rm[a] -= 1e-7
            (Jp, Ep), (Jm, Em) = f(x, rp), f(x, rm)
            assert abs((Jp - Jm) / 2e-7 - gJr[a]) <= 1e-4 * (1 + abs(gJr[a]))
            assert abs((Ep - Em) / 2e-7 - gEr[a]) <= 1e-4 * (1 + abs(gEr[a]))
    assert checked >= 5
