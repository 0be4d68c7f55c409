"""Oracle restatement of the region-based pair filtering (intersection_resolver.cpp:2232-2676)
checked on the CPU: region-match known answers and an independent numpy restatement of
filter_invalid_pairs / filter_broad_phase_pairs on seeded random inputs."""
import numpy as np

from untangling26_b200.prp import COLLISION_PAIR_DTYPE

M = 0x7FFFFFFF


def _csr(rows):
    n = len(rows)
    off = [n + 1]
    for r in rows:
        off.append(off[-1] + len(r))
    return np.array(off + [v for r in rows for v in r], np.uint32)


def test_region_match_known_answers(oracle):
    a = _csr([[], [4], [4, 9], [2, 7]])
    b = _csr([[], [5], [4], [6, 11]])
    assert oracle.region_match(a, 0, b, 0) == 0  # no regions on either side
    assert oracle.region_match(a, 1, b, 1) == 1  # 4 == 5 ^ 1: same contour, opposite sides
    assert oracle.region_match(a, 1, b, 2) == 2  # same side is not a match
    assert oracle.region_match(a, 0, b, 1) == 2  # regions on one side only
    assert oracle.region_match(a, 3, b, 3) == 1  # 7 == 6 ^ 1
    assert oracle.region_match(a, 2, b, 3) == 2


def _random_case(rng, nv=40, npairs=200):
    x = rng.normal(size=(nv, 3)).astype(np.float32) * 0.05
    off = rng.uniform(0.0, 0.02, nv).astype(np.float32)
    pairs = np.zeros(npairs, COLLISION_PAIR_DTYPE)
    pidx = np.zeros((npairs, 2), np.uint32)
    for i in range(npairs):
        t = rng.integers(0, 4)
        v = rng.choice(nv, 4, replace=False).astype(np.uint32)
        idx = v.copy()
        if t == 0:  # VF
            idx[2] |= 0x80000000
            pidx[i] = (v[0], rng.integers(0, 30))
        elif t == 1:  # EE
            idx[3] |= 0x80000000
            pidx[i] = (rng.integers(0, 50), rng.integers(0, 50))
        elif t == 2:  # VV: (v0, ~0, v1, ~0), type bit on slot 0
            idx = np.array([v[0] | 0x80000000, 0xFFFFFFFF, v[1], 0xFFFFFFFF], np.uint32)
        else:  # VE: (v, ~0, e0, e1)
            idx = np.array([v[0], 0xFFFFFFFF, v[1], v[2]], np.uint32)
        pairs[i]["indices"] = idx
        pairs[i]["vec2"] = (rng.uniform(-1, 0), rng.uniform(0, 1), rng.uniform(0, 1), rng.uniform(0, 1))
        pairs[i]["vec1"] = (0, 0, 1, 1e-3)
    rows = lambda n: [sorted(set(rng.integers(0, 8, rng.integers(0, 3)).tolist())) for _ in range(n)]
    regions = (_csr(rows(nv)), _csr(rows(50)), _csr(rows(30)))
    return x, off, pairs, pidx, regions


def _numpy_filter(pairs, pidx, x, off, regions):
    nv = len(x)
    vr, er, fr = regions

    def rows(c, i):
        return c[c[i]:c[i + 1]]

    def match(a, i, b, j):
        ra, rb = rows(a, i), rows(b, j)
        if len(ra) == 0 and len(rb) == 0:
            return 0
        return 1 if any(int(p) == (int(q) ^ 1) for p in ra for q in rb) else 2

    inv = np.zeros(nv, np.uint32)
    out = pairs.copy()
    for p in pairs:
        idx = p["indices"]
        raw = [int(v) for v in idx]
        t = (raw[0] >> 31) + ((raw[1] >> 31) << 1) + ((raw[2] >> 31) << 2) + ((raw[3] >> 31) << 3)
        b2, b3 = np.float32(p["vec2"][2]), np.float32(p["vec2"][3])
        one = np.float32(1)
        w = {4: (one, -b2, -b3, (b2 + b3) - one), 8: (b2, one - b2, -b3, b3 - one), 1: (one, 0, -one, 0),
             2: (one, 0, -b2, -b3)}.get(t, (0, 0, 0, 0))
        ids = [v & M for v in raw]
        d = np.zeros(3, np.float32)
        for k in range(4):
            if ids[k] < nv:
                d = (d + np.float32(w[k]) * x[ids[k]]).astype(np.float32)
        d2 = np.float32(np.float32(d[0] * d[0] + d[1] * d[1]) + d[2] * d[2])
        th = np.float32(off[ids[0]] + off[ids[2]])
        if d2 < np.float32(th * th + np.float32(1e-10)):
            for k in range(4):
                if ids[k] < nv:
                    inv[ids[k]] = 1
    for i, p in enumerate(out):
        raw = [int(v) for v in p["indices"]]
        ids = [v & M for v in raw]
        t = (raw[0] >> 31) + ((raw[1] >> 31) << 1) + ((raw[2] >> 31) << 2) + ((raw[3] >> 31) << 3)
        off_ = any(v < nv and inv[v] for v in ids)
        if not off_ and t == 4:
            off_ = match(vr, pidx[i][0], fr, pidx[i][1]) == 1
        elif not off_ and t == 8:
            off_ = match(er, pidx[i][0], er, pidx[i][1]) == 1
        if off_:
            out[i]["vec2"][0] = 0
            out[i]["vec2"][1] = 0
    return out, inv


def test_filter_invalid_pairs_rules(oracle):
    rng = np.random.default_rng(11)
    for _ in range(5):
        x, off, pairs, pidx, regions = _random_case(rng)
        got, inv = oracle.filter_invalid_pairs(pairs, pidx, 1, x, off, np.zeros(len(x), np.uint32), regions)
        want, inv_w = _numpy_filter(pairs, pidx, x, off, regions)
        assert np.array_equal(inv, inv_w)
        assert got.tobytes() == want.tobytes()
        assert 0 < int(inv.sum()) < len(x)
        assert (got["vec2"][:, 1] == 0).sum() > (pairs["vec2"][:, 1] == 0).sum()
    # no EF pairs: nothing happens; no regions: only the invalid-vertex rule
    got, inv = oracle.filter_invalid_pairs(pairs, pidx, 0, x, off, np.zeros(len(x), np.uint32), regions)
    assert got.tobytes() == pairs.tobytes() and inv.sum() == 0
    got_nr, _ = oracle.filter_invalid_pairs(pairs, pidx, 1, x, off, np.zeros(len(x), np.uint32), None)
    got_r, _ = oracle.filter_invalid_pairs(pairs, pidx, 1, x, off, np.zeros(len(x), np.uint32), regions)
    assert (got_nr["vec2"][:, 1] == 0).sum() <= (got_r["vec2"][:, 1] == 0).sum()


def test_filter_broad_phase_rules(oracle):
    rng = np.random.default_rng(5)
    nv, ne, nf = 40, 50, 30
    faces = rng.integers(0, nv, (nf, 3)).astype(np.uint32)
    edges = rng.integers(0, nv, (ne, 2)).astype(np.uint32)
    inv = (rng.uniform(size=nv) < 0.1).astype(np.uint32)
    rows = lambda n: [sorted(set(rng.integers(0, 8, rng.integers(0, 3)).tolist())) for _ in range(n)]
    vr, er, fr = _csr(rows(nv)), _csr(rows(ne)), _csr(rows(nf))
    vf = np.stack([rng.integers(0, nv, 300), rng.integers(0, nf, 300)], 1).astype(np.uint32)
    ee = np.stack([rng.integers(0, ne, 300), rng.integers(0, ne, 300)], 1).astype(np.uint32)
    gvf, gee = oracle.filter_broad_phase(vf, ee, 3, inv, (vr, er, fr), faces, edges)
    m = lambda a, i, b, j: oracle.region_match(a, i, b, j)
    for (v, f), (gv, gf) in zip(vf, gvf):
        near = bool(inv[v] or inv[faces[f]].any())
        fl = (0x80000000 if m(vr, v, fr, f) == 1 else 0) | (0x40000000 if near else 0)
        assert (int(gv), int(gf)) == (int(v) | fl, int(f) | fl)
    for (a, b), (ga, gb) in zip(ee, gee):
        near = bool(inv[edges[a]].any() or inv[edges[b]].any())
        fl = (0x80000000 if m(er, a, er, b) == 1 else 0) | (0x40000000 if near else 0)
        assert (int(ga), int(gb)) == (int(a) | fl, int(b) | fl)
    assert (gvf[:, 0] >> 30).any() and (gee[:, 0] >> 31).any()
    # no EF pairs or no regions: lists untouched
    u, w = oracle.filter_broad_phase(vf, ee, 0, inv, (vr, er, fr), faces, edges)
    assert np.array_equal(u, vf) and np.array_equal(w, ee)
    u, w = oracle.filter_broad_phase(vf, ee, 3, inv, None, faces, edges)
    assert np.array_equal(u, vf) and np.array_equal(w, ee)
