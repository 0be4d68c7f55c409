"""Oracle restatement of the near-zero-distance proximity -> EF conversion
(fn_add_ef_from_proximity_pairs, intersection_resolver.cpp:199-363) and of the degenerate EF
filter (intersection_resolver.cpp:841-896), checked on the CPU against an independent numpy
restatement and against the filter's rule on modified EF lists."""
import numpy as np

from untangling26_b200 import synthetic
from untangling26_b200.prp import COLLISION_PAIR_DTYPE

BIT = 0x80000000


def contact_pairs(m, n, seed=0, extra=40):
    """Proximity templates of sheets_in_contact(n): VF pairs of sheet C's vertices onto the
    faces of A holding the coincident vertex (zero distance), EE pairs of C's edges with the
    coincident edges of A (zero distance), and seeded pairs at a distance (no conversion)."""
    rng = np.random.default_rng(seed)
    nn = n * n
    fa = m.faces[: len(m.faces) // 3]
    pairs, pidx = [], []
    for f_id, f in enumerate(fa[::7]):
        f_id *= 7
        for k in range(3):
            b = [(1.0, 0.0), (0.0, 1.0), (0.0, 0.0)][k]
            pairs.append(((f[k] + 2 * nn, f[0], f[1] | BIT, f[2]), b))
            pidx.append((f[k] + 2 * nn, f_id))
    ea = {tuple(e): i for i, e in enumerate(m.edges) if e[1] < nn}
    ec = [(i, e) for i, e in enumerate(m.edges) if e[0] >= 2 * nn]
    for i, e in ec[::5]:
        j = ea[(e[0] - 2 * nn, e[1] - 2 * nn)]
        b0, b1 = m.edges[j]
        pairs.append(((e[0], e[1], b0, b1 | BIT), (1.0, 1.0)))
        pidx.append((i, j))
    for _ in range(extra):  # far pairs: sheet B vertices onto A faces with random barycentres
        v = int(rng.integers(nn, 2 * nn))
        f_id = int(rng.integers(0, len(fa)))
        f = fa[f_id]
        pairs.append(((v, f[0], f[1] | BIT, f[2]), (rng.uniform(0, 0.5), rng.uniform(0, 0.5))))
        pidx.append((v, f_id))
    out = np.zeros(len(pairs), COLLISION_PAIR_DTYPE)
    for i, (idx, b) in enumerate(pairs):
        out[i]["indices"] = idx
        out[i]["vec2"] = (0, 0, b[0], b[1])
    return out, np.array(pidx, np.uint32)


def _numpy_convert(m, pairs, pidx):
    vae, eaf = m.vert_adj_edges, m.edge_adj_faces_ext
    out = []
    for p, (s, d) in zip(pairs, pidx):
        raw = [int(v) for v in p["indices"]]
        t = (raw[0] >> 31) + ((raw[1] >> 31) << 1) + ((raw[2] >> 31) << 2) + ((raw[3] >> 31) << 3)
        ids = [v & 0x7FFFFFFF for v in raw]
        b2, b3 = np.float32(p["vec2"][2]), np.float32(p["vec2"][3])
        one = np.float32(1)
        w = (one, -b2, -b3, (b2 + b3) - one) if t == 4 else (b2, one - b2, -b3, b3 - one)
        d3 = np.zeros(3, np.float32)
        for k in range(4):
            d3 = (d3 + np.float32(w[k]) * m.x[ids[k]]).astype(np.float32)
        if np.float32(np.float32(d3[0] * d3[0] + d3[1] * d3[1]) + d3[2] * d3[2]) >= np.float32(1e-10):
            continue
        if t == 4:
            f = m.faces[d]
            for ae in vae.row(ids[0]):
                e = m.edges[ae]
                out.append((int(ae), int(d), (int(e[0]), int(e[1]), *map(int, f)), (1.0 if e[0] == ids[0] else 0.0, abs(w[1]), abs(w[2]))))
        else:
            e1, e2 = m.edges[s], m.edges[d]
            for at, other, on, emit_e, emit_id, eb in ((d, e1, e2, e1, s, abs(w[0])), (s, e2, e1, e2, d, abs(w[2]))):
                for g in eaf.row(at):
                    fv = m.faces[g]
                    if set(fv.tolist()) & set(other.tolist()):
                        continue
                    fb = [0.0, 0.0, 0.0]
                    cnt = 0
                    for c in range(3):
                        if fv[c] == on[0]:
                            fb[c], cnt = abs(w[0]), cnt + 1
                        elif fv[c] == on[1]:
                            fb[c], cnt = abs(w[1]), cnt + 1
                    if cnt == 2:
                        out.append((int(emit_id), int(g), (int(emit_e[0]), int(emit_e[1]), *map(int, fv)), (eb, fb[0], fb[1])))
    return sorted((a, b, idx, tuple(np.float32(v) for v in bary)) for a, b, idx, bary in out)


def test_proximity_conversion_rules(oracle):
    m = synthetic.sheets_in_contact(10, seed=0)
    pairs, pidx = contact_pairs(m, 10)
    vae = m.vert_adj_edges.one_array()
    eaf = m.edge_adj_faces_ext.one_array()
    ef, idx = oracle.ef_from_proximity(pairs, pidx, m.x, m.edges, m.faces, vae, eaf)
    got = sorted((int(i[0]), int(i[1]), tuple(int(v) for v in e["idx"]), tuple(np.float32(v) for v in e["bary"])) for e, i in zip(ef, idx))
    want = _numpy_convert(m, pairs, pidx)
    assert len(got) == len(want) > 0
    assert got == want
    assert np.all(ef["stiff"] == 0) and np.all(ef["grad"] == 0)
    # duplicates exist (an edge of C reached from both of its vertices): the canonical order breaks ties on the payload
    keys = [tuple(i) for i in idx.tolist()]
    assert len(set(keys)) < len(keys)
    cp, ci = oracle.canonical_ef(ef, idx)
    assert all(tuple(a) <= tuple(b) for a, b in zip(ci[:-1].tolist(), ci[1:].tolist()))


def test_degenerate_filter_rule(oracle):
    """With ignore_near_zero_dist_pairs off, a contour made wholly degenerate disappears,
    one degenerate pair inside a regular contour stays."""
    m = synthetic.folded_sheet(40, seed=2)
    ef, idx = oracle.detect_ef(m)
    base = oracle.PrpRun(m, ef, idx, oracle.prp_params(max_contours=64))
    assert len(base.contours) >= 2
    n = base.num_orig_pairs
    sizes = [len([p for p in c if p < n]) for c in base.contours]
    c_all = int(np.argmin(sizes))
    c_one = int(np.argmax(sizes))
    mod = ef.copy()
    for p in base.contours[c_all]:
        if p < n:
            mod[p]["bary"][1] = 1e-5  # a face barycentre below 1e-4
    mod[[p for p in base.contours[c_one] if p < n][0]]["bary"][0] = 0.99995  # edge barycentre 1 - 5e-5
    keep = oracle.PrpRun(m, mod, idx, oracle.prp_params(max_contours=64, ignore_near_zero_dist_pairs=1))
    drop = oracle.PrpRun(m, mod, idx, oracle.prp_params(max_contours=64, ignore_near_zero_dist_pairs=0))
    assert keep.num_orig_pairs == n
    assert drop.num_orig_pairs == n - sizes[c_all]
    assert len(drop.contours) == len(base.contours) - 1
