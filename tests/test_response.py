"""Oracle restatement of the response assembly (make_response_from_min_hitinfo,
intersection_resolver2.cpp:2105-2221) and the region labels (host_apply_untangling_constraint,
2296-2427), checked on the CPU against the reference's own golden values and against an
independent numpy restatement of the same rules."""
import numpy as np

from untangling26_b200 import synthetic
from untangling26_b200.prp import PrpResponse


def test_region_label_packing_goldens(oracle):
    # the reference's static_asserts (intersection_resolver2.cpp:135-140):
    # pack(contour 3, mesh 1, label 5) unpacks to visual region 3 * 256 + 5 and semantic region 2 * 3 + 1
    p = oracle.region_pack(3, 5, 1)
    assert p >> 1 == 3 * 256 + 5
    assert oracle.region_semantic(p) == 7
    assert oracle.region_pack(0, 4, 0) == 8


def test_solution_key_signs(oracle):
    z = [0.0, 0.0, 1.0]
    assert oracle.solution_key([0, 0, 1], [0, 0, -1], z) == 3 * 2 + 0
    assert oracle.solution_key([0, 0, 0], [0, 0, 0], z) == 4  # the (0, 0) default
    # |q| <= 0.1 counts as no sign; just above it does
    assert oracle.solution_key([np.sqrt(1 - 0.01), 0, 0.1], [0, 0, 1], z) == 3 * 1 + 2
    assert oracle.solution_key([0.99, 0, 0.11], [0, 0, 1], z) == 3 * 2 + 2
    # a zero direction gives no projections
    assert oracle.solution_key([0, 0, 1], [0, 0, 1], [0, 0, 0]) == 4
    assert oracle.solution_key([0, 0, 1], [0, 0, 1], [float("nan"), 0, 0]) == 4


def _check_rows_sorted(arr, n):
    rows = PrpResponse.csr_rows(arr)
    assert len(rows) == n
    assert arr[0] == n + 1 and arr[n] == len(arr)
    for r in rows:
        assert np.all(np.diff(r.astype(np.int64)) > 0)
    return rows


def test_response_rules_two_sheets(oracle):
    m = synthetic.two_sheets(24, seed=0)
    ef, idx = oracle.detect_ef(m)
    depth_thr, stiff = 2e-3, 3e7
    ref = oracle.PrpRun(m, ef, idx, oracle.prp_params(), response=(depth_thr, stiff))
    pairs, info = ref.response_pairs, ref.response_info
    hits = [(c, h) for c in range(len(ref.hits)) for h in ref.hits[c]]
    assert len(pairs) == len(hits) > 0
    va, ea, fa = m.rest_vert_area, m.rest_edge_area, m.rest_face_area
    for (c, h), p, inf in zip(hits, pairs, info):
        r = ref.results[c]
        d = np.asarray(r["dir"], np.float32)
        C = np.float32(max(np.float32(-r["depth"]) - np.float32(3e-3), np.float32(-depth_thr)))
        t = int(h["type"])
        if t == 0:
            a = (va[h["src_id"]], fa[h["dst_id"]])
            idx4 = [h["sv"][0], h["dv"][0], h["dv"][1] | 0x80000000, h["dv"][2]]
            want_info = [h["src_id"], h["dst_id"], 0]
            normal = d
        elif t == 2:
            a = (fa[h["src_id"]], va[h["dst_id"]])
            idx4 = [h["dv"][0], h["sv"][0], h["sv"][1] | 0x80000000, h["sv"][2]]
            want_info = [h["dst_id"], h["src_id"], 1]
            normal = -d
        else:
            a = (ea[h["src_id"]], ea[h["dst_id"]])
            idx4 = [h["sv"][0], h["sv"][1], h["dv"][0], h["dv"][1] | 0x80000000]
            want_info = [h["src_id"], h["dst_id"], 2]
            normal = d
        area = np.float32(max(np.float32(0.5) * (np.float32(a[0]) + np.float32(a[1])), np.float32(3e-6)))
        k2 = np.float32(area * np.float32(stiff))
        assert list(p["indices"]) == [int(v) for v in idx4]
        assert p["vec1"][3] == area and p["vec2"][1] == k2 and p["vec2"][0] == np.float32(k2 * C)
        assert np.array_equal(p["vec1"][:3], normal.astype(np.float32))
        assert np.array_equal(p["vec2"][2:], h["bary"]) and np.all(p["vec3"] == 0)
        assert [int(inf[0]), int(inf[1]), int(inf[3])] == want_info
        assert (int(inf[2]) >> 1) // 256 == c and int(inf[2]) & 1 == 0
    # region CSRs: rebuild the vertex rows from the rules, then edges / faces as unions
    vr = [set() for _ in range(m.num_verts)]
    for p, inf in zip(pairs, info):
        s = 2 * ((int(inf[2]) >> 1) // 256)
        lab = {0: (s, s ^ 1, s ^ 1, s ^ 1), 1: (s ^ 1, s, s, s), 2: (s, s, s ^ 1, s ^ 1)}[int(inf[3])]
        for v, l in zip(p["indices"] & 0x7FFFFFFF, lab):
            vr[int(v)].add(l)
    for (e, f), mi, ci in zip(ref.pair_indices, ref.mesh_index, ref.contour_index):
        er = 2 * int(ci) + int(mi)
        for v in m.edges[e]:
            vr[int(v)].add(er)
        for v in m.faces[f]:
            vr[int(v)].add(er ^ 1)
    rows = _check_rows_sorted(ref.vert_regions, m.num_verts)
    assert all(set(r.tolist()) == vr[i] for i, r in enumerate(rows))
    erows = _check_rows_sorted(ref.edge_regions, m.num_edges)
    for e, r in enumerate(erows):
        assert set(r.tolist()) == vr[m.edges[e][0]] | vr[m.edges[e][1]]
    frows = _check_rows_sorted(ref.face_regions, m.num_faces)
    for f, r in enumerate(frows):
        assert set(r.tolist()) == set().union(*(vr[int(v)] for v in m.faces[f]))


def _pair(idx, n, k1, k2, a, b):
    p = np.zeros(1, oracle_dtype())
    p["indices"][0] = idx
    p["vec1"][0, :3] = n
    p["vec2"][0] = (k1, k2, a, b)
    return p


def oracle_dtype():
    from oracle.oracle import COLLISION_PAIR_DTYPE
    return COLLISION_PAIR_DTYPE


def test_response_step_rules(oracle):
    """The repair loop's step: a VF pair moves its vertex by +Delta/2 n and its face's vertices by
    -Delta/2 n (Delta = -k1 / k2); vertices shared by several pairs take the weighted mean;
    pairs with k2 <= 0 or weights <= 0 move nothing."""
    tb = 0x80000000
    x = np.zeros((6, 3), np.float32)
    vf = _pair([0, 1, 2 | tb, 3], [0, 0, 1], -4e-3, 1.0, 0.5, 0.25)  # Delta = 4e-3
    out, moved = oracle.response_step(vf, x)
    assert moved == 4
    assert np.allclose(out[0], [0, 0, 2e-3]) and np.allclose(out[1:4], [[0, 0, -2e-3]] * 3)
    assert not out[4:].any()
    # an EE pair with edge parameter 1 on its first edge: its second vertex has weight 0
    ee = _pair([4, 5, 1, 3 | tb], [1, 0, 0], -2e-3, 1.0, 1.0, 0.5)
    out, moved = oracle.response_step(np.concatenate([vf, ee]), x)
    assert moved == 5  # vertex 5 has weight 0
    assert np.allclose(out[4], [1e-3, 0, 0])
    # vertex 1: -2e-3 z (VF, weight 0.5) and -1e-3 x (EE, weight 0.5): the mean of the two
    assert np.allclose(out[1], [-0.5e-3, 0, -1e-3])
    dead = _pair([0, 1, 2 | tb, 3], [0, 0, 1], -4e-3, 0.0, 0.5, 0.25)
    out, moved = oracle.response_step(dead, x)
    assert moved == 0 and not out.any()
    # scale multiplies the step; the fixed-point sums do not depend on the pairs' order
    both = np.concatenate([vf, ee])
    a, _ = oracle.response_step(both, x + 0.1, 0.5)
    b, _ = oracle.response_step(both[::-1].copy(), x + 0.1, 0.5)
    assert a.tobytes() == b.tobytes()
    assert np.allclose(a[4], [0.1 + 0.5e-3, 0.1, 0.1])
