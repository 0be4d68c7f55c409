"""Test infrastructure: ctypes wrappers over the CPU oracle (``oracle/_build/liboracle.so``).

The oracle is the checker for the CUDA path, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of ``bench.py`` import this
module. Each wrapped function names the reference source it restates in the C++ file.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_f32p = ctypes.POINTER(ctypes.c_float)


def build():
    """Compile the oracle (make in oracle/)."""
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _lib.oracle_morton32.restype = ctypes.c_uint32
        _lib.oracle_morton32.argtypes = [ctypes.c_float] * 3
        _lib.oracle_morton64.restype = ctypes.c_uint64
        _lib.oracle_morton64.argtypes = [ctypes.c_float] * 3 + [ctypes.c_uint32]
        _lib.oracle_lbvh_build.restype = ctypes.c_int
        _lib.oracle_lbvh_query.restype = ctypes.c_uint64
        _lib.oracle_ef_narrow.restype = ctypes.c_uint32
        _lib.oracle_find_split.restype = ctypes.c_int
        _lib.oracle_threads_used.restype = ctypes.c_int
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def _pn(a, t):
    return None if a is None else _p(a, t)


TREE_VERT, TREE_FACE, TREE_EDGE = 0, 1, 2


def threads():
    return lib().oracle_threads_used()


def morton32(p):
    return lib().oracle_morton32(*[ctypes.c_float(v) for v in p])


def morton64(p, idx):
    return lib().oracle_morton64(*[ctypes.c_float(v) for v in p], ctypes.c_uint32(idx))


def determine_range(keys, i):
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    out = np.zeros(2, np.int32)
    lib().oracle_determine_range(_p(keys, _u64p), ctypes.c_uint32(len(keys)), ctypes.c_uint32(i), out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    return int(out[0]), int(out[1])


def find_split(keys, i, j):
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    return lib().oracle_find_split(_p(keys, _u64p), ctypes.c_int(i), ctypes.c_int(j))


def karras(keys_sorted):
    keys_sorted = np.ascontiguousarray(keys_sorted, dtype=np.uint64)
    n = len(keys_sorted)
    parent = np.full(2 * n - 1, 0xFFFFFFFF, np.uint32)
    children = np.zeros((2 * n - 1, 2), np.uint32)
    lib().oracle_lbvh_karras(_p(keys_sorted, _u64p), ctypes.c_uint32(n), _p(parent, _u32p), _p(children, _u32p))
    return parent, children


class OracleTree:
    """Arrays of one built tree (lbvh.h:77-150 layout, node AABBs as float[8])."""

    def __init__(self, tree_type, n):
        self.tree_type = tree_type
        self.n = n
        nn = max(2 * n - 1, 1)
        self.gaabb = np.zeros(6, np.float32)
        self.keys_sorted = np.zeros(max(n, 1), np.uint64)
        self.sorted_get_original = np.zeros(max(n, 1), np.uint32)
        self.parent = np.full(nn, 0xFFFFFFFF, np.uint32)
        self.children = np.zeros((nn, 2), np.uint32)
        self.object_idx = np.full(nn, 0xFFFFFFFF, np.uint32)
        self.node_aabb = np.zeros((nn, 8), np.float32)
        self.unhealthy = 0


def lbvh_build(tree_type, x, prims, num_verts=None):
    x = np.ascontiguousarray(x, dtype=np.float32)
    nv = x.shape[0] if num_verts is None else num_verts
    if tree_type == TREE_VERT:
        n = nv
        prims_p = None
    else:
        prims = np.ascontiguousarray(prims, dtype=np.uint32)
        n = prims.shape[0]
        prims_p = _p(prims, _u32p)
    t = OracleTree(tree_type, n)
    t.unhealthy = lib().oracle_lbvh_build(
        ctypes.c_int(tree_type), _p(x, _f32p), ctypes.c_uint32(nv), prims_p, ctypes.c_uint32(n),
        _p(t.gaabb, _f32p), _p(t.keys_sorted, _u64p), _p(t.sorted_get_original, _u32p),
        _p(t.parent, _u32p), _p(t.children, _u32p), _p(t.object_idx, _u32p))
    return t


def lbvh_refit(tree, x0, x1, thickness, prims):
    x0 = np.ascontiguousarray(x0, dtype=np.float32)
    x1 = np.ascontiguousarray(x1, dtype=np.float32)
    thickness = np.ascontiguousarray(thickness, dtype=np.float32)
    prims_p = None if prims is None else _p(np.ascontiguousarray(prims, dtype=np.uint32), _u32p)
    if prims is not None:
        prims = np.ascontiguousarray(prims, dtype=np.uint32)
        prims_p = _p(prims, _u32p)
    lib().oracle_lbvh_refit(
        ctypes.c_int(tree.tree_type), ctypes.c_uint32(tree.n), _p(x0, _f32p), _p(x1, _f32p), _p(thickness, _f32p),
        prims_p, _p(tree.sorted_get_original, _u32p), _p(tree.children, _u32p), _p(tree.node_aabb, _f32p))
    return tree.node_aabb


QUERY_VERTS, QUERY_EDGES, QUERY_EDGES_UNCULLED = 0, 1, 2


def lbvh_query(tree, mode, x0, x1, edges, d_hat, thickness, max_pairs=None):
    """Broad phase (lbvh.cpp:295-363, 780-894). Returns (pairs[k,2], total, overflow)."""
    x0 = np.ascontiguousarray(x0, dtype=np.float32)
    x1 = np.ascontiguousarray(x1, dtype=np.float32)
    d_hat = np.ascontiguousarray(d_hat, dtype=np.float32)
    thickness = np.ascontiguousarray(thickness, dtype=np.float32)
    if mode == QUERY_VERTS:
        nq = x0.shape[0]
        edges_p = None
    else:
        edges = np.ascontiguousarray(edges, dtype=np.uint32)
        nq = edges.shape[0]
        edges_p = _p(edges, _u32p)
    if max_pairs is None:
        max_pairs = 1 << 20
    while True:
        pairs = np.zeros((max(max_pairs, 1), 2), np.uint32)
        overflow = np.zeros(1, np.uint32)
        total = lib().oracle_lbvh_query(
            ctypes.c_int(mode), ctypes.c_uint32(nq), _p(x0, _f32p), _p(x1, _f32p), edges_p,
            _p(d_hat, _f32p), _p(thickness, _f32p), ctypes.c_uint32(tree.n), _p(tree.children, _u32p),
            _p(tree.object_idx, _u32p), _p(tree.node_aabb, _f32p), _p(pairs, _u32p), ctypes.c_uint64(max_pairs),
            _p(overflow, _u32p))
        if total <= max_pairs:
            return pairs[:total], int(total), int(overflow[0])
        max_pairs = int(total)


EF_PAIR_DTYPE = np.dtype([("idx", np.uint32, 5), ("bary", np.float32, 3), ("grad", np.float32, 3), ("stiff", np.float32)])
# CollisionPair::CollisionPairTemplate (collision_data.h:48-140): 64 B
COLLISION_PAIR_DTYPE = np.dtype([("indices", np.uint32, 4), ("vec1", np.float32, 4), ("vec2", np.float32, 4), ("vec3", np.float32, 4)])
assert EF_PAIR_DTYPE.itemsize == 48


def ef_narrow(broad_pairs, x, edges, faces, d_hat, vprop=None):
    """EF narrow phase (intersection_resolver.cpp:86-197), canonical order."""
    broad_pairs = np.ascontiguousarray(broad_pairs, dtype=np.uint32).reshape(-1, 2)
    x = np.ascontiguousarray(x, dtype=np.float32)
    edges = np.ascontiguousarray(edges, dtype=np.uint32)
    faces = np.ascontiguousarray(faces, dtype=np.uint32)
    d_hat = np.ascontiguousarray(d_hat, dtype=np.float32)
    vp = None if vprop is None else np.ascontiguousarray(vprop, dtype=np.uint32)
    nb = broad_pairs.shape[0]
    out = np.zeros(max(nb, 1), EF_PAIR_DTYPE)
    idx = np.zeros((max(nb, 1), 2), np.uint32)
    cnt = lib().oracle_ef_narrow(
        _p(broad_pairs, _u32p), ctypes.c_uint32(nb), _p(x, _f32p), _p(edges, _u32p), _p(faces, _u32p),
        _pn(vp, _u32p), _p(d_hat, _f32p), out.ctypes.data_as(ctypes.c_void_p), _p(idx, _u32p), ctypes.c_uint32(nb))
    return out[:cnt], idx[:cnt]


def ef_recheck(broad_pairs, x, edges, faces, d_hat, vprop=None):
    """FP64 recheck counts of the EF tests over broad-phase pairs: (rechecked, flipped)."""
    broad_pairs = np.ascontiguousarray(broad_pairs, dtype=np.uint32).reshape(-1, 2)
    arrs = [np.ascontiguousarray(a, t) for a, t in ((x, np.float32), (edges, np.uint32), (faces, np.uint32), (d_hat, np.float32))]
    vp = None if vprop is None else np.ascontiguousarray(vprop, dtype=np.uint32)
    out = np.zeros(2, np.uint64)
    lib().oracle_ef_recheck(_p(broad_pairs, _u32p), ctypes.c_uint32(len(broad_pairs)), _p(arrs[0], _f32p), _p(arrs[1], _u32p),
                            _p(arrs[2], _u32p), _pn(vp, _u32p), _p(arrs[3], _f32p), _p(out, _u64p))
    return int(out[0]), int(out[1])


def line_intersection(p0, p1, a, b, c):
    arrs = [np.ascontiguousarray(v, dtype=np.float32) for v in (p0, p1, a, b, c)]
    bary = np.zeros(3, np.float32)
    t = ctypes.c_float(0)
    hit = lib().oracle_line_intersection(*[_p(v, _f32p) for v in arrs], _p(bary, _f32p), ctypes.byref(t))
    return bool(hit), bary, t.value


# ---- PRP contour evaluation (oracle_prp.cpp) -------------------------------------
class PrpParams(ctypes.Structure):
    """Parameters of one PRP pass (SceneParams fields, scene_params.h:65-81)."""
    _fields_ = [
        ("max_contours", ctypes.c_uint32),      # untangling_process_contours_count
        ("direction_mode", ctypes.c_uint32),    # 0 reference seeds, 1 the 26 lattice directions
        ("use_ccr", ctypes.c_uint32),           # PRP_use_intrinsic_contour_side_candidates
        ("ccr_tau", ctypes.c_float),            # PRP_intrinsic_tau
        ("ccr_use_rest", ctypes.c_uint32),      # PRP_use_rest_geodesic_distance_for_intrinsic_candidates
        ("ccr_use_current", ctypes.c_uint32),   # PRP_use_deformed_boundary_distance_for_intrinsic_candidates
        ("batch_size", ctypes.c_uint32),        # PRP_cpu_contour_batch_size
        ("brute_force_raycast", ctypes.c_uint32),
        ("contour_stride", ctypes.c_uint32),    # timing sample: contours c with c % stride == 0 only
        ("opt_iterations", ctypes.c_uint32),    # PRP_direction_optimization_iterations
        ("ccr_blend", ctypes.c_uint32),         # PRP_use_blended_intrinsic_coordinates
        ("ccr_blend_weight", ctypes.c_float),   # PRP_intrinsic_blend_weight
        ("solid_interior", ctypes.c_uint32),    # PRP_solid_interior_adjacency
        ("solid_all", ctypes.c_uint32),         # PRP_solid_interior_adjacency_all_meshes
        ("solid_eps_n", ctypes.c_float),        # PRP_solid_interior_adjacency_normal_eps
        ("solid_eps_d", ctypes.c_float),        # PRP_solid_interior_adjacency_dist_eps
        ("ignore_near_zero_dist_pairs", ctypes.c_uint32),  # scene_params.h:55
        ("contour_offset", ctypes.c_uint32),    # with contour_stride: contours c with c % stride == offset % stride
        ("fp64_recheck", ctypes.c_uint32),      # count the FP64 rechecks of the leaf tests inside their FP32 error band
    ]


def prp_params(**kw):
    p = PrpParams(max_contours=256, direction_mode=0, use_ccr=1, ccr_tau=0.25, ccr_use_rest=1, ccr_use_current=1,
                  batch_size=32, brute_force_raycast=0, contour_stride=0, opt_iterations=0, ccr_blend=0,
                  ccr_blend_weight=0.5, solid_interior=1, solid_all=0, solid_eps_n=1e-4, solid_eps_d=1e-5,
                  ignore_near_zero_dist_pairs=1, contour_offset=0, fp64_recheck=0)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


RESULT_DTYPE = np.dtype([
    ("contour_idx", np.uint32), ("contour_type", np.uint32), ("num_pairs", np.uint32), ("combo_idx", np.uint32),
    ("num_dirs", np.uint32), ("hit_count", np.uint32), ("unculled_hit_count", np.uint32), ("covered_anchor_count", np.uint32),
    ("boundary_anchor_count", np.uint32), ("eval_k_src", np.uint32), ("eval_k_dst", np.uint32),
    ("max_frontier_hop_src", np.uint32), ("max_frontier_hop_dst", np.uint32), ("expansion_level_count", np.uint32),
    ("flags", np.uint32), ("object_id0", np.uint32), ("object_id1", np.uint32), ("init_k_src", np.uint32),
    ("init_k_dst", np.uint32), ("diam_src", np.uint32), ("diam_dst", np.uint32), ("num_boundary_src", np.uint32),
    ("num_boundary_dst", np.uint32), ("opt_attempted", np.uint32),
    ("dir", np.float32, 3), ("depth", np.float32), ("volume", np.float32), ("objective", np.float32),
    ("area", np.float32), ("displacement_cost", np.float32), ("coverage", np.float32),
    ("normalized_objective", np.float32), ("pre_finalize_area", np.float32), ("opt_accepted", np.uint32)])
HIT_DTYPE = np.dtype([("type", np.uint32), ("src_id", np.uint32), ("dst_id", np.uint32), ("sv", np.uint32, 3),
                      ("dv", np.uint32, 3), ("bary", np.float32, 2), ("dist", np.float32)])
assert RESULT_DTYPE.itemsize == 144 and HIT_DTYPE.itemsize == 48


class PrpRun:
    """All outputs of one oracle PRP pass."""

    def __init__(self, mesh, ef_pairs, ef_indices, params=None, x=None, response=None, order_spread=0):
        """response: (depth_threshold, stiffness) to also assemble the response pairs and the
        vertex / edge / face region CSRs (attributes response_pairs, response_info,
        vert_regions, edge_regions, face_regions). order_spread = k > 0: per contour, the largest
        relative difference of the selected support's FP32 area, volume, cost and J between the
        canonical summation order and the reference's block reduce over the hits in key order
        and k seeded shuffles (attribute order_spread)."""
        L = lib()
        L.oracle_prp_run.restype = ctypes.c_void_p
        for n in ("oracle_prp_num_pairs", "oracle_prp_num_orig_pairs", "oracle_prp_num_contours", "oracle_prp_contour",
                  "oracle_prp_hits", "oracle_prp_directions"):
            getattr(L, n).restype = ctypes.c_uint32
        params = params or prp_params()
        desc = mesh.desc(x)
        ef_pairs = np.ascontiguousarray(ef_pairs)
        ef_indices = np.ascontiguousarray(ef_indices, dtype=np.uint32)
        h = ctypes.c_void_p(L.oracle_prp_run(ctypes.byref(desc), ef_pairs.ctypes.data_as(ctypes.c_void_p),
                                             _p(ef_indices, _u32p), ctypes.c_uint32(len(ef_pairs)), ctypes.byref(params)))
        try:
            n = L.oracle_prp_num_pairs(h)
            self.num_orig_pairs = L.oracle_prp_num_orig_pairs(h)
            self.pairs = np.zeros(max(n, 1), EF_PAIR_DTYPE)
            self.pair_indices = np.zeros((max(n, 1), 2), np.uint32)
            self.mesh_index = np.zeros(max(n, 1), np.uint32)
            self.contour_index = np.zeros(max(n, 1), np.uint32)
            self.pair_length = np.zeros(max(n, 1), np.float32)
            L.oracle_prp_pairs(h, self.pairs.ctypes.data_as(ctypes.c_void_p), _p(self.pair_indices, _u32p),
                               _p(self.mesh_index, _u32p), _p(self.contour_index, _u32p), _p(self.pair_length, _f32p))
            self.pairs, self.pair_indices = self.pairs[:n], self.pair_indices[:n]
            self.mesh_index, self.contour_index, self.pair_length = self.mesh_index[:n], self.contour_index[:n], self.pair_length[:n]
            nc = L.oracle_prp_num_contours(h)
            self.contours = []
            self.results = np.zeros(nc, RESULT_DTYPE)
            self.hits = []
            self.directions = []
            for c in range(nc):
                k = L.oracle_prp_contour(h, ctypes.c_uint32(c), None)
                buf = np.zeros(max(k, 1), np.uint32)
                L.oracle_prp_contour(h, ctypes.c_uint32(c), _p(buf, _u32p))
                self.contours.append(buf[:k])
                L.oracle_prp_result(h, ctypes.c_uint32(c), self.results[c:c + 1].ctypes.data_as(ctypes.c_void_p))
                nh = L.oracle_prp_hits(h, ctypes.c_uint32(c), None)
                hb = np.zeros(max(nh, 1), HIT_DTYPE)
                L.oracle_prp_hits(h, ctypes.c_uint32(c), hb.ctypes.data_as(ctypes.c_void_p))
                self.hits.append(hb[:nh])
                if self.results[c]["flags"] & 16:
                    nd = L.oracle_prp_directions(h, ctypes.c_uint32(c), None)
                    db = np.zeros((max(nd, 1), 3), np.float32)
                    L.oracle_prp_directions(h, ctypes.c_uint32(c), _p(db, _f32p))
                    self.directions.append(db[:nd])
                else:
                    self.directions.append(np.zeros((0, 3), np.float32))
            st = np.zeros(3, np.uint64)
            L.oracle_prp_stats(h, _p(st, _u64p))
            self.tested, self.requests, self.pairs_tested = int(st[0]), int(st[1]), int(st[2])
            rc = np.zeros(2, np.uint64)
            L.oracle_prp_recheck(h, _p(rc, _u64p))
            # FP64: per contour (J, D_C, max relative depth error, D_C tie, tie flip)
            f64 = np.zeros((max(nc, 1), 5), np.float64)
            L.oracle_prp_fp64(h, f64.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
            self.fp64_contours = f64[:nc]
            with np.errstate(divide="ignore", invalid="ignore"):
                has = f64[:nc, 1] > 0
                j32 = self.results["objective"].astype(np.float64)
                d32 = self.results["depth"].astype(np.float64)
                jerr = np.abs(j32 - f64[:nc, 0]) / f64[:nc, 0]
                derr = np.abs(d32 - f64[:nc, 1]) / f64[:nc, 1]
            self.order_spread = None
            if order_spread:
                self.order_spread = np.zeros(max(nc, 1), np.float64)
                L.oracle_prp_order_spread(h, ctypes.c_uint32(order_spread), ctypes.c_uint32(1),
                                          self.order_spread.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
                self.order_spread = self.order_spread[:nc]
            self.fp64 = {"rechecks": int(rc[0]), "flips": int(rc[1]), "dc_tie_rechecks": int(f64[:nc, 3].sum()),
                         "dc_tie_flips": int(f64[:nc, 4].sum()),
                         "delta_rel_err": float(f64[:nc, 2].max()) if nc else 0.0,
                         "dc_rel_err": float(derr[has].max()) if has.any() else 0.0,
                         "j_rel_err": float(jerr[(f64[:nc, 0] > 0)].max()) if (f64[:nc, 0] > 0).any() else 0.0}
            if response is not None:
                L.oracle_prp_response.restype = ctypes.c_uint32
                dt, k = ctypes.c_float(response[0]), ctypes.c_float(response[1])
                lens = np.zeros(3, np.uint32)
                npairs = L.oracle_prp_response(h, dt, k, None, None, None, None, None, _p(lens, _u32p))
                self.response_pairs = np.zeros(max(npairs, 1), COLLISION_PAIR_DTYPE)
                self.response_info = np.zeros((max(npairs, 1), 4), np.uint32)
                self.vert_regions = np.zeros(lens[0], np.uint32)
                self.edge_regions = np.zeros(lens[1], np.uint32)
                self.face_regions = np.zeros(lens[2], np.uint32)
                L.oracle_prp_response(h, dt, k, self.response_pairs.ctypes.data_as(ctypes.c_void_p), _p(self.response_info, _u32p),
                                      _p(self.vert_regions, _u32p), _p(self.edge_regions, _u32p), _p(self.face_regions, _u32p), None)
                self.response_pairs, self.response_info = self.response_pairs[:npairs], self.response_info[:npairs]
        finally:
            L.oracle_prp_free(h)


def region_pack(contour, key, mesh):
    L = lib()
    L.oracle_region_pack.restype = ctypes.c_uint32
    return int(L.oracle_region_pack(ctypes.c_uint32(contour), ctypes.c_uint32(key), ctypes.c_uint32(mesh)))


def region_semantic(packed):
    L = lib()
    L.oracle_region_semantic.restype = ctypes.c_uint32
    return int(L.oracle_region_semantic(ctypes.c_uint32(packed)))


def solution_key(n_src, n_dst, r):
    L = lib()
    L.oracle_solution_key.restype = ctypes.c_uint32
    a, b, c = (np.ascontiguousarray(v, np.float32) for v in (n_src, n_dst, r))
    return int(L.oracle_solution_key(_p(a, _f32p), _p(b, _f32p), _p(c, _f32p)))


def region_match(lcsr, l, rcsr, r):
    """fn_is_matched_invalid_region of rows l (of lcsr) and r (of rcsr): 0 / 1 / 2."""
    L = lib()
    L.oracle_region_match.restype = ctypes.c_uint32
    a = np.ascontiguousarray(lcsr, np.uint32)
    b = np.ascontiguousarray(rcsr, np.uint32)
    return int(L.oracle_region_match(_p(a, _u32p), ctypes.c_uint32(l), _p(b, _u32p), ctypes.c_uint32(r)))


def filter_invalid_pairs(pairs, pair_indices, num_ef, x, offset, invalid, regions=None):
    """IntersectionResolver::filter_invalid_pairs over the proximity pairs; returns the
    filtered (pairs, invalid) copies. regions: (vert, edge, face) CSR arrays or None."""
    L = lib()
    pairs = np.ascontiguousarray(pairs).copy()
    pidx = np.ascontiguousarray(pair_indices, np.uint32)
    x = np.ascontiguousarray(x, np.float32)
    off = np.ascontiguousarray(offset, np.float32)
    inv = np.ascontiguousarray(invalid, np.uint32).copy()
    rg = [None, None, None] if regions is None else [np.ascontiguousarray(a, np.uint32) for a in regions]
    L.oracle_filter_invalid_pairs(pairs.ctypes.data_as(ctypes.c_void_p), _p(pidx, _u32p), ctypes.c_uint32(len(pairs)),
                                  ctypes.c_uint32(num_ef), _p(x, _f32p), _p(off, _f32p), ctypes.c_uint32(len(inv)), _p(inv, _u32p),
                                  *[(_p(a, _u32p) if a is not None else None) for a in rg])
    return pairs, inv


def csr_one_array(offsets, data):
    """upload_2d_csr_from's layout (buffer_allocator.h:26-59): [n + 1] absolute offsets, then the data."""
    off = np.asarray(offsets, np.int64)
    n = len(off) - 1
    return np.concatenate([off - off[0] + n + 1, np.asarray(data, np.int64)]).astype(np.uint32)


def ef_from_proximity(pairs, pair_indices, x, edges, faces, vae_csr, eaf_csr):
    """fn_add_ef_from_proximity_pairs over all given proximity pairs, in pair order."""
    L = lib()
    L.oracle_ef_from_proximity.restype = ctypes.c_uint32
    pairs = np.ascontiguousarray(pairs)
    pidx = np.ascontiguousarray(pair_indices, np.uint32)
    arrs = [np.ascontiguousarray(a, t) for a, t in ((x, np.float32), (edges, np.uint32), (faces, np.uint32), (vae_csr, np.uint32),
                                                    (eaf_csr, np.uint32))]
    args = lambda out, idx, cap: (pairs.ctypes.data_as(ctypes.c_void_p), _p(pidx, _u32p), ctypes.c_uint32(len(pairs)),
                                  _p(arrs[0], _f32p), _p(arrs[1], _u32p), _p(arrs[2], _u32p), _p(arrs[3], _u32p), _p(arrs[4], _u32p),
                                  out, idx, ctypes.c_uint32(cap))
    n = L.oracle_ef_from_proximity(*args(None, None, 0))
    out = np.zeros(max(n, 1), EF_PAIR_DTYPE)
    idx = np.zeros((max(n, 1), 2), np.uint32)
    L.oracle_ef_from_proximity(*args(out.ctypes.data_as(ctypes.c_void_p), _p(idx, _u32p), n))
    return out[:n], idx[:n]


def canonical_ef(pairs, indices):
    """host_preprocess_ef_pairs' canonical order (intersection_resolver.cpp:693-726): (eid, fid),
    then memcmp of the 48-byte records."""
    pairs = np.ascontiguousarray(pairs)
    indices = np.ascontiguousarray(indices, np.uint32).reshape(-1, 2)
    raw = pairs.view(np.uint8).reshape(len(pairs), -1)
    order = sorted(range(len(pairs)), key=lambda i: (int(indices[i, 0]), int(indices[i, 1]), raw[i].tobytes()))
    return pairs[order], indices[order]


def response_step(pairs, x, scale=1.0):
    """The repair loop's position update: a fixed step along the assembled response pairs,
    restating u26_response_step (a library-defined update that stands in for the solver step
    of the reference's IP loop). Each pair with k2 > 0 asks its sides apart by
    Delta = -k1 / k2 along its normal: the first primitive (VF vertex, first EE edge) takes
    +Delta / 2 n, the second -Delta / 2 n, per vertex weighted by the template's barycentric
    weights (weights <= 0 are skipped). Sums are 2^-40 m / 2^-32 fixed point (round half to
    even), each moved vertex takes scale x sum(w d) / sum(w) in FP64, rounded to FP32.
    Returns (new positions [V, 3] float32, vertices moved)."""
    tb = np.uint32(0x80000000)
    p = np.ascontiguousarray(pairs)
    x = np.asarray(x, np.float32).reshape(-1, 3)
    nv = len(x)
    k1, k2 = p["vec2"][:, 0], p["vec2"][:, 1]
    p = p[(k2 > 0) & np.isfinite(k1)]
    idx = p["indices"]
    delta = (-p["vec2"][:, 0]) / p["vec2"][:, 1]
    half = p["vec1"][:, :3] * (np.float32(0.5) * delta)[:, None]
    one = np.float32(1.0)
    vf = (idx[:, 2] & tb) != 0
    ee = ~vf & ((idx[:, 3] & tb) != 0)
    b0, b1 = p["vec2"][:, 2], p["vec2"][:, 3]
    terms = []  # (vertex ids, +-half, weights) per template slot
    terms += [(idx[vf, 0], half[vf], np.ones(int(vf.sum()), np.float32)), (idx[vf, 1], -half[vf], b0[vf]),
              (idx[vf, 2] & ~tb, -half[vf], b1[vf]), (idx[vf, 3], -half[vf], (one - b0[vf]) - b1[vf])]
    terms += [(idx[ee, 0], half[ee], b0[ee]), (idx[ee, 1], half[ee], one - b0[ee]), (idx[ee, 2], -half[ee], b1[ee]),
              (idx[ee, 3] & ~tb, -half[ee], one - b1[ee])]
    acc = np.zeros((nv, 4), np.int64)
    for v, d, w in terms:
        keep = (v < nv) & (w > 0)
        v, d, w = v[keep].astype(np.int64), d[keep], w[keep]
        fx = np.rint((d * w[:, None]).astype(np.float64) * 2.0 ** 40).astype(np.int64)
        fw = np.rint(w.astype(np.float64) * 2.0 ** 32).astype(np.int64)
        for c in range(3):
            np.add.at(acc[:, c], v, fx[:, c])
        np.add.at(acc[:, 3], v, fw)
    moved = acc[:, 3] > 0
    out = x.copy()
    inv = 2.0 ** 32 / acc[moved, 3].astype(np.float64) / 2.0 ** 40
    s = np.float64(np.float32(scale))
    out[moved] = (x[moved].astype(np.float64) + s * (acc[moved, :3].astype(np.float64) * inv[:, None])).astype(np.float32)
    return out, int(moved.sum())


def filter_broad_phase(vf, ee, num_ef, invalid, regions, faces, edges):
    """IntersectionResolver::filter_broad_phase_pairs; returns flagged copies of the lists."""
    L = lib()
    vf = np.ascontiguousarray(vf, np.uint32).copy()
    ee = np.ascontiguousarray(ee, np.uint32).copy()
    inv = np.ascontiguousarray(invalid, np.uint32)
    rg = [None, None, None] if regions is None else [np.ascontiguousarray(a, np.uint32) for a in regions]
    f = np.ascontiguousarray(faces, np.uint32)
    e = np.ascontiguousarray(edges, np.uint32)
    L.oracle_filter_broad_phase(_p(vf, _u32p), ctypes.c_uint32(len(vf)), _p(ee, _u32p), ctypes.c_uint32(len(ee)),
                                ctypes.c_uint32(num_ef), _p(inv, _u32p), *[(_p(a, _u32p) if a is not None else None) for a in rg],
                                _p(f, _u32p), _p(e, _u32p))
    return vf, ee


def eigen3(S):
    S = np.ascontiguousarray(np.asarray(S, np.float32).T)  # columns
    out = np.zeros(9, np.float32)
    lib().oracle_eigen3(_p(S.reshape(-1), _f32p), _p(out, _f32p))
    return out.reshape(3, 3)


def detect_ef(mesh, d_hat=1e-3, thickness=0.0):
    """EF pairs of a mesh at its current positions (LBVH broad phase + narrow phase)."""
    dh = np.full(mesh.num_verts, d_hat, np.float32)
    th = np.full(mesh.num_verts, thickness, np.float32)
    tree = lbvh_build(TREE_FACE, mesh.x, mesh.faces)
    lbvh_refit(tree, mesh.x, mesh.x, th, mesh.faces)
    broad, _, _ = lbvh_query(tree, QUERY_EDGES_UNCULLED, mesh.x, mesh.x, mesh.edges, dh, th)
    return ef_narrow(broad, mesh.x, mesh.edges, mesh.faces, dh, mesh.vert_property)


# ---- unit entry points of the PRP decision rules (intersection_resolver2.h:405-506, 807-912;
# intersection_resolver2.cpp:311-375, 453-592, 1058-1230, 1268-1368, 1488-1569, 1883-1954)

_F, _U, _I = ctypes.c_float, ctypes.c_uint32, ctypes.c_int


def _sig(name, restype, argtypes):
    f = getattr(lib(), name)
    f.restype = restype
    f.argtypes = argtypes
    return f


def ccr_owns(own, opp, tau=0.25):
    """prp_intrinsic_contour_side_owns_vertex"""
    return bool(_sig("oracle_ccr_owns", _I, [_F, _F, _F])(own, opp, tau))


def ccr_owns_dual(rest_own, rest_opp, cur_own, cur_opp, tau=0.25, use_rest=True, use_current=True):
    """prp_dual_metric_contour_side_owns_vertex"""
    f = _sig("oracle_ccr_owns_dual", _I, [_F, _F, _F, _F, _F, _I, _I])
    return bool(f(rest_own, rest_opp, cur_own, cur_opp, tau, int(use_rest), int(use_current)))


def ccr_owns_blended(rest_own, rest_opp, cur_own, cur_opp, tau, weight):
    """prp_intrinsic_contour_side_owns_vertex_blended"""
    return bool(_sig("oracle_ccr_owns_blended", _I, [_F] * 6)(rest_own, rest_opp, cur_own, cur_opp, tau, weight))


def ccr_blended_phi(rest_own, rest_opp, cur_own, cur_opp, weight):
    """prp_intrinsic_contour_side_blended_phi"""
    return _sig("oracle_ccr_blended_phi", _F, [_F] * 5)(rest_own, rest_opp, cur_own, cur_opp, weight)


def ccr_roles_share(obj, comp):
    """prp_contour_roles_share_topology"""
    return bool(_sig("oracle_ccr_roles_share", _I, [_U] * 4)(obj[0], obj[1], comp[0], comp[1]))


def ccr_applies(enabled, obj, comp, use_deformed=False):
    """prp_intrinsic_contour_side_restriction_applies"""
    f = _sig("oracle_ccr_applies", _I, [_I, _U, _U, _U, _U, _I])
    return bool(f(int(enabled), obj[0], obj[1], comp[0], comp[1], int(use_deformed)))


RESP_DTYPE = np.dtype([("objective", np.float32), ("coverage", np.float32), ("depth", np.float32), ("cost", np.float32),
                       ("hit_count", np.uint32), ("covered", np.uint32), ("eligible", np.uint32), ("pad", np.uint32)])


def response(objective, coverage, eligible=True, depth=1.0, cost=1.0, hit_count=1, covered=1):
    """One candidate response record (the fields the comparator reads)."""
    return (objective, coverage, depth, cost, hit_count, covered, int(eligible), 0)


def select_response(responses):
    """prp_select_response: index of the best valid response, or -1."""
    a = np.array(responses, RESP_DTYPE)
    return _sig("oracle_select_response", _I, [_U, ctypes.c_void_p])(len(a), a.ctypes.data_as(ctypes.c_void_p))


def response_objective(objective, coverage):
    """prp_penetration_objective_divided_by_squared_coverage"""
    return _sig("oracle_response_objective", _F, [_F, _F])(objective, coverage)


def classify_contour(is_loop, is_boundary, adj_degree, mesh_index):
    """classify_contour_type over one contour's pairs (ContourType value)."""
    il = np.ascontiguousarray(is_loop, np.uint8)
    ib = np.ascontiguousarray(is_boundary, np.uint8)
    dg = np.ascontiguousarray(adj_degree, np.uint32)
    mi = np.ascontiguousarray(mesh_index, np.uint32)
    f = _sig("oracle_classify_contour", _U, [_U, ctypes.c_void_p, ctypes.c_void_p, _u32p, _u32p])
    return f(len(il), il.ctypes.data_as(ctypes.c_void_p), ib.ctypes.data_as(ctypes.c_void_p), _p(dg, _u32p), _p(mi, _u32p))


def _csr_call(name, row_ptr, col, flip):
    rp = np.ascontiguousarray(row_ptr, np.uint32)
    cl = np.ascontiguousarray(col, np.uint32)
    fl = np.ascontiguousarray(flip, np.uint32)
    n = len(rp) - 1
    root = np.zeros(max(n, 1), np.uint32)
    parity = np.zeros(max(n, 1), np.uint32)
    f = _sig(name, _U, [_U, _u32p, _u32p, _u32p, _u32p, _u32p])
    bad = f(n, _p(rp, _u32p), _p(cl, _u32p), _p(fl, _u32p), _p(root, _u32p), _p(parity, _u32p))
    return root[:n], parity[:n], bool(bad)


def flood_components(row_ptr, col, flip):
    """The contour flood fill with mesh parity (flood_components in oracle_prp.cpp, the one the
    PRP restatement runs) over a CSR graph: (root = smallest node of each node's component,
    parity, inconsistent)."""
    return _csr_call("oracle_flood_components", row_ptr, col, flip)


def contour_test_bfs(row_ptr, col, flip):
    """cpu_reference of test_parallel_contour_construction.cpp: breadth-first flood, same outputs."""
    return _csr_call("oracle_cc_bfs", row_ptr, col, flip)


CONTOUR_TEST_GRAPHS = ("small_fixed", "10K_chains_x10", "1K_chains_x100", "grid_100x100", "grid_200x250",
                       "random_50K_d4_c100", "random_100K_d6_c500", "singletons+pairs_100K")


def contour_test_graph(which):
    """Case `which` of test_parallel_contour_construction.cpp's main, as CSR (row_ptr, col, flip)."""
    mk = _sig("oracle_cc_graph_make", ctypes.c_void_p, [_I])
    h = mk(which)
    if not h:
        raise ValueError(f"no contour test graph {which}")
    try:
        n, m = _U(), _U()
        _sig("oracle_cc_graph_size", None, [ctypes.c_void_p, ctypes.POINTER(_U), ctypes.POINTER(_U)])(h, ctypes.byref(n), ctypes.byref(m))
        rp = np.zeros(n.value + 1, np.uint32)
        cl = np.zeros(max(m.value, 1), np.uint32)
        fl = np.zeros(max(m.value, 1), np.uint32)
        _sig("oracle_cc_graph_copy", None, [ctypes.c_void_p, _u32p, _u32p, _u32p])(h, _p(rp, _u32p), _p(cl, _u32p), _p(fl, _u32p))
        return rp, cl[:m.value], fl[:m.value]
    finally:
        _sig("oracle_cc_graph_free", None, [ctypes.c_void_p])(h)


def suppress(adjacency, pre_area, active):
    """prp_select_pre_finalize_contours_to_suppress: sorted suppressed contour ids."""
    nc = len(adjacency)
    off = np.zeros(nc + 1, np.uint32)
    for c, a in enumerate(adjacency):
        off[c + 1] = off[c] + len(a)
    adj = np.array([x for a in adjacency for x in a] or [0], np.uint32)
    area = np.ascontiguousarray(pre_area, np.float32)
    act = np.array(list(active) or [0], np.uint32)
    out = np.zeros(nc, np.uint8)
    f = _sig("oracle_suppress", None, [_U, _u32p, _u32p, _f32p, _U, _u32p, ctypes.c_void_p])
    f(nc, _p(off, _u32p), _p(adj, _u32p), _p(area, _f32p), len(active), _p(act, _u32p), out.ctypes.data_as(ctypes.c_void_p))
    return [int(c) for c in np.nonzero(out)[0]]


def penetration(hits, direction, vert_area, edge_area, face_area, vert_mass, vn, en, fn):
    """prp_eval_penetration_v2: dict of depth, volume, area, objective, cost."""
    h = np.ascontiguousarray(hits, HIT_DTYPE)
    arrs = [np.ascontiguousarray(a, np.float32) for a in (direction, vert_area, edge_area, face_area, vert_mass, vn, en, fn)]
    out = np.zeros(5, np.float32)
    f = _sig("oracle_penetration", None, [_U, ctypes.c_void_p, _f32p, _U, _U, _U] + [_f32p] * 7 + [_f32p])
    d, va, ea, fa, vm, vn_, en_, fn_ = arrs
    f(len(h), h.ctypes.data_as(ctypes.c_void_p), _p(d, _f32p), len(va), len(ea), len(fa), _p(va, _f32p), _p(ea, _f32p), _p(fa, _f32p),
      _p(vm, _f32p), _p(vn_, _f32p), _p(en_, _f32p), _p(fn_, _f32p), _p(out, _f32p))
    return dict(zip(("depth", "volume", "area", "objective", "cost"), out.tolist()))


def seed_directions(points, weights, boundary0, boundary1, x, vert_area, mode=0):
    """get_raycasting_direction on explicit inputs: (n, 3) float32."""
    P = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    W = np.ascontiguousarray(weights, np.float32)
    b0 = np.array(list(boundary0) or [0], np.uint32)
    b1 = np.array(list(boundary1) or [0], np.uint32)
    X = np.ascontiguousarray(x, np.float32).reshape(-1, 3)
    A = np.ascontiguousarray(vert_area, np.float32)
    out = np.zeros((26, 3), np.float32)
    f = _sig("oracle_seed_directions", _U, [_U, _U, _f32p, _f32p, _U, _u32p, _U, _u32p, _U, _f32p, _f32p, _f32p])
    n = f(mode, len(P), _p(P, _f32p), _p(W, _f32p), len(boundary0), _p(b0, _u32p), len(boundary1), _p(b1, _u32p), len(X), _p(X, _f32p),
          _p(A, _f32p), _p(out, _f32p))
    return out[:n]


class KInfo(ctypes.Structure):
    _fields_ = [("hit_count", _U), ("covered", _U), ("anchors", _U), ("mfs", _U), ("mfd", _U), ("eligible", _U),
                ("objective", _F), ("coverage", _F)]


_KEVAL = ctypes.CFUNCTYPE(_I, _U, _U, _U, _U, ctypes.POINTER(KInfo))


def kring_trace(init_k, diam, evaluate, active=None, cached=None, max_levels=70):
    """evaluate_current_runtime_directions_template for one runtime with a scripted evaluator.

    evaluate(level, k_src, k_dst, combo) -> dict of KInfo fields (empty dict: no hits).
    Returns dict(trace=[(k_src, k_dst) per level], finished, no_response, evaluations, eligible)."""
    n = len(active) if active is not None else 1
    act = np.ascontiguousarray(active if active is not None else [1], np.uint8)
    cache = None
    if cached is not None:
        cache = (KInfo * n)()
        for i, c in enumerate(cached):
            for k, v in (c or {}).items():
                setattr(cache[i], k, v)

    def cb(level, ks, kd, combo, out):
        for k, v in evaluate(level, ks, kd, combo).items():
            setattr(out[0], k, v)
        return 0

    trace = np.zeros(2 * max_levels, np.uint32)
    state = np.zeros(4, np.uint32)
    elig = np.zeros(n, np.uint8)
    ik = np.array(init_k, np.uint32)
    dm = np.array(diam, np.uint32)
    f = _sig("oracle_kring_trace", None, [_u32p, _u32p, _U, ctypes.c_void_p, ctypes.c_void_p, _KEVAL, _u32p, _U, _u32p, ctypes.c_void_p])
    keep = _KEVAL(cb)
    f(_p(ik, _u32p), _p(dm, _u32p), n, act.ctypes.data_as(ctypes.c_void_p), ctypes.cast(cache, ctypes.c_void_p) if cache is not None else None,
      keep, _p(trace, _u32p), max_levels, _p(state, _u32p), elig.ctypes.data_as(ctypes.c_void_p))
    lv = int(state[3])
    return dict(trace=[(int(trace[2 * i]), int(trace[2 * i + 1])) for i in range(min(lv, max_levels))], finished=bool(state[0]),
                no_response=bool(state[1]), evaluations=int(state[2]), eligible=[bool(e) for e in elig])


def direction_step(hits, x, vert_mass, direction, trust):
    """prp_compute_direction_optimization_step: (dir, predicted_reduction, gradient_norm, valid)."""
    h = np.ascontiguousarray(hits, HIT_DTYPE)
    X = np.ascontiguousarray(x, np.float32).reshape(-1, 3)
    M = np.ascontiguousarray(vert_mass, np.float32)
    d = np.ascontiguousarray(direction, np.float32)
    out = np.zeros(6, np.float32)
    f = _sig("oracle_direction_step", None, [_U, ctypes.c_void_p, _U, _f32p, _f32p, _f32p, _F, _f32p])
    f(len(h), h.ctypes.data_as(ctypes.c_void_p), len(X), _p(X, _f32p), _p(M, _f32p), _p(d, _f32p), trust, _p(out, _f32p))
    return out[:3].copy(), float(out[3]), float(out[4]), bool(out[5])


def hit(type_, src_id, dst_id, src_verts, dst_verts, bary, dist):
    """One HIT_DTYPE record; unused vertex slots ~0."""
    sv = list(src_verts) + [0xFFFFFFFF] * (3 - len(src_verts))
    dv = list(dst_verts) + [0xFFFFFFFF] * (3 - len(dst_verts))
    return np.array([(type_, src_id, dst_id, sv, dv, bary, dist)], HIT_DTYPE)
