"""PRP contour evaluation: Python side of u26_prp_resolve (include/u26.h).

``PrpParams`` mirrors the SceneParams fields of the PRP path (scene_params.h:65-81);
``PrpResult`` holds one pass's outputs (augmented EF list, contours, per-contour results
and selected supports S(r)) as numpy arrays.
"""
import ctypes

import numpy as np

from . import _native as nat

c_u32, c_f32, c_u64, c_vp = ctypes.c_uint32, ctypes.c_float, ctypes.c_uint64, ctypes.c_void_p


class PrpParams(ctypes.Structure):
    _fields_ = [
        ("max_contours", c_u32),      # untangling_process_contours_count
        ("direction_mode", c_u32),    # 0 reference seed directions, 1 the 26 lattice directions
        ("use_ccr", c_u32),           # PRP_use_intrinsic_contour_side_candidates
        ("ccr_tau", c_f32),           # PRP_intrinsic_tau
        ("ccr_use_rest", c_u32),      # PRP_use_rest_geodesic_distance_for_intrinsic_candidates
        ("ccr_use_current", c_u32),   # PRP_use_deformed_boundary_distance_for_intrinsic_candidates
        ("batch_size", c_u32),        # PRP_cpu_contour_batch_size
        ("opt_iterations", c_u32),    # PRP_direction_optimization_iterations (0 = off)
        ("ccr_blend", c_u32),         # PRP_use_blended_intrinsic_coordinates
        ("ccr_blend_weight", c_f32),  # PRP_intrinsic_blend_weight
        ("form", c_u32),              # 0 batched packet ray casting (default), 1 plain form (baseline)
        ("solid_interior", c_u32),    # PRP_solid_interior_adjacency
        ("solid_all", c_u32),         # PRP_solid_interior_adjacency_all_meshes
        ("solid_eps_n", c_f32),       # PRP_solid_interior_adjacency_normal_eps
        ("solid_eps_d", c_f32),       # PRP_solid_interior_adjacency_dist_eps
        ("ignore_near_zero_dist_pairs", c_u32),  # 0: drop isolated degenerate EF pairs (the CLI's setting)
        ("fp64_recheck", c_u32),  # 1: FP64 recheck of the leaf tests inside their FP32 error band, FP64 metrics
        ("autotune", c_u32),      # 1: the scene's first pass picks the fastest ray-casting configuration
        ("raycast_config", c_u32),  # 0: default / autotuned; k: configuration k - 1 of RAYCAST_CONFIGS
    ]


def prp_params(**kw):
    p = PrpParams(max_contours=256, direction_mode=0, use_ccr=1, ccr_tau=0.25, ccr_use_rest=1, ccr_use_current=1,
                  batch_size=32, opt_iterations=0, ccr_blend=0, ccr_blend_weight=0.5,
                  form=0, solid_interior=1, solid_all=0, solid_eps_n=1e-4, solid_eps_d=1e-5, ignore_near_zero_dist_pairs=1, fp64_recheck=1, autotune=0, raycast_config=0)
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
EF_PAIR_DTYPE = np.dtype([("idx", np.uint32, 5), ("bary", np.float32, 3), ("grad", np.float32, 3), ("stiff", np.float32)])
assert RESULT_DTYPE.itemsize == 144 and HIT_DTYPE.itemsize == 48

STAGES = ("preprocess", "runtime", "candidates", "raycast", "cull", "control", "finalize", "total")


class PrpOutputView(ctypes.Structure):
    _fields_ = [
        ("num_pairs", c_u32), ("num_orig_pairs", c_u32), ("num_contours", c_u32), ("num_hits", c_u32),
        ("pairs", c_vp), ("pair_indices", c_vp), ("mesh_index", c_vp), ("contour_index", c_vp), ("pair_length", c_vp),
        ("contour_offsets", c_vp), ("contour_pairs", c_vp), ("results", c_vp), ("hit_offsets", c_vp), ("hits", c_vp),
        ("directions", c_vp), ("ray_tests", c_u64), ("ray_requests", c_u64), ("ray_pairs", c_u64), ("levels", c_u32),
        ("device_error_flags", c_u32), ("stage_ms", ctypes.c_double * 8), ("ray_nodes", c_u64),
        ("ray_edge_tests", c_u64), ("gpu_ms", ctypes.c_double * 6), ("ray_node_fetches", c_u64), ("ray_tri_fetches", c_u64),
        ("ray_edge_fetches", c_u64), ("ray_visits", c_u64), ("ray_candidate_tests", c_u64),
        ("fp64_rechecks", c_u64), ("fp64_flips", c_u64), ("dc_tie_rechecks", c_u64), ("dc_tie_flips", c_u64),
        ("fp64_delta_rel_err", ctypes.c_double), ("fp64_dc_rel_err", ctypes.c_double), ("fp64_j_rel_err", ctypes.c_double),
        ("tune_ms", ctypes.c_double * 18), ("raycast_parts", c_u32), ("raycast_blocks_per_sm", c_u32), ("tuned", c_u32),
        ("raycast_queue", c_u32),
    ]

# (subtree parts, blocks / SM, persistent work-queue grid)
RAYCAST_CONFIGS = tuple((p, b, q) for q in (False, True) for p in (4, 8, 16) for b in (6, 7, 8))
def config_name(c):
    """'8x7' (parts x blocks per SM, a warp per item) or '8x7q' (persistent work-queue grid)."""
    return f"{c[0]}x{c[1]}" + ("q" if c[2] else "")


GPU_PHASES = ("raycast", "sort", "union", "entries", "select", "download")

# CollisionPair::CollisionPairTemplate (collision_data.h:48-140), u26_collision_pair: 64 B
COLLISION_PAIR_DTYPE = np.dtype([("indices", np.uint32, 4), ("vec1", np.float32, 4), ("vec2", np.float32, 4), ("vec3", np.float32, 4)])


class ResponseParams(ctypes.Structure):
    """untangling_response_depth and stiffness_untangling (scene_params.h:66, 121-122)."""
    _fields_ = [("depth_threshold", ctypes.c_float), ("stiffness", ctypes.c_float)]


def response_params(depth_threshold=3e-3, stiffness=1e8):
    return ResponseParams(depth_threshold, stiffness)


class ResponseView(ctypes.Structure):
    _fields_ = [
        ("num_pairs", c_u32), ("pairs", c_vp), ("pair_info", c_vp), ("vert_regions", c_vp), ("edge_regions", c_vp),
        ("face_regions", c_vp), ("vert_regions_len", c_u32), ("edge_regions_len", c_u32), ("face_regions_len", c_u32),
    ]


class _DeviceWords:
    """__cuda_array_interface__ over words of device memory owned by the library."""

    def __init__(self, p, count):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<i4", "data": (p or 0, False), "version": 3}


def _device_words(torch, p, count, device):
    if count == 0 or not p:
        return torch.zeros(0, dtype=torch.int32, device=device)
    return torch.as_tensor(_DeviceWords(p, count), device=device).clone()


class PrpResponse:
    """Response pairs and region CSRs of one pass as device tensors (int32 words):
    pairs [n, 16] (u26_collision_pair), info [n, 4] (src, dst, packed region, type), and the
    vertex / edge / face region arrays in upload_2d_csr_from's layout."""

    def __init__(self, view, device):
        import torch
        n = view.num_pairs
        self.num_pairs = n
        self.pairs = _device_words(torch, view.pairs, 16 * n, device).view(-1, 16)
        self.info = _device_words(torch, view.pair_info, 4 * n, device).view(-1, 4)
        self.vert_regions = _device_words(torch, view.vert_regions, view.vert_regions_len, device)
        self.edge_regions = _device_words(torch, view.edge_regions, view.edge_regions_len, device)
        self.face_regions = _device_words(torch, view.face_regions, view.face_regions_len, device)

    def host_pairs(self):
        return self.pairs.cpu().numpy().view(np.uint32).copy().view(COLLISION_PAIR_DTYPE).reshape(-1)

    @staticmethod
    def csr_rows(arr):
        """[rows] of a upload_2d_csr_from array (host numpy)."""
        a = np.asarray(arr, np.uint32)
        if len(a) == 0:
            return []
        n = int(a[0]) - 1
        return [a[a[i]:a[i + 1]] for i in range(n)]


def _host_array(p, count, dtype):
    if count == 0 or not p:
        return np.zeros(0, dtype)
    nbytes = count * np.dtype(dtype).itemsize
    buf = (ctypes.c_char * nbytes).from_address(p)
    return np.frombuffer(bytes(buf), dtype=dtype, count=count).copy()


class PrpResult:
    """One pass's outputs, copied out of the u26_prp_output handle."""

    def __init__(self, lib, handle):
        v = PrpOutputView()
        st = lib.u26_prp_output_view_get(handle, ctypes.byref(v))
        if st != 0:
            raise nat.U26Error(st, "u26_prp_output_view_get")
        n, nc, nh = v.num_pairs, v.num_contours, v.num_hits
        self.num_orig_pairs = v.num_orig_pairs
        self.pairs = _host_array(v.pairs, n, EF_PAIR_DTYPE)
        self.pair_indices = _host_array(v.pair_indices, 2 * n, np.uint32).reshape(-1, 2)
        self.mesh_index = _host_array(v.mesh_index, n, np.uint32)
        self.contour_index = _host_array(v.contour_index, n, np.uint32)
        self.pair_length = _host_array(v.pair_length, n, np.float32)
        coff = _host_array(v.contour_offsets, nc + 1, np.uint32)
        cp = _host_array(v.contour_pairs, int(coff[-1]) if nc else 0, np.uint32)
        self.contours = [cp[coff[c]:coff[c + 1]] for c in range(nc)]
        self.results = _host_array(v.results, nc, RESULT_DTYPE)
        hoff = _host_array(v.hit_offsets, nc + 1, np.uint32)
        hits = _host_array(v.hits, nh, HIT_DTYPE)
        self.hits = [hits[hoff[c]:hoff[c + 1]] for c in range(nc)]
        dirs = _host_array(v.directions, nc * 26 * 3, np.float32).reshape(nc, 26, 3)
        self.directions = [dirs[c, :self.results[c]["num_dirs"]] for c in range(nc)]
        self.tested = int(v.ray_tests)
        self.requests = int(v.ray_requests)
        self.pairs_tested = int(v.ray_pairs)
        self.levels = int(v.levels)
        self.device_error_flags = int(v.device_error_flags)
        self.stage_ms = dict(zip(STAGES, list(v.stage_ms)))
        self.gpu_ms = dict(zip(GPU_PHASES, list(v.gpu_ms)))
        self.nodes_visited = int(v.ray_nodes)
        self.edge_tests = int(v.ray_edge_tests)
        self.node_fetches = int(v.ray_node_fetches)
        self.tri_fetches = int(v.ray_tri_fetches)
        self.edge_fetches = int(v.ray_edge_fetches)
        self.ray_visits = int(v.ray_visits)
        self.candidate_tests = int(v.ray_candidate_tests)
        self.raycast_config = {"parts": int(v.raycast_parts), "blocks_per_sm": int(v.raycast_blocks_per_sm),
                               "queue": bool(v.raycast_queue), "tuned_this_pass": bool(v.tuned)}
        if v.tuned:
            self.raycast_config["tune_ms"] = {config_name(c): round(float(ms), 3) for c, ms in zip(RAYCAST_CONFIGS, v.tune_ms)}
        self.fp64 = {"rechecks": int(v.fp64_rechecks), "flips": int(v.fp64_flips), "dc_tie_rechecks": int(v.dc_tie_rechecks),
                     "dc_tie_flips": int(v.dc_tie_flips), "delta_rel_err": float(v.fp64_delta_rel_err),
                     "dc_rel_err": float(v.fp64_dc_rel_err), "j_rel_err": float(v.fp64_j_rel_err)}
