"""LBVH — Python mirror of lcs::LBVH (Solver/CollisionDetector/lbvh.h:164-325) over libu26.

Method names and argument meanings follow the reference class; buffers are torch CUDA
tensors (float32 positions [V,3], int32/uint32 index arrays). Every call enqueues
sm_100a kernels on the context's stream through the C ABI.
"""
import ctypes

import numpy as np
import torch

from . import _native as nat
from ._native import ptr

TREE_VERT, TREE_FACE, TREE_EDGE = nat.TREE_VERT, nat.TREE_FACE, nat.TREE_EDGE


class LBVH:
    def __init__(self, ctx, tree_type, num_leaves):
        """LbvhData::allocate (lbvh.h:99-140)."""
        self.ctx = ctx
        self.tree_type = tree_type
        self.num_leaves = int(num_leaves)
        h = ctypes.c_void_p()
        ctx.check(ctx.lib.u26_lbvh_create(ctx.handle, tree_type, self.num_leaves, ctypes.byref(h)), "u26_lbvh_create")
        self.handle = h
        self._keep = []

    def close(self):
        if getattr(self, "handle", None):
            self.ctx.lib.u26_lbvh_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- construction (lbvh.cpp:988-1047)
    def reduce_vert_tree_aabb(self, x):
        self._reduce(x, None)

    def reduce_edge_tree_aabb(self, x, edges):
        self._reduce(x, edges)

    def reduce_face_tree_aabb(self, x, faces):
        self._reduce(x, faces)

    def _reduce(self, x, prims):
        self._keep = [x, prims]  # construct_tree reads these
        self.ctx.check(self.ctx.lib.u26_lbvh_reduce_aabb(self.handle, ptr(x), x.shape[0], ptr(prims)), "reduce_aabb")

    def construct_tree(self):
        self.ctx.check(self.ctx.lib.u26_lbvh_construct_tree(self.handle), "construct_tree")

    # ---- refit (lbvh.cpp:1050-1092)
    def update_vert_tree_leave_aabb(self, thickness, x_start, x_end):
        self.ctx.check(self.ctx.lib.u26_lbvh_update_leaves(self.handle, ptr(thickness), ptr(x_start), ptr(x_end), None), "update_leaves")

    def update_edge_tree_leave_aabb(self, thickness, x_start, x_end, edges):
        self.ctx.check(self.ctx.lib.u26_lbvh_update_leaves(self.handle, ptr(thickness), ptr(x_start), ptr(x_end), ptr(edges)), "update_leaves")

    def update_face_tree_leave_aabb(self, thickness, x_start, x_end, faces):
        self.ctx.check(self.ctx.lib.u26_lbvh_update_leaves(self.handle, ptr(thickness), ptr(x_start), ptr(x_end), ptr(faces)), "update_leaves")

    def refit(self):
        self.ctx.check(self.ctx.lib.u26_lbvh_refit(self.handle), "refit")

    def update_and_refit(self, thickness, x_start, x_end, prims=None):
        """Leaf update and bottom-up refit in one launch."""
        self.ctx.check(self.ctx.lib.u26_lbvh_update_and_refit(self.handle, ptr(thickness), ptr(x_start), ptr(x_end), ptr(prims)), "update_and_refit")

    def set_full_global_aabb(self, on=True):
        """Morton codes over the AABB of all leaves instead of the reference's partial
        second-pass reduction (lbvh.cpp:999-1021). Query results are unchanged."""
        self.ctx.check(self.ctx.lib.u26_lbvh_set_option(self.handle, 1, int(bool(on))), "set_option")

    def check_health(self):
        h = ctypes.c_int(0)
        self.ctx.check(self.ctx.lib.u26_lbvh_check_health(self.handle, ctypes.byref(h)), "check_health")
        return bool(h.value)

    # ---- broad phase (lbvh.cpp:1193-1262)
    def _query(self, mode, x_begin, x_end, edges, count, pairs, d_hat, thickness):
        nq = x_begin.shape[0] if mode == nat.QUERY_VERTS else edges.shape[0]
        max_pairs = pairs.numel() // 2
        self.ctx.check(self.ctx.lib.u26_lbvh_query(self.handle, mode, ptr(x_begin), ptr(x_end), ptr(edges), nq, ptr(d_hat),
                                                   ptr(thickness), ptr(count), ptr(pairs), max_pairs), "query")

    def broad_phase_query_from_verts(self, x_begin, x_end, count, pairs, d_hat, thickness):
        self._query(nat.QUERY_VERTS, x_begin, x_end, None, count, pairs, d_hat, thickness)

    def broad_phase_query_from_edges(self, x_begin, x_end, edges, count, pairs, d_hat, thickness):
        self._query(nat.QUERY_EDGES, x_begin, x_end, edges, count, pairs, d_hat, thickness)

    def broad_phase_query_from_edges_unculled(self, x_begin, x_end, edges, count, pairs, d_hat, thickness):
        self._query(nat.QUERY_EDGES_UNCULLED, x_begin, x_end, edges, count, pairs, d_hat, thickness)

    # ---- inspection
    def arrays(self):
        """Copies of the tree arrays as numpy (synchronises)."""
        a = nat.U26LbvhArrays()
        self.ctx.check(self.ctx.lib.u26_lbvh_arrays_get(self.handle, ctypes.byref(a)), "arrays_get")
        n, nn = a.num_leaves, a.num_nodes
        self.ctx.synchronize()

        def dl(p, count, dtype):
            return device_view(p, count, dtype).cpu().numpy().copy()

        return {
            "morton_sorted": dl(a.morton_sorted, n, np.uint64),
            "sorted_get_original": dl(a.sorted_get_original, n, np.uint32),
            "parent": dl(a.parent, nn, np.uint32),
            "children": dl(a.children, 2 * nn, np.uint32).reshape(nn, 2),
            "object_idx": dl(a.object_idx, nn, np.uint32),
            "node_aabb": dl(a.node_aabb, 8 * nn, np.float32).reshape(nn, 8),
            "global_aabb": dl(a.global_aabb, 6, np.float32),
        }


_TYPESTR = {np.uint64: "<u8", np.uint32: "<u4", np.float32: "<f4", np.int32: "<i4"}


class _CudaArray:
    def __init__(self, p, count, dtype):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": _TYPESTR[dtype], "data": (int(p or 0), False),
                                         "version": 3, "strides": None}


def device_view(p, count, dtype):
    """A torch tensor viewing `count` elements at raw device pointer p (no copy)."""
    if count == 0:
        return torch.empty(0, dtype={np.uint64: torch.int64, np.uint32: torch.int32, np.float32: torch.float32,
                                      np.int32: torch.int32}[dtype], device="cuda")
    t = torch.as_tensor(_CudaArray(p, count, dtype), device="cuda")
    return t
