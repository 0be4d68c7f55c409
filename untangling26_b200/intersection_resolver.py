"""Collision detection stages of the untangling hot path behind the reference's interfaces.

* ``IntersectionResolver.ef_dcd_intersection_query`` mirrors
  IntersectionResolver::ef_dcd_intersection_query (intersection_resolver.h:41-52,
  intersection_resolver.cpp:365-423): EF narrow phase over a broad-phase list.
* ``CollisionScene`` owns the face/edge LBVHs and the per-vertex buffers of one mesh and
  exposes the solver's call sites (NewtonSolver::device_construct_lbvh,
  device_broadphase_dcd, device_narrowphase_dcd; newton_solver.cpp:1218-1380) for the
  EF path, plus the fused detection form.

EF pairs come back as a structured numpy array with the reference's 48-byte EfPair
layout (collision_data.h:150-220) and (eid, fid) indices, in canonical (eid, fid) order.
"""
import ctypes
import time

import numpy as np
import torch

from . import _native as nat
from ._native import ptr
from .lbvh import LBVH, TREE_EDGE, TREE_FACE, device_view

EF_PAIR_DTYPE = np.dtype([("idx", np.uint32, 5), ("bary", np.float32, 3), ("grad", np.float32, 3), ("stiff", np.float32)])


def _u32(t):
    return t.view(torch.int32) if t.dtype != torch.int32 else t


class IntersectionResolver:
    def __init__(self, ctx, max_ef_pairs):
        self.ctx = ctx
        self.max_ef = int(max_ef_pairs)
        dev = torch.device("cuda", ctx.device)
        self.ef_count = torch.zeros(1, dtype=torch.int32, device=dev)
        self.ef_list = torch.zeros((self.max_ef, 12), dtype=torch.int32, device=dev)  # 48 B rows
        self.ef_indices = torch.zeros((self.max_ef, 2), dtype=torch.int32, device=dev)

    def reset(self):
        self.ef_count.zero_()

    def ef_dcd_intersection_query(self, broad_pairs, broad_count, x, edges, faces, vert_property, d_hat):
        """Narrow phase over the broad-phase (eid, fid) list (count read on the device)."""
        max_broad = broad_pairs.numel() // 2
        self.ctx.check(self.ctx.lib.u26_ef_narrow_phase(
            self.ctx.handle, ptr(broad_pairs), ptr(broad_count), max_broad, ptr(x), ptr(edges), ptr(faces),
            ptr(vert_property), ptr(d_hat), ptr(self.ef_count), ptr(self.ef_list), ptr(self.ef_indices), self.max_ef),
            "ef_narrow_phase")

    def add_ef_from_proximity_pairs(self, narrow_list, narrow_indices, narrow_count, x, edges, faces, vae_csr, eaf_csr,
                                    max_proximity=None):
        """fn_add_ef_from_proximity_pairs (intersection_resolver.cpp:199-363): near-zero-distance
        VF / EE pairs of the device narrow-phase list ([n, 16] templates, [n, 2] indices, count
        on the device) appended to the EF list as zero-stiffness EF pairs."""
        cap = int(narrow_list.shape[0]) if max_proximity is None else max_proximity
        self.ctx.check(self.ctx.lib.u26_ef_add_from_proximity(
            self.ctx.handle, ptr(narrow_list), ptr(narrow_indices), ptr(narrow_count), cap, ptr(x), ptr(edges), ptr(faces),
            ptr(vae_csr), ptr(eaf_csr), ptr(self.ef_count), ptr(self.ef_list), ptr(self.ef_indices), self.max_ef),
            "ef_add_from_proximity")

    def canonicalize(self, num_edges, num_faces):
        """Sort the EF list by (eid, fid) on the device (synchronises for the count)."""
        n = int(self.ef_count.item())
        if n > self.max_ef:
            raise nat.U26Error(1, f"EF list overflow: {n} pairs > capacity {self.max_ef}")
        self.ctx.check(self.ctx.lib.u26_ef_canonicalize(self.ctx.handle, n, ptr(self.ef_list), ptr(self.ef_indices),
                                                        num_edges, num_faces), "ef_canonicalize")
        return n

    def download(self, n):
        pairs = self.ef_list[:n].cpu().numpy().view(EF_PAIR_DTYPE).reshape(-1)
        idx = self.ef_indices[:n].cpu().numpy().view(np.uint32)
        return pairs.copy(), idx.copy()


class CollisionScene:
    """Device-resident mesh + face/edge trees for the EF detection path of one scene."""

    def __init__(self, ctx, mesh, d_hat=1e-3, thickness=0.0, max_broad_pairs=None, max_ef_pairs=None, parity_tree=False):
        self.ctx = ctx
        self.mesh = mesh
        dev = torch.device("cuda", ctx.device)
        self.dev = dev
        self.x = torch.from_numpy(mesh.x).to(dev)
        self.edges = torch.from_numpy(mesh.edges.view(np.int32)).to(dev)
        self.faces = torch.from_numpy(mesh.faces.view(np.int32)).to(dev)
        self.vert_property = torch.from_numpy(mesh.vert_property.view(np.int32)).to(dev)
        nv = mesh.num_verts
        self.d_hat = torch.full((nv,), float(d_hat), dtype=torch.float32, device=dev)
        self.thickness = torch.full((nv,), float(thickness), dtype=torch.float32, device=dev)
        self.face_tree = LBVH(ctx, TREE_FACE, mesh.num_faces)
        self.edge_tree = LBVH(ctx, TREE_EDGE, mesh.num_edges)
        # chosen form: Morton codes over the full scene AABB and Morton-ordered queries
        # (parity_tree=True keeps the reference's tree topology bit for bit)
        self.parity_tree = parity_tree
        if not parity_tree:
            self.face_tree.set_full_global_aabb(True)
            self.edge_tree.set_full_global_aabb(True)
        self.edge_order = None
        self.max_broad = int(max_broad_pairs or max(1 << 16, 8 * mesh.num_edges))
        self.broad_count = torch.zeros(1, dtype=torch.int32, device=dev)
        self.broad_pairs = torch.zeros((self.max_broad, 2), dtype=torch.int32, device=dev)
        self.resolver = IntersectionResolver(ctx, max_ef_pairs or max(1 << 14, mesh.num_edges))
        self.stats = torch.zeros(4, dtype=torch.int64, device=dev)

    def set_positions(self, x):
        self.x.copy_(torch.as_tensor(x, dtype=torch.float32).reshape(-1, 3))

    # NewtonSolver::device_construct_lbvh (newton_solver.cpp:1218-1224)
    def construct_lbvh(self, x_step_start=None):
        xs = self.x if x_step_start is None else x_step_start
        self.face_tree.reduce_face_tree_aabb(xs, self.faces)
        self.edge_tree.reduce_edge_tree_aabb(xs, self.edges)
        self.face_tree.construct_tree()
        self.edge_tree.construct_tree()
        if not self.parity_tree:
            # edge queries in the edge tree's Morton order: a warp walks nearby edges
            a = nat.U26LbvhArrays()
            self.ctx.check(self.ctx.lib.u26_lbvh_arrays_get(self.edge_tree.handle, ctypes.byref(a)), "arrays")
            self.edge_order = device_view(a.sorted_get_original, self.mesh.num_edges, np.uint32)

    # NewtonSolver::device_broadphase_dcd, EF part (newton_solver.cpp:1260-1299)
    def broadphase_dcd_ef(self, fused_refit=True):
        if fused_refit:
            self.face_tree.update_and_refit(self.thickness, self.x, self.x, self.faces)
        else:
            self.face_tree.update_face_tree_leave_aabb(self.thickness, self.x, self.x, self.faces)
            self.face_tree.refit()
        self.broad_count.zero_()
        self.face_tree.broad_phase_query_from_edges_unculled(self.x, self.x, self.edges, self.broad_count, self.broad_pairs,
                                                             self.d_hat, self.thickness)

    # NewtonSolver::device_narrowphase_dcd, EF part (newton_solver.cpp:1340-1380)
    def narrowphase_dcd_ef(self):
        self.resolver.reset()
        self.resolver.ef_dcd_intersection_query(self.broad_pairs, self.broad_count, self.x, self.edges, self.faces,
                                                self.vert_property, self.d_hat)

    def detect_ef_fused(self, with_stats=False):
        """Refit + fused broad/narrow EF detection (no broad-phase list)."""
        self.refit_face_tree()
        self.resolver.reset()
        if with_stats:
            self.stats.zero_()
        self.ef_detect(with_stats)

    def refit_face_tree(self):
        self.face_tree.update_and_refit(self.thickness, self.x, self.x, self.faces)

    def ef_detect(self, with_stats=False):
        """The fused EF kernel alone (face tree already refit, counter already reset)."""
        self.ctx.check(self.ctx.lib.u26_ef_detect(
            self.face_tree.handle, ptr(self.x), ptr(self.edges), self.mesh.num_edges, ptr(self.faces),
            ptr(self.vert_property), ptr(self.d_hat), ptr(self.thickness), ptr(self.edge_order), ptr(self.resolver.ef_count),
            ptr(self.resolver.ef_list), ptr(self.resolver.ef_indices), self.resolver.max_ef,
            ptr(self.stats) if with_stats else None), "ef_detect")

    def ef_pairs(self):
        """Canonical EF pairs (numpy) of the last detection."""
        n = self.resolver.canonicalize(self.mesh.num_edges, self.mesh.num_faces)
        return self.resolver.download(n)

    # ---- PRP contour evaluation (IntersectionResolver::host_resolve, intersection_resolver.cpp:2131-2218)
    def _ensure_prp_scene(self):
        if getattr(self, "prp_scene", None) is None:
            desc = self.mesh.desc()
            h = ctypes.c_void_p()
            self.ctx.check(self.ctx.lib.u26_scene_create(self.ctx.handle, ctypes.byref(desc), ctypes.byref(h)), "scene_create")
            self.prp_scene = h
            self._desc = desc

    def host_resolve(self, params=None, num_pairs=None, response=None, narrow_list=None, narrow_indices=None, first=0):
        """PRP pass over the canonical EF list of the last detection (call ef_pairs() or
        canonicalize first). Returns a PrpResult. response: ResponseParams to also assemble
        the response pairs and region CSRs (result.response, a PrpResponse); narrow_list
        ([capacity, 16] int32) / narrow_indices ([capacity, 2] int32) receive the pairs at
        [first, first + n) after the penalty pairs (upload_response_pairs_to_gpu)."""
        from .prp import PrpResponse, PrpResult, ResponseView, prp_params
        self._ensure_prp_scene()
        params = params or prp_params()
        n = int(self.resolver.ef_count.item()) if num_pairs is None else num_pairs
        # the edge tree is refit at x for the EE ray casts (the face tree already is)
        self.edge_tree.update_and_refit(self.thickness, self.x, self.x, self.edges)
        out = ctypes.c_void_p()
        self.ctx.check(self.ctx.lib.u26_prp_resolve(
            self.prp_scene, self.face_tree.handle, self.edge_tree.handle, ptr(self.x), ptr(self.resolver.ef_list),
            ptr(self.resolver.ef_indices), n, ctypes.byref(params), ctypes.byref(out)), "prp_resolve")
        try:
            res = PrpResult(self.ctx.lib, out)
            if response is not None:
                view = ResponseView()
                cap = 0 if narrow_list is None else int(narrow_list.shape[0])
                if narrow_list is not None and (narrow_indices is None or int(narrow_indices.shape[0]) != cap):
                    raise ValueError("narrow_indices must match narrow_list")
                t0 = time.perf_counter()
                self.ctx.check(self.ctx.lib.u26_prp_make_response(
                    self.prp_scene, out, ctypes.byref(response), ptr(narrow_list) if narrow_list is not None else None,
                    ptr(narrow_indices) if narrow_indices is not None else None, first, cap, ctypes.byref(view)), "prp_make_response")
                ms = (time.perf_counter() - t0) * 1e3  # the call synchronises
                res.response = PrpResponse(view, self.x.device)
                res.response.ms = ms
            return res
        finally:
            self.ctx.lib.u26_prp_output_destroy(out)

    def _adjacency_csrs(self):
        """sa_vert_adj_edges_csr / edge_adj_faces_csr in upload_2d_csr_from's one-array layout."""
        if getattr(self, "_vae_csr", None) is None:
            dev = self.x.device
            self._vae_csr = torch.from_numpy(self.mesh.vert_adj_edges.one_array().view(np.int32)).to(dev)
            self._eaf_csr = torch.from_numpy(self.mesh.edge_adj_faces_ext.one_array().view(np.int32)).to(dev)
        return self._vae_csr, self._eaf_csr

    def add_ef_from_proximity_pairs(self, narrow_list, narrow_indices, narrow_count, max_proximity=None):
        """Near-zero-distance proximity pairs as EF pairs (the reference's
        ignore_near_zero_dist_pairs = false, intersection_resolver.cpp:404-422)."""
        vae, eaf = self._adjacency_csrs()
        self.resolver.add_ef_from_proximity_pairs(narrow_list, narrow_indices, narrow_count, self.x, self.edges, self.faces, vae, eaf,
                                                  max_proximity)

    def untangle_pass(self, params=None, response=None, proximity=None, **narrow):
        """One untangling pass at the current positions: refit, fused EF detection (plus, with
        proximity = (narrow_list, narrow_indices, narrow_count), the near-zero-distance proximity
        pairs as EF pairs), canonical EF order, PRP contour evaluation (and, with response, its
        response pairs). The EF detection counts its node / leaf tests and FP64 rechecks into
        self.stats ([nodes, leaf tests, rechecked, flipped])."""
        self.detect_ef_fused(with_stats=True)
        if proximity is not None:
            self.add_ef_from_proximity_pairs(*proximity)
        n = self.resolver.canonicalize(self.mesh.num_edges, self.mesh.num_faces)
        return self.host_resolve(params, num_pairs=n, response=response, **narrow)

    def response_step(self, response, scale=1.0):
        """x <- x + a fixed step along the pass's assembled response (u26_response_step): every
        pair asks its sides apart by -k1 / k2 along its normal, each vertex moves by scale x the
        weighted mean of its requests. Returns the number of vertices moved."""
        nv = self.mesh.num_verts
        if getattr(self, "_step_scratch", None) is None:
            self._step_scratch = torch.zeros(4 * nv, dtype=torch.int64, device=self.dev)
            self._step_moved = torch.zeros(1, dtype=torch.int64, device=self.dev)
        self.ctx.check(self.ctx.lib.u26_response_step(
            self.ctx.handle, ptr(response.pairs), response.num_pairs, ptr(self.x), nv, float(scale), ptr(self._step_scratch),
            ptr(self._step_moved)), "response_step")
        return int(self._step_moved.item())

    # ---- region-based pair filtering (IntersectionResolver::filter_invalid_pairs /
    # filter_broad_phase_pairs, intersection_resolver.cpp:2586-2676): the contour regions of
    # the last pass's response applied to the solver's contact pairs
    def _num_ef(self, num_ef):
        return int(self.resolver.ef_count.item()) if num_ef is None else num_ef

    def filter_invalid_pairs(self, narrow_list, narrow_indices, num_proximity_pairs, vert_offset, vert_is_invalid,
                             response=None, num_ef=None):
        """Disable (k1 = k2 = 0) the proximity pairs [0, num_proximity_pairs) of the device
        narrow-phase list ([n, 16] int32 templates, [n, 2] indices) that touch a vertex made
        invalid by a too-close proximity pair or, with a PrpResponse, whose region match is 1."""
        rg = (None, None, None) if response is None else (response.vert_regions, response.edge_regions, response.face_regions)
        self.ctx.check(self.ctx.lib.u26_filter_invalid_pairs(
            self.ctx.handle, ptr(narrow_list), ptr(narrow_indices), num_proximity_pairs, self._num_ef(num_ef), ptr(self.x),
            ptr(vert_offset), self.mesh.num_verts, ptr(vert_is_invalid), *[ptr(t) for t in rg]), "filter_invalid_pairs")

    def filter_broad_phase_pairs(self, vf_list, num_vf, ee_list, num_ee, vert_is_invalid, response, num_ef=None):
        """Flag the CCD broad-phase VF / EE lists ([n, 2] int32): bit 31 region match,
        bit 30 an invalid vertex."""
        rg = (None, None, None) if response is None else (response.vert_regions, response.edge_regions, response.face_regions)
        self.ctx.check(self.ctx.lib.u26_filter_broad_phase_pairs(
            self.ctx.handle, ptr(vf_list), num_vf, ptr(ee_list), num_ee, self._num_ef(num_ef), ptr(vert_is_invalid),
            *[ptr(t) for t in rg], ptr(self.faces), ptr(self.edges)), "filter_broad_phase_pairs")

    def close(self):
        if getattr(self, "prp_scene", None) is not None:
            self.ctx.lib.u26_scene_destroy(self.prp_scene)
            self.prp_scene = None
        self.face_tree.close()
        self.edge_tree.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
