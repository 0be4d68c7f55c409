"""The allocation-free EF sort (u26_ef_canonicalize_noalloc) against the allocating one.

Callers that own all of their GPU memory (a fixed arena) or that must not trigger a
cudaMalloc / cudaFree (those can synchronise the device) use the no-alloc variant, whose
scratch is a fixed array in the library's static device memory. It must give exactly the
result of u26_ef_canonicalize. Two calls in a row, on different inputs, check that the
shared scratch left behind by one call does not leak into the next.

This file is collected last on purpose: if it fails, a run that stops at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

from untangling26_b200 import synthetic
from untangling26_b200._native import ptr
from untangling26_b200.intersection_resolver import CollisionScene

pytestmark = pytest.mark.gpu


def _unsorted_ef(ctx, mesh):
    sc = CollisionScene(ctx, mesh, d_hat=1e-3, thickness=0.0)
    sc.construct_lbvh()
    sc.detect_ef_fused()
    n = int(sc.resolver.ef_count.item())
    pairs = sc.resolver.ef_list[:n].clone()
    idx = sc.resolver.ef_indices[:n].clone()
    sc.close()
    return pairs, idx, n


def _sort_both(ctx, mesh):
    pairs, idx, n = _unsorted_ef(ctx, mesh)
    assert 1 < n <= 32768
    pa, ia = pairs.clone(), idx.clone()
    pb, ib = pairs.clone(), idx.clone()
    ctx.check(ctx.lib.u26_ef_canonicalize(ctx.handle, n, ptr(pa), ptr(ia), mesh.num_edges, mesh.num_faces), "canonicalize")
    ctx.check(ctx.lib.u26_ef_canonicalize_noalloc(ctx.handle, n, ptr(pb), ptr(ib), mesh.num_edges, mesh.num_faces),
              "canonicalize_noalloc")
    torch.cuda.synchronize()
    return (pa.cpu().numpy(), ia.cpu().numpy()), (pb.cpu().numpy(), ib.cpu().numpy()), n


def test_noalloc_matches_allocating_sort_twice(u26ctx):
    first = synthetic.folded_sheet(96, seed=5)
    second = synthetic.two_sheets(48, seed=2)
    for mesh in (first, second):
        (pa, ia), (pb, ib), n = _sort_both(u26ctx, mesh)
        assert np.array_equal(ia, ib)
        assert pa.tobytes() == pb.tobytes()
        keys = ia[:, 0].astype(np.int64) * mesh.num_faces + ia[:, 1]
        assert np.all(np.diff(keys) >= 0), "not in canonical (eid, fid) order"


def test_noalloc_allocates_nothing():
    """On a context that has never sorted, the no-alloc sort (its first call included, which
    looks up the scratch address) leaves the library's allocation count unchanged."""
    from untangling26_b200 import Context
    ctx = Context(0)
    try:
        mesh = synthetic.two_sheets(40, seed=4)
        pairs, idx, n = _unsorted_ef(ctx, mesh)
        torch.cuda.synchronize()
        before = ctx.lib.u26_alloc_count()
        for _ in range(2):
            ctx.check(ctx.lib.u26_ef_canonicalize_noalloc(ctx.handle, n, ptr(pairs), ptr(idx), mesh.num_edges, mesh.num_faces),
                      "canonicalize_noalloc")
        torch.cuda.synchronize()
        assert ctx.lib.u26_alloc_count() == before
    finally:
        ctx.close()


def test_noalloc_rejects_oversize(u26ctx):
    st = u26ctx.lib.u26_ef_canonicalize_noalloc(u26ctx.handle, 32769, ctypes.c_void_p(16), ctypes.c_void_p(16), 10, 10)
    assert st == 1  # U26_ERR_CAPACITY, nothing launched
    assert b"fixed scratch limit" in u26ctx.lib.u26_ctx_last_error(u26ctx.handle)
