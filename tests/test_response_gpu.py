"""Response assembly on the GPU (u26_prp_make_response) against the CPU oracle.

Bit-exact: the collision pair templates (indices with type bits, normal, area, k1, k2,
barycentric coordinates), their (src, dst, packed region, type) records, the narrow-phase
list append after the penalty pairs, and the vertex / edge / face region CSRs.
"""
import numpy as np
import pytest
import torch

from untangling26_b200 import synthetic
from untangling26_b200 import _native as nat
from untangling26_b200.intersection_resolver import CollisionScene
from untangling26_b200.prp import PrpResponse, prp_params, response_params

pytestmark = pytest.mark.gpu


def _run(oracle, ctx, mesh, rp=(3e-3, 1e8), narrow=None, first=0, **kw):
    sc = CollisionScene(ctx, mesh, d_hat=1e-3, thickness=0.0)
    sc.construct_lbvh()
    nl, ni = narrow if narrow is not None else (None, None)
    res = sc.untangle_pass(prp_params(**kw), response=response_params(*rp), narrow_list=nl, narrow_indices=ni, first=first)
    ef_ref, idx_ref = oracle.detect_ef(mesh)
    ref = oracle.PrpRun(mesh, ef_ref, idx_ref, oracle.prp_params(**kw), response=rp)
    sc.close()
    return res, ref


def _compare(res, ref):
    r = res.response
    assert r.num_pairs == len(ref.response_pairs) == sum(len(h) for h in ref.hits)
    assert r.host_pairs().tobytes() == ref.response_pairs.tobytes()
    assert np.array_equal(r.info.cpu().numpy().view(np.uint32), ref.response_info)
    for name in ("vert_regions", "edge_regions", "face_regions"):
        assert np.array_equal(getattr(r, name).cpu().numpy().view(np.uint32), getattr(ref, name)), name


@pytest.mark.parametrize("n,seed", [(32, 0), (64, 3)])
def test_response_two_sheets(oracle, u26ctx, n, seed):
    m = synthetic.two_sheets(n, seed=seed)
    res, ref = _run(oracle, u26ctx, m)
    assert len(ref.response_pairs) > 0
    _compare(res, ref)
    # every vertex of a response pair carries the contour region of its side
    rows = PrpResponse.csr_rows(ref.vert_regions)
    for p, inf in zip(ref.response_pairs, ref.response_info):
        c = (int(inf[2]) >> 1) // 256
        for v in p["indices"] & 0x7FFFFFFF:
            assert set(rows[v]) & {2 * c, 2 * c + 1}


def test_response_folded_sheet_depth_clamp(oracle, u26ctx):
    """A small response depth clamps C for the deeper contours: k1 = -area stiffness depth_threshold."""
    m = synthetic.folded_sheet(48, seed=2)
    res, ref = _run(oracle, u26ctx, m, rp=(1e-4, 5e7), max_contours=64)
    assert len(ref.contours) > 1
    _compare(res, ref)
    pairs = ref.response_pairs
    k1, k2 = pairs["vec2"][:, 0], pairs["vec2"][:, 1]
    assert np.all(k2 > 0)
    assert np.allclose(k1, -1e-4 * k2, rtol=1e-6)


def test_response_batch_of_scenes(oracle, u26ctx):
    m = synthetic.batch_scenes(num=3, seed=13, tris_lo=2000, tris_hi=5000)
    res, ref = _run(oracle, u26ctx, m, max_contours=64)
    _compare(res, ref)
    types = set(ref.response_info[:, 3].tolist())
    assert types <= {0, 1, 2}


def test_response_narrow_list_append(oracle, u26ctx):
    """Pairs land after the penalty pairs with (src, dst) indices; the penalty part is untouched."""
    m = synthetic.two_sheets(32, seed=0)
    dev = torch.device("cuda", u26ctx.device)
    first, cap = 7, 4096
    nl = torch.full((cap, 16), -5, dtype=torch.int32, device=dev)
    ni = torch.full((cap, 2), -9, dtype=torch.int32, device=dev)
    res, ref = _run(oracle, u26ctx, m, narrow=(nl, ni), first=first)
    _compare(res, ref)
    n = res.response.num_pairs
    assert n > 0 and first + n <= cap
    nl_h, ni_h = nl.cpu().numpy(), ni.cpu().numpy()
    assert np.all(nl_h[:first] == -5) and np.all(ni_h[:first] == -9)
    assert nl_h[first:first + n].view(np.uint32).tobytes() == ref.response_pairs.tobytes()
    assert np.array_equal(ni_h[first:first + n].view(np.uint32), ref.response_info[:, :2])
    assert np.all(nl_h[first + n:] == -5) and np.all(ni_h[first + n:] == -9)


def test_response_narrow_list_capacity(oracle, u26ctx):
    """A list too small for the pairs returns U26_ERR_CAPACITY and writes nothing."""
    m = synthetic.two_sheets(32, seed=0)
    dev = torch.device("cuda", u26ctx.device)
    nl = torch.full((4, 16), -5, dtype=torch.int32, device=dev)
    ni = torch.full((4, 2), -9, dtype=torch.int32, device=dev)
    with pytest.raises(nat.U26Error) as e:
        _run(oracle, u26ctx, m, narrow=(nl, ni), first=2)
    assert e.value.status == 1
    assert torch.all(nl == -5) and torch.all(ni == -9)


def test_response_without_intersections(oracle, u26ctx):
    """No EF pairs: no response pairs, every region row empty, a narrow list left untouched."""
    m = synthetic.two_sheets(16, seed=0)
    m.x[m.num_verts // 2:, 2] += 3.0
    dev = torch.device("cuda", u26ctx.device)
    nl = torch.full((16, 16), -5, dtype=torch.int32, device=dev)
    ni = torch.full((16, 2), -9, dtype=torch.int32, device=dev)
    res, ref = _run(oracle, u26ctx, m, narrow=(nl, ni), first=3)
    assert res.response.num_pairs == 0 and len(ref.response_pairs) == 0
    _compare(res, ref)
    vr = res.response.vert_regions.cpu().numpy().view(np.uint32)
    assert len(vr) == m.num_verts + 1 and np.all(vr == m.num_verts + 1)
    assert torch.all(nl == -5) and torch.all(ni == -9)
