"""Near-zero-distance proximity pairs as EF pairs on the GPU (u26_ef_add_from_proximity), the
payload tie-break of the canonical EF sort, and a PRP pass with ignore_near_zero_dist_pairs
off (degenerate EF filter), each against the CPU oracle, bit-exact."""
import numpy as np
import pytest
import torch

from untangling26_b200 import synthetic
from untangling26_b200.intersection_resolver import CollisionScene
from untangling26_b200.prp import prp_params

from test_proximity import contact_pairs
from test_prp_gpu import _compare

pytestmark = pytest.mark.gpu


def _device_lists(u26ctx, pairs, pidx):
    dev = torch.device("cuda", u26ctx.device)
    nl = torch.from_numpy(pairs.view(np.int32).reshape(-1, 16).copy()).to(dev)
    ni = torch.from_numpy(pidx.view(np.int32).copy()).to(dev)
    cnt = torch.tensor([len(pairs)], dtype=torch.int32, device=dev)
    return nl, ni, cnt


@pytest.mark.parametrize("n,seed", [(16, 0), (32, 1)])
def test_proximity_conversion_and_pass(oracle, u26ctx, n, seed):
    m = synthetic.sheets_in_contact(n, seed=seed)
    pairs, pidx = contact_pairs(m, n, seed)
    sc = CollisionScene(u26ctx, m, d_hat=1e-3, thickness=0.0)
    sc.construct_lbvh()
    kw = dict(ignore_near_zero_dist_pairs=0, max_contours=64)
    res = sc.untangle_pass(prp_params(**kw), proximity=_device_lists(u26ctx, pairs, pidx))
    # the canonical EF list the pass ran on: narrow-phase pairs + converted pairs
    n_ef = int(sc.resolver.ef_count.item())
    g_pairs, g_idx = sc.resolver.download(n_ef)
    ef0, idx0 = oracle.detect_ef(m)
    vae, eaf = m.vert_adj_edges.one_array(), m.edge_adj_faces_ext.one_array()
    efp, idxp = oracle.ef_from_proximity(pairs, pidx, m.x, m.edges, m.faces, vae, eaf)
    assert len(efp) > 0
    ef, idx = oracle.canonical_ef(np.concatenate([ef0, efp]), np.concatenate([idx0, idxp]))
    assert n_ef == len(ef)
    assert g_pairs.tobytes() == ef.tobytes() and np.array_equal(g_idx, idx)
    # the pass: the degenerate zero-distance pairs are filtered the same way on both sides
    ref = oracle.PrpRun(m, ef, idx, oracle.prp_params(**kw))
    assert ref.num_orig_pairs < len(ef)
    _compare(res, ref)
    sc.close()


def test_canonical_tiebreak_on_shuffled_duplicates(oracle, u26ctx):
    """Duplicate (eid, fid) keys in any input order come out in payload memcmp order."""
    m = synthetic.sheets_in_contact(16, seed=0)
    pairs, pidx = contact_pairs(m, 16)
    vae, eaf = m.vert_adj_edges.one_array(), m.edge_adj_faces_ext.one_array()
    efp, idxp = oracle.ef_from_proximity(pairs, pidx, m.x, m.edges, m.faces, vae, eaf)
    want_p, want_i = oracle.canonical_ef(efp, idxp)
    sc = CollisionScene(u26ctx, m, d_hat=1e-3, thickness=0.0)
    for seed in range(3):
        perm = np.random.default_rng(seed).permutation(len(efp))
        k = len(efp)
        sc.resolver.ef_list[:k] = torch.from_numpy(efp[perm].view(np.int32).reshape(k, 12).copy()).to(sc.resolver.ef_list.device)
        sc.resolver.ef_indices[:k] = torch.from_numpy(idxp[perm].view(np.int32).copy()).to(sc.resolver.ef_list.device)
        sc.resolver.ef_count.fill_(k)
        sc.resolver.canonicalize(m.num_edges, m.num_faces)
        g_p, g_i = sc.resolver.download(k)
        assert g_p.tobytes() == want_p.tobytes() and np.array_equal(g_i, want_i)
    sc.close()


def test_degenerate_filter_pass(oracle, u26ctx):
    """A contour whose pairs are all degenerate is dropped; the rest matches the oracle."""
    m = synthetic.folded_sheet(40, seed=2)
    ef, idx = oracle.detect_ef(m)
    base = oracle.PrpRun(m, ef, idx, oracle.prp_params(max_contours=64))
    n = base.num_orig_pairs
    sizes = [len([p for p in c if p < n]) for c in base.contours]
    mod = ef.copy()
    for p in base.contours[int(np.argmin(sizes))]:
        if p < n:
            mod[p]["bary"][1] = 1e-5
    kw = dict(max_contours=64, ignore_near_zero_dist_pairs=0)
    ref = oracle.PrpRun(m, mod, idx, oracle.prp_params(**kw))
    assert ref.num_orig_pairs == n - min(sizes)
    sc = CollisionScene(u26ctx, m, d_hat=1e-3, thickness=0.0)
    sc.construct_lbvh()
    dev = sc.resolver.ef_list.device
    sc.resolver.ef_list[:len(mod)] = torch.from_numpy(mod.view(np.int32).reshape(-1, 12).copy()).to(dev)
    sc.resolver.ef_indices[:len(mod)] = torch.from_numpy(idx.view(np.int32).copy()).to(dev)
    sc.resolver.ef_count.fill_(len(mod))
    sc.refit_face_tree()
    res = sc.host_resolve(prp_params(**kw), num_pairs=len(mod))
    _compare(res, ref)
    sc.close()


def test_proximity_conversion_overflow(oracle, u26ctx):
    """An EF list too small for the converted pairs: the count still reaches the full total (so the
    caller can grow the list), every slot below the capacity is written and none past it."""
    from untangling26_b200._native import ptr
    m = synthetic.sheets_in_contact(16, seed=0)
    pairs, pidx = contact_pairs(m, 16)
    vae, eaf = m.vert_adj_edges.one_array(), m.edge_adj_faces_ext.one_array()
    efp, _ = oracle.ef_from_proximity(pairs, pidx, m.x, m.edges, m.faces, vae, eaf)
    cap = 8
    assert len(efp) > cap
    dev = torch.device("cuda", u26ctx.device)
    nl, ni, cnt = _device_lists(u26ctx, pairs, pidx)
    up = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32).copy()).to(dev)
    x, edges, faces, d_vae, d_eaf = up(m.x), up(m.edges), up(m.faces), up(vae), up(eaf)
    ef_list = torch.full((2 * cap, 12), -7, dtype=torch.int32, device=dev)
    ef_idx = torch.full((2 * cap, 2), -7, dtype=torch.int32, device=dev)
    ef_count = torch.zeros(1, dtype=torch.int32, device=dev)
    u26ctx.check(u26ctx.lib.u26_ef_add_from_proximity(u26ctx.handle, ptr(nl), ptr(ni), ptr(cnt), len(pairs), ptr(x), ptr(edges),
                                                      ptr(faces), ptr(d_vae), ptr(d_eaf), ptr(ef_count), ptr(ef_list), ptr(ef_idx), cap),
                 "ef_add_from_proximity")
    assert int(ef_count.item()) == len(efp)
    assert bool((ef_list[:cap] != -7).any(1).all()) and bool((ef_idx[:cap] != -7).any(1).all())
    assert bool((ef_list[cap:] == -7).all()) and bool((ef_idx[cap:] == -7).all())
