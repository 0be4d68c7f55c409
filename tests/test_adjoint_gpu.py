"""The CUDA adjoint (u26_prp_adjoint through torch_ops.JFunction) on real supports S(r) of
the two-sheet scenes at 32 x 32 and 128 x 128: J, E and their gradients in x and r against
the FP64 restatement (tolerance 2e-3 relative to each quantity's scale, fp32 forward),
dE/dr against the reference's refinement gradient, and the torch.autograd path."""
import numpy as np
import pytest
import torch

from oracle import adjoint as adj
from untangling26_b200 import synthetic
from untangling26_b200.intersection_resolver import CollisionScene
from untangling26_b200.prp import prp_params
from untangling26_b200.torch_ops import JFunction, Support

pytestmark = pytest.mark.gpu


def _support(ctx, n, seed):
    m = synthetic.two_sheets(n, seed=seed)
    sc = CollisionScene(ctx, m, d_hat=1e-3, thickness=0.0)
    sc.construct_lbvh()
    res = sc.untangle_pass(prp_params())
    sc.close()
    cs = [c for c in range(len(res.hits)) if len(res.hits[c])]
    assert cs
    return m, res, Support(ctx, res, m, cs)


def _fp64(m, res, c):
    hits = res.hits[c]
    r = np.asarray(res.results[c]["dir"], np.float64)
    return hits, r, (m.rest_vert_area, m.rest_edge_area, m.rest_face_area, m.vert_mass)


@pytest.mark.parametrize("n,seed", [(32, 0), (128, 1)])
def test_adjoint_matches_fp64(u26ctx, n, seed):
    """Forward J, E and the displacement-cost gradients (all hits) against FP64; dE/dr against
    the reference refinement's gradient."""
    m, res, sup = _support(u26ctx, n, seed)
    dev = torch.device("cuda", u26ctx.device)
    x = torch.from_numpy(m.x).to(dev).requires_grad_(True)
    dirs = sup.dirs.clone().requires_grad_(True)
    J, E = JFunction.apply(x, dirs, sup)
    wE = torch.rand(len(J), device=dev, generator=torch.Generator(device=dev).manual_seed(4))
    (E * wE).sum().backward()
    Jh, Eh, gx, gd = J.detach().cpu().numpy(), E.detach().cpu().numpy(), x.grad.cpu().numpy(), dirs.grad.cpu().numpy()
    wEh = wE.cpu().numpy()
    x64 = m.x.astype(np.float64)
    gx_ref = np.zeros_like(x64)
    for i, c in enumerate(sup.contours):
        hits, r, mc = _fp64(m, res, c)
        J64, E64, _ = adj.objective(hits, x64, r, *mc)
        assert abs(Jh[i] - J64) <= 2e-3 * abs(J64) + 1e-12
        assert abs(Eh[i] - E64) <= 2e-3 * abs(E64) + 1e-12
        _, _, gEx, gEr = adj.gradients(hits, x64, r, *mc)
        assert np.abs(gd[i] - wEh[i] * gEr).max() <= 2e-3 * np.abs(wEh[i] * gEr).max() + 1e-12
        gx_ref += wEh[i] * gEx
        # dE/dr is the reference refinement's gradient (stored distances, unit normals)
        ref = adj.refine_gradient(hits, x64, r, m.vert_mass)
        assert np.abs(gEr - ref).max() <= 2e-3 * np.abs(ref).max() + 1e-12
    assert np.abs(gx - gx_ref).max() <= 2e-3 * np.abs(gx_ref).max()


@pytest.mark.parametrize("n,seed", [(32, 0), (128, 1)])
def test_adjoint_objective_subgradient(u26ctx, n, seed):
    """dJ/dx and dJ/dr run through one maximal hit: 2 A D d(delta_h). Near-ties between fp32
    and FP64 distances may pick different maxima, so the GPU gradient must equal the FP64
    gradient through one of the hits within 1e-4 D of the maximum."""
    m, res, sup = _support(u26ctx, n, seed)
    dev = torch.device("cuda", u26ctx.device)
    x64 = m.x.astype(np.float64)
    for i, c in list(enumerate(sup.contours))[:8]:
        x = torch.from_numpy(m.x).to(dev).requires_grad_(True)
        dirs = sup.dirs.clone().requires_grad_(True)
        J, E = JFunction.apply(x, dirs, sup)
        J[i].backward()
        gx, gd = x.grad.cpu().numpy(), dirs.grad.cpu().numpy()
        hits, r, mc = _fp64(m, res, c)
        A = sum(adj.source_area(h, *mc[:3]) for h in hits)
        ds = [adj.delta(h, x64[adj.hit_vertices(h)], r) for h in hits]
        D = max(ds)
        best = np.inf
        for h, d in zip(hits, ds):
            if d < D - 1e-4 * abs(D):
                continue
            V = adj.hit_vertices(h)
            gP, gr = adj.delta_grads(h, x64[V], r)
            ref = np.zeros_like(x64)
            np.add.at(ref, V, 2 * A * d * gP)
            err = max(np.abs(gx - ref).max() / (np.abs(ref).max() + 1e-30), np.abs(gd[i] - 2 * A * d * gr).max() / (np.abs(2 * A * d * gr).max() + 1e-30))
            best = min(best, err)
        assert best <= 2e-3, (c, best)
        if len(gd) > 1:
            assert np.abs(np.delete(gd, i, axis=0)).max() == 0.0


def test_adjoint_forward_matches_pass_metrics(u26ctx):
    """On the pass's own supports the recomputed J and E agree with the pass's objective and
    displacement cost (which used the ray-cast distances) to fp32 accuracy."""
    m, res, sup = _support(u26ctx, 32, 0)
    J, E = JFunction.apply(torch.from_numpy(m.x).cuda(u26ctx.device), sup.dirs, sup)
    for i, c in enumerate(sup.contours):
        assert abs(float(J[i]) - float(res.results[c]["objective"])) <= 1e-3 * abs(float(res.results[c]["objective"]))
        assert abs(float(E[i]) - float(res.results[c]["displacement_cost"])) <= 1e-3 * abs(float(res.results[c]["displacement_cost"]))
