"""torch.autograd binding of the PRP objective over fixed supports (u26_prp_adjoint).

JFunction.apply(x, dirs, support) -> (J, E), one value per contour:
    J = (sum of the support's rest source areas) * (max_h delta_h)^2   (the penetration objective)
    E = sum_h (delta_h + 3e-3)^2 / kappa_h                             (the displacement cost)
with every hit distance recomputed from the positions x [V, 3] and the directions dirs [C, 3]
as delta = (w . n) / (r . n) on the supports S(r) of a u26_prp_resolve pass (held fixed: the
function is the smooth branch of the objective around the pass). backward gives dJ/dx, dE/dx
(dense [V, 3]) and dJ/dr, dE/dr through one hand-written adjoint kernel; dE/dr is the
gradient the reference's direction refinement uses (intersection_resolver2.cpp:1268-1320).
There is no CPU path: the tensors live on the context's CUDA device.
"""
import ctypes

import numpy as np
import torch

from . import _native as nat
from .prp import HIT_DTYPE


class Support:
    """The selected hits of one PRP pass as device tensors, with the mesh constants the
    objective reads (rest areas, vertex masses)."""

    def __init__(self, ctx, result, mesh, contours=None):
        dev = torch.device("cuda", ctx.device)
        idx = range(len(result.hits)) if contours is None else contours
        self.contours = list(idx)
        hits = [result.hits[c] for c in self.contours]
        off = np.zeros(len(hits) + 1, np.uint32)
        for i, h in enumerate(hits):
            off[i + 1] = off[i] + len(h)
        flat = np.concatenate(hits) if hits else np.zeros(0, HIT_DTYPE)
        raw = np.frombuffer(flat.tobytes(), np.uint8) if len(flat) else np.zeros(HIT_DTYPE.itemsize, np.uint8)
        self.ctx = ctx
        self.hits = torch.from_numpy(raw.copy()).to(dev)
        self.offsets = torch.from_numpy(off.astype(np.int32)).to(dev)
        self.vert_area = torch.from_numpy(mesh.rest_vert_area.astype(np.float32)).to(dev)
        self.edge_area = torch.from_numpy(mesh.rest_edge_area.astype(np.float32)).to(dev)
        self.face_area = torch.from_numpy(mesh.rest_face_area.astype(np.float32)).to(dev)
        self.vert_mass = torch.from_numpy(mesh.vert_mass.astype(np.float32)).to(dev)
        self.num_contours = len(hits)
        self.num_hits = int(off[-1])
        self.dirs = torch.from_numpy(np.stack([result.results[c]["dir"] for c in self.contours]).astype(np.float32)
                                     if hits else np.zeros((0, 3), np.float32)).to(dev)

    def launch(self, x, dirs, J=None, E=None, gJ=None, gE=None, grad_dirs=None, grad_x=None):
        p = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None
        st = self.ctx.lib.u26_prp_adjoint(self.ctx.handle, p(x), p(self.hits), p(self.offsets), self.num_contours, p(dirs),
                                          p(self.vert_area), p(self.edge_area), p(self.face_area), p(self.vert_mass), p(J), p(E),
                                          p(gJ), p(gE), p(grad_dirs), p(grad_x))
        self.ctx.check(st, "u26_prp_adjoint")


class JFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, dirs, support):
        x = x.detach().contiguous().float()
        dirs = dirs.detach().contiguous().float()
        J = torch.empty(support.num_contours, device=x.device, dtype=torch.float32)
        E = torch.empty_like(J)
        support.launch(x, dirs, J=J, E=E)
        ctx.save_for_backward(x, dirs)
        ctx.support = support
        return J, E

    @staticmethod
    def backward(ctx, gJ, gE):
        x, dirs = ctx.saved_tensors
        s = ctx.support
        gJ = gJ.contiguous().float() if gJ is not None else None
        gE = gE.contiguous().float() if gE is not None else None
        grad_x = torch.zeros_like(x)
        grad_dirs = torch.empty_like(dirs)
        s.launch(x, dirs, gJ=gJ, gE=gE, grad_dirs=grad_dirs, grad_x=grad_x)
        return grad_x, grad_dirs, None


def objective(x, dirs, support):
    """(J, E) per contour of `support`, differentiable in x and dirs."""
    return JFunction.apply(x, dirs, support)
