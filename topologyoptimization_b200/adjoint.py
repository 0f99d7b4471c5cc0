"""Differentiable SIMP objective: a torch.autograd.Function over tpo_forward_dev /
tpo_backward_dev.

    J = FEObjective.apply(x, problem, design, solve_opts, l)

x is the FP64 design on the device (reference element order).  The forward pass filters
it (density filter of radius design.filter_radius), builds E = Emin + xPhys^p (E0 - Emin)
and the multigrid hierarchy, solves K u = F and returns J = l.u (the compliance F.u when
l is None).  The backward pass is the hand-written adjoint: for the compliance it needs
no second solve (lambda = u); for any other l it solves K lambda = l, forms
dJ/dxPhys_e = -p xPhys_e^(p-1) (E0 - Emin) lambda_e^T Ke u_e on the device and applies
the filter transpose.  The reference has only the compliance sensitivity
(js/optimizer-worker-3d.js:2175-2192, with E0 in place of E0 - Emin and no filter
transpose); the displacement objective with an output spring (Problem.set_spring) is
the compliant-mechanism case.
"""
from . import _native as N


def _torch():
    import torch
    return torch


def design_opts(penal=3.0, E0=1.0, Emin=1e-9, filter_radius=1.5):
    return N.DesignOpts(penal=penal, E0=E0, Emin=Emin, filter_radius=filter_radius)


def _make_function():
    torch = _torch()

    class FEObjective(torch.autograd.Function):
        """forward(ctx, x, problem, design, solve_opts, l=None) -> J (0-d FP64 tensor)."""

        @staticmethod
        def forward(ctx, x, problem, design, solve_opts, l=None):
            x = x.detach().contiguous().double()
            J, info = problem.forward_dev(x, design, solve_opts, d_l=l)
            ctx.problem, ctx.solve_opts, ctx.l = problem, solve_opts, l
            ctx.nel = x.numel()
            ctx.info = info
            return torch.tensor(J, dtype=torch.float64, device=x.device)

        @staticmethod
        def backward(ctx, gJ):
            grad = torch.empty(ctx.nel, dtype=torch.float64, device=gJ.device)
            ctx.problem.backward_dev(grad, ctx.solve_opts, d_l=ctx.l)
            return gJ * grad, None, None, None, None

    return FEObjective


_fn = None


def FEObjective():
    """The torch.autograd.Function class (built on first use so that importing the package
    does not import torch)."""
    global _fn
    if _fn is None:
        _fn = _make_function()
    return _fn
