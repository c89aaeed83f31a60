"""torch.autograd binding of the DOS-loss gradient (gbn_dos_gradient): a differentiable DOS of a
twisted bilayer with respect to (t, Vpp_sigma0, delta, w).

    problem = DosProblem(ctx, job, target_dos, nrecurs=600, eta_ev=0.005, n_en=2000, emin_ev=-1, emax_ev=1)
    theta = torch.tensor([2.7, 0.48, 0.319, 0.5], dtype=torch.float64, requires_grad=True)
    loss = DosLoss.apply(theta, problem)
    loss.backward()            # theta.grad = dL/d(t [eV], Vpp_sigma0 [eV], delta [Ang], w [Ang])

The forward call assembles the Hamiltonian with theta on the device, runs the FP64 recursion and the
continued fraction, and the reverse sweep of the library returns the gradient at the same time; backward
only scales it by the incoming gradient.
"""
import ctypes as C
import math

import numpy as np

from . import GBN_FP64, Model, build_cell, cart_roundtrip, rng_uniform

PARAMS = ("t", "vppsigma0", "delta", "w")


def model_with(base, g0, theta):
    """A copy of the gbn_model `base` with theta = (t, Vpp_sigma0, delta, w) applied."""
    m = Model()
    C.memmove(C.byref(m), C.byref(base), C.sizeof(Model))
    m.gn_cc[0] = theta[0] / g0
    m.vppsigma0 = -theta[1] / g0
    m.bl_delta = theta[2]
    m.inter_smooth_w = theta[3]
    return m


class DosProblem:
    """The fixed part of a DOS-fitting problem: geometry, neighbour tables, start vector and target."""

    def __init__(self, ctx, job, target, nrecurs, eta_ev, n_en, emin_ev, emax_ev, checkpoint=32, cut_rho=None,
                 precision=None):
        self.ctx, self.job = ctx, job
        self.g0 = job["g0"]
        cell = build_cell(**job["cell"])
        ctx.set_geometry(cell["rat"], cell["species"], cell["layer"], cell["ucell"])
        ctx.neighbours(job["cut2intra"], job["cut2inter"], job["second_layer"], tables=False)
        self.rat_on = self.rat_hop = None
        if job["moire"]:
            self.rat_on = cart_roundtrip(cell["rat"], cell["ucell"])
            self.rat_hop = cart_roundtrip(self.rat_on, cell["ucell"])
        self.n = cell["n"]
        self.u = rng_uniform(job["kubo"]["seed"], self.n)
        self.base = job["model"]
        self.base.inter_cut_rho = math.sqrt(job["cut2inter"]) if cut_rho is None else cut_rho
        self.target = np.ascontiguousarray(target, np.float64) if target is not None else np.zeros(n_en + 1)
        self.nrecurs, self.n_en, self.checkpoint = nrecurs, n_en, checkpoint
        self.eta, self.emin, self.emax = eta_ev / self.g0, emin_ev / self.g0, emax_ev / self.g0
        # GBN_FP64 (default) or GBN_MIXED: the FP32-vector variant of the recursion and its adjoint
        self.precision = GBN_FP64 if precision is None else precision

    def evaluate(self, theta):
        """(loss, gradient [4], DOS [n_en + 1]) at theta."""
        m = model_with(self.base, self.g0, theta)
        uni = self.u if m.anderson else None
        self.ctx.assemble(m, self.rat_on, self.rat_hop, uni)
        loss, grad, dos, _, _ = self.ctx.dos_gradient(m, self.g0, self.u, self.nrecurs, self.eta, self.n_en,
                                                      self.emin, self.emax, self.target, self.checkpoint,
                                                      self.precision)
        return loss, grad, dos


try:
    import torch

    class DosLoss(torch.autograd.Function):
        """L(theta) = sum_E (DOS(E; theta) - target(E))^2 with its gradient from the library's adjoint."""

        @staticmethod
        def forward(fctx, theta, problem):
            th = theta.detach().cpu().to(torch.float64).numpy()
            loss, grad, _ = problem.evaluate(th)
            fctx.save_for_backward(torch.as_tensor(grad, dtype=theta.dtype, device=theta.device))
            return theta.new_tensor(loss)

        @staticmethod
        def backward(fctx, grad_output):
            (grad,) = fctx.saved_tensors
            return grad_output * grad, None
except ImportError:   # the binding needs torch; the rest of the package does not
    DosLoss = None
