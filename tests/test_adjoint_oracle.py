"""The DOS-loss gradient of the library (gbn_dos_gradient, FP64, and its FP32-vector variant) against an
independent FP64 reference gradient: central differences (h = 1e-6 relative; Richardson-extrapolated
steps of 2e-3 and 4e-3 for the much smaller w derivative) of the loss computed
entirely by the oracle -- its own geometry, neighbour tables and hoppings with the smooth interlayer
cutoff (orc_hopping), the reference's three-pass recursion (KuboRecursion, kubosubs.F90:26-138) and
continued fraction (KuboFrac, kubosubs.F90:222-288).  Nothing of the library's assembly, recursion or
continued fraction enters the reference, so an error shared by the library's forward pass and its
adjoint cannot cancel.

Cases: the 1.08 degree twisted bilayer cell (11 164 atoms, 80 steps), a scaled copy of the gradient
workload (1.05 degree cell tiled 3 x 3 = 107 172 atoms, 600 steps, checkpoints every 32, eta 5 meV,
2001 energies), and the gradient workload itself (tiled 9 x 9 = 964 548 atoms).  The loss parameters
theta = (t, Vpp_sigma0, delta, w); the target DOS is the oracle's at theta perturbed by 2 % (seed 3).
"""
import math

import numpy as np
import pytest

import refcases as R
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

G = pytest.importorskip("grabnes_b200")
from grabnes_b200 import autograd as AD  # noqa: E402
from grabnes_b200 import model as M  # noqa: E402

THETA0 = np.array([2.7, 0.48, 0.319, 0.5])


def _keys(m, super_cell):
    short = dict(TypeOfSystem="TwistedBilayerBasedOnMoireCell", MoireCellParameters=m, SuperCell=super_cell,
                 TypeOfBL="Koshino", Vpppi0=2.7, Vppsigma0=0.48, BLdelta=0.319, LayerNeighbors=100,
                 LayerDistFactor=3.2005, Hopping=2.7, SeedValue=3)
    sect = {"Run.TypeOfSystem": "TwistedBilayerBasedOnMoireCell", "Structure.MoireCellParameters": m,
            "Structure.SuperCell": super_cell, "Interlayer.TypeOfBL": "Koshino", "Interlayer.Vpppi0": 2.7,
            "Interlayer.Vppsigma0": 0.48, "Interlayer.BLdelta": 0.319, "Neigh.LayerNeighbors": 100,
            "Neigh.LayerDistFactor": 3.2005, "TB.Hopping": 2.7, "Kubo.SeedValue": 3}
    return short, sect


class OracleProblem:
    """The same DOS-fitting problem evaluated by the oracle alone."""

    def __init__(self, short_keys, nrecurs, eta_ev, n_en, emin_ev, emax_ev):
        r = R.build(short_keys)
        self.r, self.g0 = r, r["g0"]
        self.base = r["model"]
        self.base.inter_cut_rho = math.sqrt(r["cut2inter"])
        n = r["geo"]["n"]
        self.u = orc.rng_draws(short_keys["SeedValue"], n)
        self.nrecurs, self.n_en = nrecurs, n_en
        self.eta, self.emin, self.emax = eta_ev / self.g0, emin_ev / self.g0, emax_ev / self.g0
        self.target = np.zeros(n_en + 1)

    def model(self, theta):
        m = orc.Model()
        for name, _ in orc.Model._fields_:
            v = getattr(self.base, name)
            if hasattr(v, "__len__"):
                arr = getattr(m, name)
                for i in range(len(arr)):
                    arr[i] = v[i]
            else:
                setattr(m, name, v)
        m.gn_cc[0] = theta[0] / self.g0
        m.vppsigma0 = -theta[1] / self.g0
        m.bl_delta = theta[2]
        m.inter_smooth_w = theta[3]
        return m

    def loss(self, theta):
        """The oracle's loss with a fixed number of OpenMP threads (8), so that its summation order, and with
        it the last bits the central differences of w resolve, does not depend on the machine."""
        r = self.r
        return orc.dos_loss(self.model(theta), r["rat_hop"], r["geo"]["species"], r["geo"]["layer"], r["nb"], r["h0"],
                            self.u, self.nrecurs, self.eta, self.n_en, self.emin, self.emax, self.target, nthreads=8)

    def _cd(self, theta, k, h):
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        return (self.loss(tp)[0] - self.loss(tm)[0]) / (2.0 * h)

    def central_differences(self, theta, rel=1e-6, rel_w=2e-3, spread=False):
        """Central differences with h = 1e-6 theta_k for t, Vpp_sigma0 and delta.  The w derivative is
        three to four orders of magnitude below the others, under the rounding noise that h = 1e-6 meets
        after hundreds of recursion steps (about 5e-6 absolute at 600 steps, the agreement of the large
        components); it is differenced with h = 2e-3 w and 4e-3 w and extrapolated (Richardson), which
        leaves a truncation error of order (h / w)^4 and the noise divided by 2000.  At 5e-4 the noise
        still moved the 107k-atom w difference by 1.4e-5 relative between 8 and 16 threads; at 2e-3 by
        1.2e-6.  With spread, also the same extrapolation at 2.5 times the steps, and returns (fd, the
        difference of the two w values): the resolution of the w reference.  The smooth cutoff is C1 (its
        second derivative jumps where a bond enters the taper), so on large cells, where millions of bonds
        cross the taper's edges as w moves, the differences keep an error that the extrapolation does not
        remove: on the 964,548-atom cell the w values at 2e-3 and 5e-3 differ by 1.1e-5 relative, 40 times
        the thread noise."""
        fd = np.zeros(4)
        for k in range(3):
            fd[k] = self._cd(theta, k, rel * theta[k])
        h = rel_w * theta[3]
        fd[3] = (4.0 * self._cd(theta, 3, h) - self._cd(theta, 3, 2.0 * h)) / 3.0
        if not spread:
            return fd
        h2 = 2.5 * h
        w2 = (4.0 * self._cd(theta, 3, h2) - self._cd(theta, 3, 2.0 * h2)) / 3.0
        return fd, abs(w2 - fd[3])


def _pair(m, super_cell, nrecurs, eta_ev, n_en, emin_ev, emax_ev, checkpoint, ctx):
    short, sect = _keys(m, super_cell)
    op = OracleProblem(short, nrecurs, eta_ev, n_en, emin_ev, emax_ev)
    job = M.job_from_keys(sect)
    assert job["g0"] == op.g0 and job["cut2inter"] == op.r["cut2inter"]
    gp = AD.DosProblem(ctx, job, None, nrecurs, eta_ev, n_en, emin_ev, emax_ev, checkpoint=checkpoint)
    assert gp.n == op.r["geo"]["n"] and np.array_equal(gp.u, op.u)
    rng = np.random.default_rng(3)
    _, target = op.loss(THETA0 * (1.0 + 0.02 * rng.uniform(-1, 1, 4)))
    op.target = target
    gp.target = target
    return op, gp


def _check(grad, fd, tol=1e-5, w_spread=0.0):
    """Every component to `tol` relative; w, where the reference's own resolution (w_spread: the difference
    of its values at two step sizes) is coarser, to twice that resolution."""
    print("gradient", grad, "oracle central differences", fd, "relative", np.abs(grad - fd) / np.abs(fd),
          "w spread", w_spread)
    for k in range(4):
        bound = tol * abs(fd[k]) if k < 3 else max(tol * abs(fd[k]), 2.0 * w_spread)
        assert abs(grad[k] - fd[k]) <= bound, (AD.PARAMS[k], grad, fd, w_spread)


@pytest.fixture(scope="module")
def ctx():
    with G.Context(0) as c:
        yield c


@pytest.fixture(scope="module")
def small(ctx):
    return _pair((31, 30, 30, 31), 1, 80, 0.03, 400, -1.0, 1.0, 16, ctx)


def test_loss_and_dos_match_oracle(small):
    """The library's forward pass (assembly with the smooth cutoff, FP64 recursion, continued fraction)
    against the oracle's at theta0: DOS within 1e-10 of its scale, loss within 1e-9 relative."""
    op, gp = small
    l0, d0 = op.loss(THETA0)
    l1, _, d1 = gp.evaluate(THETA0)
    assert np.abs(d1 - d0).max() <= 1e-10 * np.abs(d0).max()
    assert abs(l1 - l0) <= 1e-9 * l0


def test_gradient_matches_oracle_central_differences(small):
    op, gp = small
    _, grad, _ = gp.evaluate(THETA0)
    _check(grad, op.central_differences(THETA0))


def test_fp32_variant_gradient(small):
    """The FP32-vector variant against the FP64 gradient and the oracle's central differences: within
    1e-3 relative per component, the rounding of complex64 vectors over 80 steps."""
    op, gp = small
    _, g64, _ = gp.evaluate(THETA0)
    gp.precision = G.GBN_MIXED
    try:
        l32, g32, _ = gp.evaluate(THETA0)
    finally:
        gp.precision = G.GBN_FP64
    err = np.abs(g32 - g64) / np.abs(g64)
    print("FP32-variant gradient, relative error per component against FP64:", err)
    _check(g32, op.central_differences(THETA0), tol=1e-3)


def test_gradient_scaled_workload(ctx):
    """The gradient workload's parameters (600 steps, checkpoints every 32, eta 5 meV, 2001 energies on
    [-1, 1] eV) on the 1.05 degree cell tiled 3 x 3 (107 172 atoms)."""
    op, gp = _pair((32, 31, 31, 32), 3, 600, 0.005, 2000, -1.0, 1.0, 32, ctx)
    assert gp.n >= 100_000
    _, grad, _ = gp.evaluate(THETA0)
    _check(grad, op.central_differences(THETA0))


def test_gradient_full_workload(ctx):
    """The gradient workload itself: 964 548 atoms, 600 steps, checkpoints every 32 (the bench's
    dos_gradient leg), against the oracle's central differences; t, Vpp_sigma0 and delta to 1e-5 relative,
    w (1e-4 of the largest component) to 1e-5 relative or twice the resolution of its reference."""
    op, gp = _pair((32, 31, 31, 32), 9, 600, 0.005, 2000, -1.0, 1.0, 32, ctx)
    assert gp.n == 964_548
    _, grad, _ = gp.evaluate(THETA0)
    fd, w_spread = op.central_differences(THETA0, spread=True)
    assert w_spread <= 3e-5 * abs(fd[3])   # the reference itself is resolved to a few 1e-5 of w's derivative
    _check(grad, fd, w_spread=w_spread)
