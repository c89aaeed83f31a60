"""Host routines of the Chebyshev propagator (KuboInterval, KuboCn) against the oracle (CPU only)."""
import numpy as np
import pytest

import refcases as R
from oracle import oracle as orc

G = pytest.importorskip("grabnes_b200")


@pytest.fixture(scope="module")
def coeffs():
    r = R.build(dict(TypeOfSystem="Graphene", CellSize=30, Hopping=2.7, LatticeParameter=2.4595, MagFieldInteger=3))
    n = r["geo"]["n"]
    return orc.recursion(r["nb"], r["hop"], r["h0"], orc.init_wf(n, 9), 400, 0)


def test_interval_matches_tridiagonal_eigenvalues(coeffs):
    a, b = coeffs
    ac, bc = G.cheb_interval(a, b)
    ac0, bc0 = orc.interval(a, b)
    assert abs(ac - ac0) <= 1e-12 * max(1.0, abs(ac0)) and abs(bc - bc0) <= 1e-12 * bc0


@pytest.mark.parametrize("dt,npol", [(5.0, 100), (4.5408, 150), (0.5, 30), (-2.0, 80)])
def test_coefficients_match_jacobi_quadrature(coeffs, dt, npol):
    a, b = coeffs
    ac, bc = orc.interval(a, b)
    c = G.cheb_coef(dt, ac, bc, npol)
    c0 = orc.cheb_coef(dt, ac, bc, npol)
    assert np.abs(c - c0).max() <= 1e-12


def test_coefficients_unitary_sum():
    """The c_n are the first row of the unitary exp(-i J t) of the Jacobi matrix, so sum |c_n|^2 = 1 once
    the expansion has converged."""
    c = G.cheb_coef(7.0, 0.3, 2.5, 200)
    assert abs(np.sum(np.abs(c) ** 2) - 1.0) <= 1e-13


def test_kubo_msd_arithmetic():
    """gbn_kubo_msd (host code of the library): the mean of the norms over the vectors, the time of each
    write step, MSD / t and the central differences of MSD (from MSD = 0 at t = 0, one-sided at the end)."""
    rng = np.random.default_rng(1)
    norms = rng.uniform(0.5, 2.0, (4, 5)).cumsum(axis=1)
    t, msd, dr, ds = G.kubo_msd(norms, 3, 0.75)
    m = norms.mean(axis=0)
    tt = 0.75 * 3 * np.arange(1, 6)
    assert np.allclose(t, tt, rtol=0, atol=1e-15) and np.allclose(msd, m, rtol=1e-15, atol=0)
    assert np.allclose(dr, m / tt, rtol=1e-15, atol=0)
    mm = np.concatenate([[0.0], m])
    t0 = np.concatenate([[0.0], tt])
    slope = [(mm[k + 2] - mm[k]) / (t0[k + 2] - t0[k]) for k in range(4)] + [(m[4] - m[3]) / (tt[4] - tt[3])]
    assert np.allclose(ds, slope, rtol=1e-14, atol=0)
    with pytest.raises(G.GbnError):
        G.kubo_msd(norms, 0, 0.75)
