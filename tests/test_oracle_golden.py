"""The oracle against the reference's own golden data (CPU only).

* Hamiltonian fingerprints of tests/regression/model_survey_reference.json: geometry, neighbour
  search, shell hoppings, effective moire on-site and bond terms (per atom and at the bond
  midpoint, with and without twist), two-centre interlayer hoppings, Peierls phases.
* Recursion DOS of examples/06 (fields m = 2, 16, 64) and examples/07 (0 and 0.61 degrees):
  random-phase start vector from the GNU Fortran intrinsic RNG (seed 123456), Lanczos recursion and
  continued fraction, against tables made by a GNU build, at the reference's own tolerance 1e-5
  states/eV/atom (tests/regression/run_long_examples.sh).
"""
import json
import math
import os

import numpy as np
import pytest

import refcases as R
from oracle import oracle as orc

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FP = json.load(open(os.path.join(GOLDEN, "model_survey_fingerprints.json")))


@pytest.mark.parametrize("case", sorted(FP))
def test_fingerprint(case):
    r = R.build(R.case_keys(case))
    assert R.fingerprint(r["nb"], r["hop"], r["h0"]) == FP[case]


def test_rng_first_draws_are_uniform_and_seeded():
    a = orc.rng_draws(123456, 1000)
    b = orc.rng_draws(123456, 1000)
    c = orc.rng_draws(123457, 1000)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert a.min() >= 0.0 and a.max() < 1.0 and abs(a.mean() - 0.5) < 0.05
    # 53-bit mantissa draws: every value is a multiple of 2^-53
    assert np.all(np.ldexp(a, 53) == np.floor(np.ldexp(a, 53)))


EX06 = dict(TypeOfSystem="Graphene", CellSize=55, SuperCell=8, LatticePercent=-0.018181818181818,
            MoirePotential=True, MoireJeil=True, MoireH0AndHZ=True, MoireOffDiag=True, MoireOffDiagMidpoint=True)


def _dos(keys, n_en, emin, emax, eta, nrec=3000):
    r = R.build(keys)
    g0 = r["g0"]
    psi = orc.init_wf(r["geo"]["n"], 123456)
    a, b = orc.recursion(r["nb"], r["hop"], r["h0"], psi, nrec, 0)
    e, d = orc.frac(a, b, eta / g0, n_en, emin / g0, emax / g0)
    return e * g0, d / g0


@pytest.mark.slow
@pytest.mark.parametrize("col,m", [(2, 2), (3, 16)])
def test_example06_landau_levels(col, m):
    ref = np.loadtxt(os.path.join(GOLDEN, "ex06_dos_fields.txt"))
    e, d = _dos(dict(EX06, MagFieldInteger=m), 601, -0.3, 0.3, 0.004)
    assert np.abs(e - ref[:, 0]).max() < 1e-6
    assert np.abs(d - ref[:, col]).max() < 1e-5


@pytest.mark.slow
def test_example07_twist_0p61():
    ref = np.loadtxt(os.path.join(GOLDEN, "ex07_dos_twists.txt"))
    keys = dict(TypeOfSystem="Graphene", CellSize=83, SuperCell=16, LatticePercent=-0.018016854251615,
                MoireTwisted=True, MoireTwistAngle=0.608806541588, MoirePotential=True, MoireJeil=True,
                MoireH0AndHZ=True, MoireOffDiag=True, MoireOffDiagMidpoint=True)
    e, d = _dos(keys, 1201, -0.6, 0.6, 0.005)
    assert np.abs(d - ref[:, 2]).max() < 1e-5


@pytest.mark.parametrize("case", ["graphene", "eff", "eff+MoireAddSecondMoire", "eff+MoireAddSecondMoire+Twisted2"])
def test_onsite_bottom_and_top(case):
    """H0Bottom and H0Top of HamOnSite (ham.F90:2703, 3639): 0 without the moire branch; with it, H0Bottom is
    the on-site energy after the first moire (the same model without the second moire gives it as H0), and
    H0Top = H0 - H0Bottom is the second moire's term, 0 without one."""
    r = R.build(R.case_keys(case))
    h0, bottom, top = r["h0"], r["h0_bottom"], r["h0_top"]
    if case == "graphene":
        assert not bottom.any() and not top.any()
        return
    first = R.build(R.case_keys("eff"))["h0"]
    assert np.array_equal(bottom, first)
    if r["model"].second_moire:
        assert np.array_equal(top, h0 - bottom) and np.abs(top).max() > 0.0
    else:
        assert np.array_equal(bottom, h0) and not top.any()
