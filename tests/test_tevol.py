"""KuboTEvol on the device (gbn_kubo_tevol) against the same loop run step by step through gbn_kubo_evol
with the states on the host, and against the oracle's KuboEvol loop."""
import numpy as np
import pytest

import refcases as R
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

G = pytest.importorskip("grabnes_b200")


@pytest.fixture(scope="module")
def setup():
    r = R.build(dict(TypeOfSystem="Graphene", CellSize=60, Hopping=2.7, MagFieldInteger=3))
    n = r["geo"]["n"]
    a, b = orc.recursion(r["nb"], r["hop"], r["h0"], orc.init_wf(n, 2), 80, 0)
    ac, bc = orc.interval(a, b)
    c = orc.cheb_coef(2.0, ac, bc, 40)
    psi = np.stack([orc.init_wf(n, 10 + k) for k in range(3)])
    return r, n, ac, bc, c, psi


def _load(ctx, r):
    ctx.load_hamiltonian(r["nb"]["nneigh"], r["nb"]["nlist"], r["hop"], r["h0"])
    ctx.set_neighd(r["nb"]["neighd"])


@pytest.mark.parametrize("prec", [G.GBN_FP64, G.GBN_MIXED])
def test_tevol_matches_step_by_step(setup, prec):
    r, n, ac, bc, c, psi = setup
    with G.Context(0) as ctx:
        _load(ctx, r)
        p1, z1, norms, a1, b1 = ctx.kubo_tevol(c, ac, bc, psi, np.zeros_like(psi), 4, 2, 80, 1, prec)
        p, z = psi.copy(), np.zeros_like(psi)
        for it in range(1, 5):
            p, z = ctx.kubo_evol(c, ac, bc, p, z, direction=1, precision=prec)
            if it % 2:
                continue
            w = it // 2 - 1
            nrm = np.sum(np.abs(z) ** 2, axis=1)
            assert np.abs(norms[:, w] - nrm).max() <= 1e-12 * nrm.max()
            a0, b0 = ctx.lanczos(z / np.sqrt(nrm)[:, None], 80, prec)
            tol = 1e-12 if prec == G.GBN_FP64 else 1e-6
            assert np.abs(a1[:, w] - a0).max() <= tol * np.abs(b0).max()
            assert np.abs(b1[:, w] - b0).max() <= tol * np.abs(b0).max()
        assert np.abs(p1 - p).max() <= 1e-12 and np.abs(z1 - z).max() <= 1e-12 * np.abs(z).max()


def test_tevol_against_oracle(setup):
    r, n, ac, bc, c, psi = setup
    with G.Context(0) as ctx:
        _load(ctx, r)
        _, _, norms, a1, b1 = ctx.kubo_tevol(c, ac, bc, psi[:1], np.zeros_like(psi[:1]), 4, 2, 80, 1, G.GBN_FP64)
    p, z = psi[0].copy(), np.zeros(n, np.complex128)
    for it in range(1, 5):
        p, z = orc.evol(r["nb"], r["hop"], r["h0"], c, ac, bc, p, z, 1)
        if it % 2:
            continue
        w = it // 2 - 1
        nrm = float(np.vdot(z, z).real)
        assert abs(norms[0, w] - nrm) <= 1e-9 * nrm
        a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], z / np.sqrt(nrm), 80, 0)
        assert np.abs(a1[0, w] - a0).max() <= 1e-9 * np.abs(b0).max()
        assert np.abs(b1[0, w] - b0).max() <= 1e-9 * np.abs(b0).max()
