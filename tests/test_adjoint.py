"""Gradient of a DOS loss through the recursion and the continued fraction (gbn_dos_gradient, the
torch.autograd binding): against central finite differences of the same loss, and independent of the
checkpoint interval.  Twisted bilayer (1.08 degree cell, 11 164 atoms) with the two-centre interlayer
hopping and a smooth interlayer cutoff of width 0.5 Ang; target DOS from parameters perturbed by 2 %."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

G = pytest.importorskip("grabnes_b200")
torch = pytest.importorskip("torch")
from grabnes_b200 import autograd as AD  # noqa: E402
from grabnes_b200 import model as M  # noqa: E402

KEYS = {"Run.TypeOfSystem": "TwistedBilayerBasedOnMoireCell", "Structure.MoireCellParameters": (31, 30, 30, 31),
        "Structure.SuperCell": 1, "Interlayer.TypeOfBL": "Koshino", "Interlayer.Vpppi0": 2.7,
        "Interlayer.Vppsigma0": 0.48, "Interlayer.BLdelta": 0.319, "Neigh.LayerNeighbors": 100,
        "Neigh.LayerDistFactor": 3.2005, "TB.Hopping": 2.7, "Kubo.SeedValue": 3}
THETA0 = np.array([2.7, 0.48, 0.319, 0.5])
NREC, NEN = 80, 400


@pytest.fixture(scope="module")
def problem():
    with G.Context(0) as ctx:
        job = M.job_from_keys(KEYS)
        p = AD.DosProblem(ctx, job, None, NREC, 0.03, NEN, -1.0, 1.0, checkpoint=16)
        rng = np.random.default_rng(3)
        _, _, target = p.evaluate(THETA0 * (1.0 + 0.02 * rng.uniform(-1, 1, 4)))
        p.target = target
        yield p


def test_gradient_matches_central_differences(problem):
    """Central differences with h = 1e-6 of each parameter: 1e-5 relative, per component, with the
    tolerance of a component no tighter than 1e-7 of the largest one (the w derivative comes from the
    few entries near the cutoff, and is four orders of magnitude below the others, where the finite
    difference itself is at the level of the loss's rounding)."""
    loss, grad, _ = problem.evaluate(THETA0)
    assert loss > 0.0
    fd = np.zeros(4)
    for k in range(4):
        h = 1e-6 * THETA0[k]
        tp, tm = THETA0.copy(), THETA0.copy()
        tp[k] += h
        tm[k] -= h
        fd[k] = (problem.evaluate(tp)[0] - problem.evaluate(tm)[0]) / (2.0 * h)
    scale = np.abs(fd).max()
    for k in range(4):
        assert abs(grad[k] - fd[k]) <= 1e-5 * max(abs(fd[k]), 1e-2 * scale), (AD.PARAMS[k], grad, fd)


def test_checkpoint_interval_does_not_change_the_gradient(problem):
    problem.checkpoint = NREC   # every vector of the forward pass kept
    l1, g1, _ = problem.evaluate(THETA0)
    problem.checkpoint = 3      # recomputed from a checkpoint every 3 steps
    l2, g2, _ = problem.evaluate(THETA0)
    problem.checkpoint = 16
    assert l1 == l2
    assert np.abs(g1 - g2).max() <= 1e-13 * np.abs(g1).max()


def test_torch_autograd_binding(problem):
    theta = torch.tensor(THETA0, dtype=torch.float64, requires_grad=True)
    loss = AD.DosLoss.apply(theta, problem)
    (2.0 * loss).backward()
    _, grad, _ = problem.evaluate(THETA0)
    assert torch.allclose(theta.grad, torch.as_tensor(2.0 * grad), rtol=0, atol=0)
