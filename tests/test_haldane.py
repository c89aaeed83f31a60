"""The Haldane second-neighbour term (gbn_haldane, HamHopHaldane) against the oracle's restatement, on
its own, after the Peierls phases of a field, with the paper orientation and with layer control; and the
driver's Haldane phase sweep (HaldPhase.*) against the oracle's recursion."""
import math
import os
import subprocess

import numpy as np
import pytest

import refcases as R
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

G = pytest.importorskip("grabnes_b200")
DRIVER = os.path.join(os.path.dirname(G.__file__), "grabnes")


@pytest.fixture(scope="module")
def ctx():
    with G.Context(0) as c:
        yield c


def _device(ctx, r, model=None):
    geo = r["geo"]
    ctx.set_geometry(geo["rat"], geo["species"], geo["layer"], geo["ucell"])
    ctx.neighbours(r["cut2intra"], r["cut2inter"], r["second_layer"], tables=False)
    ctx.assemble(R.gpu_model(model if model is not None else r["model"]), r["rat_on"], r["rat_hop"], None)
    if r["flux"] != 0.0:
        ctx.peierls(r["flux"])


CASES = {
    "graphene_nnn": (dict(TypeOfSystem="Graphene", CellSize=20, NeighLevels=2), {}),
    "graphene_nnn_field": (dict(TypeOfSystem="Graphene", CellSize=20, NeighLevels=2, MagFieldInteger=3), {}),
    "paper_orientation": (dict(TypeOfSystem="Graphene", CellSize=20, NeighLevels=2, MagFieldInteger=1),
                          dict(paper=True, gn2=-0.07)),
    "tbg_layer2_only": (dict(TypeOfSystem="TwistedBilayerBasedOnMoireCell", MoireCellParameters=(9, 8, 8, 9),
                             TypeOfBL="Koshino", NeighLevels=2, LayerNeighbors=100, LayerDistFactor=3.2005),
                        dict(layer_mask=0b10)),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_haldane_matches_oracle(ctx, name):
    keys, opt = CASES[name]
    r = R.build(keys)
    m = r["model"]
    if "gn2" in opt:   # a second-neighbour hopping of the model itself, for the paper orientation
        m.gn_cc[1] = opt["gn2"]
        r["hop"] = orc.hopping(m, r["rat_hop"], r["geo"]["species"], r["geo"]["layer"], r["nb"])
        if r["flux"] != 0.0:
            r["hop"] = orc.peierls(r["rat_hop"], r["geo"]["ucell"], r["nb"], r["flux"], r["hop"])
    t2, phase = 0.05, 0.7 * math.pi
    ref, miss = orc.haldane(r["geo"]["species"], r["geo"]["layer"], r["nb"], 2.46, t2, phase, r["hop"],
                            opt.get("paper", False), opt.get("layer_mask", 0))
    assert miss == 0
    _device(ctx, r, m)
    ctx.haldane(2.46, t2, phase, opt.get("paper", False), opt.get("layer_mask", 0))
    _, hop = ctx.hamiltonian()
    assert np.abs(hop - ref).max() <= 1e-13
    assert np.abs(hop - r["hop"]).max() > 1e-3   # the term did something


def test_haldane_recursion(ctx):
    """100 steps: the Haldane cell in a field is small and symmetric, and two FP64 recursions whose
    Hamiltonians differ in the last bit (device sincos against glibc) part ways after about 120 steps."""
    r = R.build(dict(TypeOfSystem="Graphene", CellSize=60, NeighLevels=2, MagFieldInteger=2))
    n = r["geo"]["n"]
    hop, _ = orc.haldane(r["geo"]["species"], r["geo"]["layer"], r["nb"], 2.46, 0.1, 0.5, r["hop"])
    a0, b0 = orc.recursion(r["nb"], hop, r["h0"], orc.init_wf(n, 4), 100, 0)
    _device(ctx, r)
    ctx.haldane(2.46, 0.1, 0.5)
    a, b = ctx.lanczos_phases(orc.rng_draws(4, n), 100, G.GBN_FP64)
    scale = max(np.abs(a0).max(), np.abs(b0).max())
    assert np.abs(a[0] - a0).max() <= 1e-10 * scale and np.abs(b[0] - b0).max() <= 1e-10 * scale


def test_driver_haldane_phase_sweep(tmp_path):
    """Haldane.SpecifyRange with HaldPhase 0..4 step 2: one folder per phase (named like a field's, with the
    phase in rad), T2 in eV, Haldane.OppositePhase flipping the sign; 100 recursion steps (small cell)."""
    lines = {"Run.Prefix": "hal", "Run.TypeOfSystem": "Graphene", "Structure.CellSize": 40, "TB.Hopping": 2.7,
             "TB.NeighLevels": 2, "Haldane.NNN": ".true.", "Haldane.SpecifyRange": ".true.", "Haldane.T2": 0.27,
             "Haldane.OppositePhase": ".true.", "HaldPhase.InitialInteger": 0, "HaldPhase.FinalInteger": 4,
             "HaldPhase.Step": 2, "Kubo.RecursionNumber": 100, "Kubo.SeedValue": 3, "Calculate.OnlyDOS": ".true."}
    with open(tmp_path / "Gendata.in", "w") as f:
        for k, v in lines.items():
            f.write(f"{k} {v}\n")
    subprocess.run([DRIVER, "Gendata.in"], check=True, cwd=str(tmp_path), capture_output=True, text=True)
    folders = sorted(d for d in os.listdir(tmp_path) if d.startswith("m0"))
    assert folders == ["m00000_B0.0000", "m00002_B3.1416", "m00004_B6.2832"]
    r = R.build(dict(TypeOfSystem="Graphene", CellSize=40, Hopping=2.7, NeighLevels=2))
    n = r["geo"]["n"]
    for folder, mphi in zip(folders, (0, 2, 4)):
        phase = -(1.0 / 4 * mphi * 2.0 * math.pi)
        hop, _ = orc.haldane(r["geo"]["species"], r["geo"]["layer"], r["nb"], 2.46, 0.27 / 2.7, phase, r["hop"])
        a0, b0 = orc.recursion(r["nb"], hop, r["h0"], orc.init_wf(n, 3), 100, 0)
        a = np.loadtxt(tmp_path / folder / "hal.a0.dat")
        b = np.loadtxt(tmp_path / folder / "hal.b0.dat")
        scale = max(np.abs(a0).max(), np.abs(b0).max())
        assert np.abs(a - a0).max() <= 1e-10 * scale and np.abs(b - b0).max() <= 1e-10 * scale, folder
