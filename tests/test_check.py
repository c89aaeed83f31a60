"""The Hamiltonian checks at the end of HamHopping (gbn_check_hamiltonian: HamCheckFinite and the pair scan of
HamCheckHermiticity) against the oracle's restatement: counts exact, the largest asymmetry to 1e-12 g0."""
import numpy as np
import pytest

import refcases as R
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

G = pytest.importorskip("grabnes_b200")

MOIRE = dict(TypeOfSystem="Graphene", CellSize=11, SuperCell=4, LatticePercent=-1.0 / 11.0, MoirePotential=True,
             MoireJeil=True, MoireH0AndHZ=True, MoireOffDiag=True)
CASES = {
    "moire_midpoint": dict(MOIRE, MoireOffDiagMidpoint=True, MagFieldInteger=2),
    "moire_first_atom": dict(MOIRE, MagFieldInteger=2),   # not Hermitian: evaluated at the first atom of a bond
    "tbg": dict(TypeOfSystem="TwistedBilayerBasedOnMoireCell", MoireCellParameters=(9, 8, 8, 9), TypeOfBL="Koshino",
                LayerNeighbors=100, LayerDistFactor=3.2005, MagFieldInteger=1),
}


@pytest.fixture(scope="module")
def ctx():
    with G.Context(0) as c:
        yield c


@pytest.mark.parametrize("name", sorted(CASES))
def test_checks_match_oracle(ctx, name):
    r = R.build(CASES[name])
    geo = r["geo"]
    ctx.set_geometry(geo["rat"], geo["species"], geo["layer"], geo["ucell"])
    ctx.neighbours(r["cut2intra"], r["cut2inter"], r["second_layer"], tables=False)
    ctx.assemble(R.gpu_model(r["model"]), r["rat_on"], r["rat_hop"], None)
    if r["flux"] != 0.0:
        ctx.peierls(r["flux"])
    got = ctx.check_hamiltonian()
    ref = orc.check_hamiltonian(r["nb"], r["hop"], r["h0"])
    assert got[:5] == ref[:5]
    assert abs(got[5] - ref[5]) <= 1e-12
    if name == "moire_first_atom":
        assert got[5] > 1e-6
    else:
        assert got[5] <= 1e-12


def test_checks_find_non_finite_values(ctx):
    r = R.build(dict(TypeOfSystem="Graphene", CellSize=10))
    nb, geo = r["nb"], r["geo"]
    hop, h0 = r["hop"].copy(), r["h0"].copy()
    hop[5, 1] = complex(np.nan, 0.0)
    h0[9] = np.inf
    ctx.set_geometry(geo["rat"], geo["species"], geo["layer"], geo["ucell"])
    ctx.load_hamiltonian(nb["nneigh"], nb["nlist"], hop, h0)
    ctx.set_images(nb["ncell"])
    got = ctx.check_hamiltonian()
    ref = orc.check_hamiltonian(nb, hop, h0)
    assert got[:5] == ref[:5] and got[0] == 1 and got[1] == 1 and got[2] == 6
