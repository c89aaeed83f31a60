"""Cell and atom positions of the library (host code behind the C ABI) against the oracle's CellGet /
AtomsConstruct / AtomsSetCart restatement, bitwise.

gbn_cell_atoms, gbn_build_cell and gbn_cart_roundtrip replace lanczosKuboCode/Src/cell.F90:108-140,
207-240 and atoms.F90:124-230, 330-380, 1506-1607, 1768-1794 (the fractional/Cartesian round trip the
moire routines make).  The positions feed the neighbour search, whose tables are compared bit-exactly
on the GPU, so the positions themselves must agree to the last bit: rat is compared as int64 words,
species, layer and the cell exactly.  The cases are the workloads' own cells: pristine graphene
200 x 200 (80,000 atoms), example 06's graphene/hBN supercell (CellSize 55, SuperCell 8), the twisted
bilayer (31, 30, 30, 31) tiled 2 x 2, and example 07's 0.61 degree cell (CellSize 83, SuperCell 16,
3,527,168 atoms).
"""
import numpy as np
import pytest

from oracle import oracle as orc

G = pytest.importorskip("grabnes_b200")

CELLS = {
    "graphene_200": dict(kind=0, aG=2.4595, cell_size=200, super_cell=1),
    "example06_55x8": dict(kind=0, aG=2.46, cell_size=55, super_cell=8),
    "tbg_31_30_30_31_x2": dict(kind=1, aG=2.4595, super_cell=2, m=(31, 30, 30, 31), d_interlayer=3.35),
    "example07_83x16": dict(kind=0, aG=2.46, cell_size=83, super_cell=16),
    # the moire cell with its second layer offset (Structure.TwistedBLAddShift, atoms.F90:352-366): an AB
    # (Bernal) bilayer, and a twisted cell with the bridge offset plus 0.3 A along a1+a2
    "ab_bilayer_6060_x4_bernal": dict(kind=1, aG=2.46, super_cell=4, m=(6, 0, 6, 0), d_interlayer=3.34, add_shift=1),
    "tbg_3223_x3_bridge": dict(kind=1, aG=2.46, super_cell=3, m=(3, 2, 2, 3), d_interlayer=3.34, add_shift=2,
                               shift_factor=0.3),
}


def _bits(x):
    return np.ascontiguousarray(x, np.float64).view(np.int64)


@pytest.mark.parametrize("name", sorted(CELLS))
def test_cell_and_atoms_bitwise(name):
    p = CELLS[name]
    ref = orc.geometry(**p)
    got = G.build_cell(**p)
    assert got["n"] == ref["n"]
    assert np.array_equal(_bits(got["ucell"]), _bits(ref["ucell"]))
    assert np.array_equal(_bits(got["rat"]), _bits(ref["rat"]))
    assert np.array_equal(got["species"], ref["species"])
    assert np.array_equal(got["layer"], ref["layer"])
    assert np.array_equal(_bits([got["twist"]]), _bits([ref["twist"]]))


@pytest.mark.parametrize("name", sorted(CELLS))
def test_cartesian_roundtrip_bitwise(name):
    """AtomsSetFrac then AtomsSetCart, once and twice (the on-site and the hopping routines each make
    one), on the cell's own positions."""
    p = CELLS[name]
    ref = orc.geometry(**p)
    r1 = G.cart_roundtrip(ref["rat"], ref["ucell"])
    o1 = orc.roundtrip(ref["rat"], ref["ucell"])
    assert np.array_equal(_bits(r1), _bits(o1))
    assert np.array_equal(_bits(G.cart_roundtrip(r1, ref["ucell"])), _bits(orc.roundtrip(o1, ref["ucell"])))


def test_cell_rejects_bad_input():
    """An unknown cell kind or a non-positive size is an error, not an abort."""
    with pytest.raises(G.GbnError):
        G.build_cell(kind=7)
    with pytest.raises(G.GbnError):
        G.build_cell(kind=0, cell_size=0)
