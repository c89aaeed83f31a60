"""Kubo.PDOS: the atom and layer selections of CalcKubo (host, CPU tests) against the oracle's literal
restatement, and the batched local / layer DOS recursions (GPU tests) against the oracle's recursion
from the reference's start vectors."""
import numpy as np
import pytest

import refcases as R
from oracle import oracle as orc
from oracle import pdos as OP

G = pytest.importorskip("grabnes_b200")

GRAPHENE = dict(kind=G.CELL_GRAPHENE, aG=2.46, cell_size=12, super_cell=3)
TBG = dict(kind=G.CELL_TBG_MOIRE, aG=2.46, cell_size=50, super_cell=2, m=(9, 8, 8, 9), height=40.0, d_interlayer=3.35)


def _params(mode, cell, **kw):
    p = G.Pdos()
    p.mode = mode
    p.xmin, p.xmax, p.ymin, p.ymax = kw.get("xmin", 0.0), kw.get("xmax", 5.0), kw.get("ymin", 0.0), kw.get("ymax", 5.0)
    p.min_value = kw.get("min_value", 0)
    p.super_cell, p.cell_size = cell["super_cell"], cell["cell_size"]
    p.supermoire_length = kw.get("supermoire_length", 135.0)
    p.aG = cell["aG"]
    p.ignore_layers_1_4 = int(kw.get("ignore_layers_1_4", False))
    for k, v in enumerate(kw.get("atom_list", (1, 2, 3, 4, 5, 6))):
        p.atom_list[k] = v
    p.atom_number = kw.get("atom_number", 1)
    p.pnp_delta = kw.get("pnp_delta", 10.0)
    p.number_of_layers = kw.get("number_of_layers", 2)
    p.stack = kw.get("stack", 0)
    p.n_bn1, p.n_bn2, p.n_c = kw.get("n_bn1", 5832), kw.get("n_bn2", 5832), kw.get("n_c", 6050)
    return p


ATOM_CASES = {
    "dist": (GRAPHENE, OP.DIST, dict(xmin=2.0, xmax=20.0, ymin=1.0, ymax=15.0, min_value=10)),
    "sc1": (GRAPHENE, OP.MOIRE_SC1, dict(min_value=10)),
    "supermoire": (GRAPHENE, OP.SUPERMOIRE, dict(supermoire_length=12.0)),
    "supermoire2": (GRAPHENE, OP.SUPERMOIRE2, dict(supermoire_length=12.0, min_value=3)),
    "supermoire3": (GRAPHENE, OP.SUPERMOIRE3, dict(supermoire_length=12.0)),
    "supermoire_default": (GRAPHENE, OP.SUPERMOIRE, dict()),
    "atom_list": (GRAPHENE, OP.ATOM_LIST, dict(atom_list=(5, 9, 100, 2592, 1, 7))),
    "by_number": (GRAPHENE, OP.BY_NUMBER, dict(atom_number=77)),
    "pnp": (GRAPHENE, OP.PNP, dict(pnp_delta=5.0)),
    "tbg_sc1_ignore14": (TBG, OP.MOIRE_SC1, dict(ignore_layers_1_4=True)),
    "tbg_sc1": (TBG, OP.MOIRE_SC1, dict()),
    "tbg_supermoire": (TBG, OP.SUPERMOIRE, dict(supermoire_length=40.0)),
}


def _cell(cell):
    keys = {k: v for k, v in cell.items()}
    return G.build_cell(**keys)


@pytest.mark.parametrize("name", sorted(ATOM_CASES))
def test_atom_selection_matches_oracle(name):
    cell, mode, kw = ATOM_CASES[name]
    c = _cell(cell)
    atoms, coords = G.pdos_atoms(_params(mode, cell, **kw), c["rat"], c["species"], c["layer"], c["ucell"])
    ref = OP.select_atoms(mode, c["rat"], c["species"], c["layer"], c["ucell"], super_cell=cell["super_cell"],
                          cell_size=cell["cell_size"], aG=cell["aG"], **kw)
    assert len(ref) > 0
    assert [int(a) for a in atoms] == [i for i, _ in ref]
    for (i, vals), xyz in zip(ref, coords):
        k = 2 if mode == OP.MOIRE_SC1 else 3   # the SC1 coords line holds x, y, species, layer
        assert np.array_equal(np.asarray(vals[:k], np.float64).view(np.int64), xyz[:k].view(np.int64)), i


SET_CASES = {
    "layers": (OP.LAYER, dict(number_of_layers=2)),
    "layers_renormalised": (OP.LAYER, dict(number_of_layers=3)),
    "layers_t3bg": (OP.LAYER, dict(number_of_layers=2, stack=2, n_c=100)),
    "layers_encapsulated": (OP.LAYER, dict(number_of_layers=4, stack=1, n_bn1=10, n_bn2=20, n_c=30)),
    "layer_species": (OP.LAYER_SPECIES, dict(number_of_layers=2)),
}


@pytest.mark.parametrize("name", sorted(SET_CASES))
def test_layer_sets_match_oracle(name):
    mode, kw = SET_CASES[name]
    c = _cell(TBG)
    so, sl, ss, asm = G.pdos_sets(_params(mode, TBG, **kw), c["species"], c["layer"])
    ref = OP.layer_sets(mode, c["species"], c["layer"], super_cell=TBG["super_cell"], **kw)
    assert len(sl) == len(ref)
    for k, (lay, spc, m, mask) in enumerate(ref):
        assert (sl[k], ss[k], asm[k]) == (lay, spc, m)
        assert np.array_equal(so == k, mask)


# ---------------------------------------------------------------------------------------------- GPU
CASES = {
    "tbg": dict(TypeOfSystem="TwistedBilayerBasedOnMoireCell", MoireCellParameters=(31, 30, 30, 31), SuperCell=1,
                TypeOfBL="Koshino", Hopping=2.7, LatticeParameter=2.4595, Vpppi0=2.7, Vppsigma0=0.48,
                BLdelta=0.319, InterlayerDistance=3.35, LayerNeighbors=100, LayerDistFactor=3.2005),
    "graphene_field": dict(TypeOfSystem="Graphene", CellSize=60, Hopping=2.7, MagFieldInteger=3),
}
_built = {}


def built(name):
    if name not in _built:
        _built[name] = R.build(CASES[name])
    return _built[name]


def _close(a, b, a0, b0, tol=1e-10):
    """a_n, b_n within tol of the spectral scale (a_n vanish identically for a site of a bipartite lattice
    without on-site terms, so they cannot set the scale)."""
    scale = max(np.abs(a0).max(), np.abs(b0).max())
    return np.abs(a - a0).max() <= tol * scale and np.abs(b - b0).max() <= tol * scale


@pytest.fixture(scope="module")
def ctx():
    with G.Context(0) as c:
        yield c


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_local_dos_batch_matches_oracle(ctx, name):
    """37 single-atom start vectors (two tiles of right-hand sides), FP64, 150 steps."""
    r = built(name)
    n = r["geo"]["n"]
    sites = np.unique(np.r_[1, n, np.random.default_rng(3).integers(1, n + 1, 35)])
    ctx.load_hamiltonian(r["nb"]["nneigh"], r["nb"]["nlist"], r["hop"], r["h0"])
    a, b = ctx.lanczos_sites(sites, 150, G.GBN_FP64)
    for k, i in enumerate(sites):
        a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], OP.site_start_vector(n, int(i)), 150, 0)
        assert _close(a[k], b[k], a0, b0), i


@pytest.mark.gpu
def test_local_dos_mixed_precision(ctx):
    """FP32 storage of vectors and hoppings: a single-site DOS is not averaged over the cell as a
    random-phase one is, and its normalised L1 error after 150 steps is about 1.2e-5 here, hence the
    bar of 1e-4 (the FP64 path is the reference-exact one)."""
    r = built("tbg")
    n, g0 = r["geo"]["n"], r["g0"]
    sites = np.array([1, 17, 5000, n])
    ctx.load_hamiltonian(r["nb"]["nneigh"], r["nb"]["nlist"], r["hop"], r["h0"])
    a, b = ctx.lanczos_sites(sites, 150, G.GBN_MIXED)
    for k, i in enumerate(sites):
        a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], OP.site_start_vector(n, int(i)), 150, 0)
        _, d0 = orc.frac(a0, b0, 0.05 / g0, 400, -1.5 / g0, 1.5 / g0)
        _, d = orc.frac(a[k], b[k], 0.05 / g0, 400, -1.5 / g0, 1.5 / g0)
        assert np.abs(d - d0).sum() <= 1e-4 * np.abs(d0).sum(), i


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(SET_CASES))
def test_layer_dos_batch_matches_oracle(ctx, name):
    mode, kw = SET_CASES[name]
    r = built("tbg")
    geo = r["geo"]
    n = geo["n"]
    p = _params(mode, dict(super_cell=1, cell_size=50, aG=2.4595), **kw)
    so, sl, ss, asm = G.pdos_sets(p, geo["species"], geo["layer"])
    u = orc.rng_draws(1235, n)
    ctx.load_hamiltonian(r["nb"]["nneigh"], r["nb"]["nlist"], r["hop"], r["h0"])
    a, b = ctx.lanczos_sets(so, u, asm, 150, G.GBN_FP64)
    for k in range(len(sl)):
        mask = so == k
        if not mask.any():   # an empty layer: no DOS (the reference divides by a zero norm)
            assert np.isnan(a[k]).all() and np.isnan(b[k]).all()
            continue
        psi = OP.layer_start_vector(mask, asm[k], u)
        a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], psi, 150, 0)
        assert _close(a[k], b[k], a0, b0), (sl[k], ss[k])
