"""Parity of the CUDA library (through its C ABI) with the oracle, on a B200.

Bars (from the task's contract): neighbour and index arrays bit-exact; NeighD bitwise; FP64 Lanczos
a_n, b_n within 1e-10 relative for the first 200 steps; hoppings and on-site energies to 1e-13 g0
(the device's sin/cos/exp differ from glibc's in the last bit); continued fraction to 1e-12.
"""
import math

import numpy as np
import pytest

import refcases as R
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

G = pytest.importorskip("grabnes_b200")

MOIRE = dict(MoirePotential=True, MoireJeil=True, MoireH0AndHZ=True, MoireOffDiag=True, MoireOffDiagMidpoint=True)
# Sizes are chosen so that 200 Lanczos steps stay below the onset of the recursion's sensitivity to
# rounding: in small, highly symmetric cells the spectrum is degenerate and two FP64 runs that differ
# only in summation order part ways after 120-150 steps (measured with the oracle, 1 vs 8 threads).
CASES = {
    # pristine graphene, nearest neighbours (config 1 model)
    "graphene": dict(TypeOfSystem="Graphene", CellSize=100, Hopping=2.7, LatticeParameter=2.4595),
    # graphene/hBN effective moire model with a field (config 3 model, example 06 at small size)
    "moire_field": dict(TypeOfSystem="Graphene", CellSize=11, SuperCell=4, LatticePercent=-1.0 / 11.0,
                        MagFieldInteger=2, **MOIRE),
    # twisted moire model (example 07 model at small size)
    "moire_twist": dict(TypeOfSystem="Graphene", CellSize=27, SuperCell=2, LatticePercent=-0.017989,
                        MoireTwisted=True, MoireTwistAngle=1.872, **MOIRE),
    # twisted bilayer, two-centre interlayer, 5 A in-plane interlayer radius (config 2 model)
    "tbg": dict(TypeOfSystem="TwistedBilayerBasedOnMoireCell", MoireCellParameters=(31, 30, 30, 31), SuperCell=1,
                TypeOfBL="Koshino", Hopping=2.7, LatticeParameter=2.4595, Vpppi0=2.7, Vppsigma0=0.48,
                BLdelta=0.319, InterlayerDistance=3.35, LayerNeighbors=100, LayerDistFactor=3.2005),
    # example 08's twisted bilayer model: F2G2 intralayer to the fifth shell, on-site 0.4914 eV, KoshinoSR
    # two-centre interlayer to 6.25 A in plane, coupling renormalised by 1.008
    "tbg_sr": dict(TypeOfSystem="TwistedBilayerBasedOnMoireCell", MoireCellParameters=(31, 30, 30, 31), SuperCell=1,
                   TypeOfBL="Koshino", Hopping=3.5, OnSiteC=0.4914, NeighLevels=5, InterlayerDistance=3.35,
                   LayerNeighbors=400, LayerDistFactor=4.0, KoshinoSR=True, RenormalizeCoupling=True,
                   CouplingFactor=1.008),
    # Anderson disorder (config 5 model) on graphene
    "anderson": dict(TypeOfSystem="Graphene", CellSize=30, Anderson=True, AndersonAmp=1.0, SeedValue=5),
    # a second moire on the same graphene (Moire.AddSecondMoire): twisted, scaled mismatch, shifted, mass factor
    # < 0 (flip, Im flip, del(2)/del(3) swap), bond terms at the midpoints, with Anderson disorder (added before
    # the moire terms)
    "moire_second": dict(TypeOfSystem="Graphene", CellSize=11, SuperCell=4, LatticePercent=-1.0 / 11.0,
                         MoireAddSecondMoire=True, MoireTwisted2=True, MoireTwistAngle2=0.7, LatticepercentFactor=1.3,
                         MoireLayerShift2=0.9, MoireSecondMoireMassFactor=-1.0, Anderson=True, AndersonAmp=0.2,
                         SeedValue=9, **MOIRE),
    # the encapsulated bilayer (MoireEncapsulatedBilayerBasedOnMoireCell) on an AB cell: Bernal offset, the
    # bilayer F2G2 interlayer set on the dimer sites found from the structure, the bilayer moire on-site model
    # with bottom / top angles and layer shifts, its bond terms, Anderson disorder
    "enc_bernal": dict(TypeOfSystem="MoireEncapsulatedBilayerBasedOnMoireCell", MoireCellParameters=(6, 0, 6, 0),
                       SuperCell=4, TwistedBLAddShift=True, BernalShift=True, InterlayerDistance=3.34,
                       TypeOfBL="Koshino", NeighLevels=5, LayerNeighbors=100, LayerDistFactor=3.2,
                       MoirePotential=True, MoireJeil=True, MoireH0AndHZ=True, MoireOffDiag=True,
                       LatticePercent=-0.0166, MoireBilayerBottomAngle=0.4, MoireBilayerTopAngle=-0.9,
                       MoireBilayerBottomXShift=0.3, MoireBilayerBottomYShift=-0.2, MoireBilayerTopXShift=0.5,
                       MoireBilayerTopYShift=0.7, Anderson=True, AndersonAmp=0.1, SeedValue=4),
    # a twisted encapsulated cell (the vertical pairs only, as the reference falls back to), the top shift
    # inside the rotation, no moire term on layer 2, bond terms at the midpoints
    "enc_twisted": dict(TypeOfSystem="MoireEncapsulatedBilayerBasedOnMoireCell", MoireCellParameters=(3, 2, 2, 3),
                        SuperCell=6, InterlayerDistance=3.34, TypeOfBL="Koshino", NeighLevels=5, LayerNeighbors=100,
                        LayerDistFactor=3.2, MoirePotential=True, MoireJeil=True, MoireOnlyHZ=True, MoireOffDiag=True,
                        MoireOffDiagMidpoint=True, LatticePercent=-0.018, MoireBilayerTopAngle=1.1,
                        MoireBilayerTopYShift=0.6, MoireBilayerBottomXShift=-0.4, MoireSecondMoireRotateFirst=False,
                        MoireBLDeactivateUpperLayer=True, Anderson=True, AndersonAmp=0.1, SeedValue=6),
    # the same without SecondMoireRotateFirst (shift inside the rotation), per-atom bond terms
    "moire_second_norot": dict(TypeOfSystem="Graphene", CellSize=11, SuperCell=4, LatticePercent=-1.0 / 11.0,
                               MoirePotential=True, MoireJeil=True, MoireH0AndHZ=True, MoireOffDiag=True,
                               MoireAddSecondMoire=True, MoireTwisted2=True, MoireTwistAngle2=-0.4,
                               LatticepercentFactor=0.8, MoireLayerShift2=0.5, MoireSecondMoireRotateFirst=False),
}

_built = {}


def built(name):
    if name not in _built:
        _built[name] = R.build(CASES[name])
    return _built[name]


@pytest.fixture(scope="module")
def ctx():
    with G.Context(0) as c:
        yield c


def gpu_pipeline(ctx, r):
    geo = r["geo"]
    ctx.set_geometry(geo["rat"], geo["species"], geo["layer"], geo["ucell"])
    nb = ctx.neighbours(r["cut2intra"], r["cut2inter"], r["second_layer"])
    m = r["model"]
    uni = orc.rng_draws(m.seed, geo["n"]) if m.anderson else None
    ctx.assemble(R.gpu_model(m), r["rat_on"], r["rat_hop"], uni)
    if r["flux"] != 0.0:
        ctx.peierls(r["flux"])
    return nb


@pytest.mark.parametrize("name", sorted(CASES))
def test_neighbour_tables_bit_exact(ctx, name):
    r = built(name)
    nb = gpu_pipeline(ctx, r)
    ref = r["nb"]
    assert nb["max_neigh"] == ref["max_neigh"]
    assert np.array_equal(nb["nneigh"], ref["nneigh"])
    assert np.array_equal(nb["nlist"], ref["nlist"])
    assert np.array_equal(nb["ncell"], ref["ncell"])
    assert np.array_equal(nb["neighd"].view(np.int64), ref["neighd"].view(np.int64))  # bitwise


@pytest.mark.parametrize("name", sorted(CASES))
def test_hamiltonian_assembly(ctx, name):
    r = built(name)
    gpu_pipeline(ctx, r)
    h0, hop = ctx.hamiltonian()
    assert np.abs(h0 - r["h0"]).max() <= 1e-13
    assert np.abs(hop - r["hop"]).max() <= 1e-13


@pytest.mark.parametrize("name", ["graphene", "moire_field", "moire_second", "moire_second_norot"])
def test_onsite_bottom_and_top(ctx, name):
    """gbn_get_onsite_layers: H0Bottom (after the first moire's terms) and H0Top (the second moire's) against
    the oracle to 1e-13 g0; both 0 where the model has no moire branch, H0Top 0 without the second moire."""
    r = built(name)
    gpu_pipeline(ctx, r)
    bottom, top = ctx.onsite_layers()
    assert np.abs(bottom - r["h0_bottom"]).max() <= 1e-13
    assert np.abs(top - r["h0_top"]).max() <= 1e-13
    if name == "graphene":
        assert not bottom.any() and not top.any()
    if name.startswith("moire_second"):
        assert np.abs(top).max() > 1e-4


def test_encapsulated_interlayer_branch(ctx):
    """The AB cell takes the bilayer F2G2 set (its dimer coupling tBA0 appears, on the vertical pairs), the
    twisted cell the vertical pairs only (-tAB1), as the reference decides from the dimer sites."""
    for name, value in (("enc_bernal", lambda m: m.tbl[4]), ("enc_twisted", lambda m: -m.tbl[2])):
        r = built(name)
        gpu_pipeline(ctx, r)
        _, hop = ctx.hamiltonian()
        geo, nb = r["geo"], r["nb"]
        lay = geo["layer"]
        n = geo["n"]
        inter = [(i, j) for i in range(n) for j in range(nb["nneigh"][i]) if lay[nb["nlist"][i, j] - 1] != lay[i]]
        vals = {hop[i, j].real for i, j in inter}
        assert value(r["model"]) in vals, name
        if name == "enc_twisted":
            assert vals <= {0.0, -r["model"].tbl[2]}


def _rel(x, y):
    return np.abs(x - y).max() / np.abs(y).max()


@pytest.mark.parametrize("name", sorted(CASES))
def test_lanczos_fp64_dropin(ctx, name):
    """gbn_load_hamiltonian with the oracle's arrays (the Fortran-host drop-in), FP64 recursion."""
    r = built(name)
    n = r["geo"]["n"]
    psi = orc.init_wf(n, 123456)
    a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], psi, 200, 0)
    ctx.load_hamiltonian(r["nb"]["nneigh"], r["nb"]["nlist"], r["hop"], r["h0"])
    a, b = ctx.lanczos(psi, 200, G.GBN_FP64)
    assert _rel(a[0], a0) <= 1e-10 and _rel(b[0], b0) <= 1e-10


@pytest.mark.parametrize("name", ["graphene", "tbg", "moire_field"])
def test_lanczos_full_pipeline_phases(ctx, name):
    """Search + assembly + Peierls + random-phase start vector, all on the device."""
    r = built(name)
    n = r["geo"]["n"]
    psi = orc.init_wf(n, 123456)
    a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], psi, 200, 0)
    gpu_pipeline(ctx, r)
    u = orc.rng_draws(123456, n)
    a, b = ctx.lanczos_phases(u, 200, G.GBN_FP64)
    assert _rel(a[0], a0) <= 1e-10 and _rel(b[0], b0) <= 1e-10


def test_lanczos_batched_matches_single(ctx):
    r = built("tbg")
    n = r["geo"]["n"]
    ctx.load_hamiltonian(r["nb"]["nneigh"], r["nb"]["nlist"], r["hop"], r["h0"])
    u = np.stack([orc.rng_draws(7 + k, n) for k in range(16)])
    a16, b16 = ctx.lanczos_phases(u, 150, G.GBN_FP64)
    for k in (0, 5, 15):
        a1, b1 = ctx.lanczos_phases(u[k], 150, G.GBN_FP64)
        assert _rel(a16[k], a1[0]) <= 1e-10 and _rel(b16[k], b1[0]) <= 1e-10


def test_lanczos_uneven_lengths_and_odd_batch(ctx):
    r = built("graphene")
    n = r["geo"]["n"]
    ctx.load_hamiltonian(r["nb"]["nneigh"], r["nb"]["nlist"], r["hop"], r["h0"])
    u = np.stack([orc.rng_draws(11 + k, n) for k in range(5)])
    steps = np.array([40, 120, 80, 200, 10], np.int32)
    a, b = ctx.lanczos_phases(u, steps, G.GBN_FP64)
    for k in range(5):
        psi = orc.init_wf(n, 11 + k)
        a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], psi, int(steps[k]), 0)
        assert _rel(a[k, :steps[k]], a0) <= 1e-10 and _rel(b[k, :steps[k]], b0) <= 1e-10


def test_continued_fraction(ctx):
    r = built("graphene")
    n = r["geo"]["n"]
    psi = orc.init_wf(n, 1)
    a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], psi, 300, 0)
    g0 = r["g0"]
    e_ref, d_ref = orc.frac(a0, b0, 0.01 / g0, 4000, -9.0 / g0, 9.0 / g0)
    e, d = ctx.cf_dos(a0, b0, 0.01 / g0, 4000, -9.0 / g0, 9.0 / g0)
    assert np.abs(e - e_ref).max() == 0.0
    assert np.abs(d[0] - d_ref).max() <= 1e-12 * np.abs(d_ref).max()


def test_mixed_precision_dos(ctx):
    """Complex FP32 vectors and hoppings with FP64 a_n/b_n: broadened DOS against the FP64 oracle.

    44 656-atom twisted bilayer, 300 steps, eta = 10 meV.  (In a cell ten times smaller the DOS after
    300 steps resolves single levels and even two FP64 runs that differ only in summation order
    disagree at 1e-3; at this size FP32 storage costs about 1e-8.)"""
    r = R.build(dict(CASES["tbg"], SuperCell=2))
    n = r["geo"]["n"]
    psi = orc.init_wf(n, 3)
    g0 = r["g0"]
    a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], psi, 300, 0)
    e, d_ref = orc.frac(a0, b0, 0.01 / g0, 1000, -9.0 / g0, 9.0 / g0)
    ctx.load_hamiltonian(r["nb"]["nneigh"], r["nb"]["nlist"], r["hop"], r["h0"])
    a, b = ctx.lanczos(psi, 300, G.GBN_MIXED)
    _, d = ctx.cf_dos(a, b, 0.01 / g0, 1000, -9.0 / g0, 9.0 / g0)
    l1 = np.abs(d[0] - d_ref).sum() / np.abs(d_ref).sum()
    print("mixed-precision DOS error (normalised L1):", l1)
    assert l1 <= 1e-6, l1


@pytest.mark.parametrize("rpt", [1, 2, 4])
def test_layout_variants_agree(ctx, rpt):
    """Rows per group 1, 2 and 4 of the matrix layout, records staged in shared memory (without a
    prefetch, with the gather-row prefetch into L2 or L1, with the epilogue-row prefetch into L1 or L2,
    with that and the bulk L2 prefetch of u_k rows 1, 2 or 4 sweeps ahead) or read from global memory, for every split of the right-hand sides over threads: the same products
    summed in another order (union columns of a group instead of a row's own columns), so mixed-precision
    a_n, b_n agree to FP32 rounding over 60 steps; a prefetch is only a hint, so every prefetch mode
    gives exactly the results of the staged path without one."""
    r = built("tbg")
    n = r["geo"]["n"]
    ctx.load_hamiltonian(r["nb"]["nneigh"], r["nb"]["nlist"], r["hop"], r["h0"])
    u = np.stack([orc.rng_draws(21 + k, n) for k in range(16)])
    out = []
    try:
        for grp in (1, 2, 4):
            staged_runs = []
            for staged, pf in ((0, 0), (1, 0), (1, 1), (1, 2), (1, 3), (1, 4), (1, 5), (1, 6), (1, 7)):
                ctx.set_tuning(rpt, 0, grp, staged, pf)
                out.append(ctx.lanczos_phases(u, 60, G.GBN_MIXED))
                if staged:
                    staged_runs.append(out[-1])
            for a, b in staged_runs[1:]:
                assert np.array_equal(a, staged_runs[0][0]) and np.array_equal(b, staged_runs[0][1])
    finally:
        ctx.set_tuning()
    for k in range(1, len(out)):
        assert _rel(out[0][0], out[k][0]) <= 1e-6 and _rel(out[0][1], out[k][1]) <= 1e-6


@pytest.mark.parametrize("prec", [G.GBN_MIXED, G.GBN_FP64])
@pytest.mark.parametrize("grp", [1, 2, 4])
def test_kernel_variants_agree(ctx, grp, prec):
    """The product's variants (4 or 8 union columns in flight, staged records with values or with the
    column indices only, registers bounded for 1, 2 or 3 blocks per SM, and in mixed precision the
    tile-local product that gathers from a shared-memory copy of each tile's rows) add each row's products in the same
    order; only the grid, and with it the split of the dot products over blocks, follows the occupancy of
    the variant.  So a_n, b_n agree to the rounding of the sums: 1e-6 relative in mixed precision, 1e-10
    in FP64, and FP64 matches the oracle (1e-10)."""
    r = built("tbg")
    n = r["geo"]["n"]
    ctx.load_hamiltonian(r["nb"]["nneigh"], r["nb"]["nlist"], r["hop"], r["h0"])
    u = np.stack([orc.rng_draws(31 + k, n) for k in range(16)])
    runs = []
    try:
        ctx.set_tuning(0, 0, grp, 1, 4)
        for un, sv, mb, tl in ((4, 1, 1, 0), (8, 1, 1, 0), (4, 0, 1, 0), (8, 0, 1, 0), (8, 1, 2, 0), (8, 1, 3, 0),
                               (8, 0, 3, 0), (8, 1, 1, 1), (8, 1, 2, 1)):
            ctx.set_kernel_variant(un, sv, mb, -1, tl)
            runs.append(ctx.lanczos_phases(u, 200, prec))
    finally:
        ctx.set_tuning()
        ctx.set_kernel_variant()
    tol = 1e-6 if prec == G.GBN_MIXED else 1e-10
    for a, b in runs[1:]:
        assert _rel(a, runs[0][0]) <= tol and _rel(b, runs[0][1]) <= tol
    if prec == G.GBN_FP64:
        psi = np.exp(2j * np.pi * u[0]) / np.sqrt(n)
        a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], psi, 200, 0)
        assert _rel(runs[0][0][0], a0) <= 1e-10 and _rel(runs[0][1][0], b0) <= 1e-10


@pytest.mark.parametrize("name", ["graphene", "moire_twist", "anderson"])
def test_fused_step_single_vector(ctx, name):
    """The fused step with one vector (one right-hand side per thread): FP64 a_n, b_n within 1e-10 of the
    oracle over 200 steps; mixed precision (the default there on low-degree cells): its DOS within three
    times the two-launch mixed path's deviation from the oracle's DOS (these cells are small, and 200
    mixed steps part from FP64 whatever the step form)."""
    r = built(name)
    n, g0 = r["geo"]["n"], r["g0"]
    ctx.load_hamiltonian(r["nb"]["nneigh"], r["nb"]["nlist"], r["hop"], r["h0"])
    u = orc.rng_draws(61, n)[None, :]
    psi = np.exp(2j * np.pi * u[0]) / np.sqrt(n)
    a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], psi, 200, 0)
    try:
        ctx.set_kernel_variant(8, 1, 2, -1, -1, 1)
        a1, b1 = ctx.lanczos_phases(u, 200, G.GBN_FP64)
        a2, b2 = ctx.lanczos_phases(u, 200, G.GBN_MIXED)
        ctx.set_kernel_variant(8, 1, 0, -1, -1, 0)
        a3, b3 = ctx.lanczos_phases(u, 200, G.GBN_MIXED)
    finally:
        ctx.set_kernel_variant()
    assert _rel(a1[0], a0) <= 1e-10 and _rel(b1[0], b0) <= 1e-10
    args = (0.01 / g0, 800, -1.0 / g0, 1.0 / g0)
    _, d0 = orc.frac(a0, b0, *args)
    _, d2 = ctx.cf_dos(a2, b2, *args)
    _, d3 = ctx.cf_dos(a3, b3, *args)
    e2 = np.abs(d2[0] - d0).sum() / np.abs(d0).sum()
    e3 = np.abs(d3[0] - d0).sum() / np.abs(d0).sum()
    print(name, "mixed DOS deviation: fused", e2, "two launches", e3)
    assert e2 <= 3.0 * e3 + 1e-7


def test_fused_step_fp64(ctx):
    """The fused step with FP64 vectors (u_k formed by FP64 FMAs, alpha unrounded): a_n, b_n against the
    oracle within 1e-10 relative over 200 steps, as every FP64 path, and against the FP64 two-launch step;
    layouts of one and two rows per group, 8 and 16 vectors."""
    for name in ("moire_twist", "tbg", "graphene"):
        r = built(name)
        n = r["geo"]["n"]
        ctx.load_hamiltonian(r["nb"]["nneigh"], r["nb"]["nlist"], r["hop"], r["h0"])
        psi0 = None
        for nv, grp in ((16, 1), (8, 2)):
            u = np.stack([orc.rng_draws(51 + k, n) for k in range(nv)])
            try:
                ctx.set_tuning(2, 0, grp, 1, 4)
                ctx.set_kernel_variant(4, 1, 0, -1, -1, 0)
                a2, b2 = ctx.lanczos_phases(u, 200, G.GBN_FP64)
                ctx.set_kernel_variant(4, 1, 2, -1, -1, 1)
                a1, b1 = ctx.lanczos_phases(u, 200, G.GBN_FP64)
            finally:
                ctx.set_tuning()
                ctx.set_kernel_variant()
            assert _rel(a1, a2) <= 1e-10 and _rel(b1, b2) <= 1e-10, (name, nv, grp)
            psi = np.exp(2j * np.pi * u[0]) / np.sqrt(n)
            if psi0 is None or not np.array_equal(psi, psi0):
                a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], psi, 200, 0)
                psi0 = psi
            assert _rel(a1[0], a0) <= 1e-10 and _rel(b1[0], b0) <= 1e-10, (name, nv, grp)


@pytest.mark.parametrize("name", ["tbg", "moire_twist", "graphene"])
@pytest.mark.parametrize("grp,mb", [(1, 2), (2, 2), (2, 1), (4, 1)])
def test_fused_step(ctx, name, grp, mb):
    """The fused step (the update folded into the product: each gathered column forms u_k = v_k - alpha
    u_{k-1} in FP32 with an FP32 alpha, b_k from |v_{k+1}|^2, Re<v_{k+1}, u_k> and b_{k-1}) in mixed
    precision, 137 steps (eager steps, graph replays and a remainder), against the oracle's FP64 recursion:
    a_n, b_n of vector 0 within three times the two-launch mixed path's own deviation (the two round u_k
    differently, so they part in the last bits and drift apart like any two mixed runs), and the DOS
    within the mixed path's bar, 1e-6 normalised L1; one launch per step instead of two."""
    r = built(name)
    n = r["geo"]["n"]
    ctx.load_hamiltonian(r["nb"]["nneigh"], r["nb"]["nlist"], r["hop"], r["h0"])
    u = np.stack([orc.rng_draws(41 + k, n) for k in range(16)])
    nsteps = 137
    try:
        ctx.set_tuning(4, 0, grp, 1, 6)
        ctx.set_kernel_variant(8, 1, mb, -1, -1, 0)
        l0 = ctx.launches
        a2, b2 = ctx.lanczos_phases(u, nsteps, G.GBN_MIXED)
        two = ctx.launches - l0
        ctx.set_kernel_variant(8, 1, mb, -1, -1, 1)
        l0 = ctx.launches
        a1, b1 = ctx.lanczos_phases(u, nsteps, G.GBN_MIXED)
        one = ctx.launches - l0
    finally:
        ctx.set_tuning()
        ctx.set_kernel_variant()
    assert two - one >= nsteps   # the update launches are gone
    psi = np.exp(2j * np.pi * u[0]) / np.sqrt(n)
    a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], psi, nsteps, 0)
    e2 = max(_rel(a2[0], a0), _rel(b2[0], b0))
    e1 = max(_rel(a1[0], a0), _rel(b1[0], b0))
    print(name, grp, mb, "deviation from FP64: two-launch", e2, "fused", e1)
    assert e1 <= 3.0 * e2 + 1e-7
    g0 = r["g0"]
    args = (0.01 / g0, 800, -1.0 / g0, 1.0 / g0)
    _, d0 = orc.frac(a0, b0, *args)
    _, d1 = ctx.cf_dos(a1[:1], b1[:1], *args)
    assert np.abs(d1[0] - d0).sum() <= 1e-6 * np.abs(d0).sum()


@pytest.mark.parametrize("grp", [1, 2, 4])
def test_fp64_every_layout(ctx, grp):
    """FP64 recursion through each matrix layout and matrix path against the oracle (1e-10 relative,
    200 steps)."""
    r = built("tbg")
    n = r["geo"]["n"]
    psi = orc.init_wf(n, 5)
    a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], psi, 200, 0)
    ctx.load_hamiltonian(r["nb"]["nneigh"], r["nb"]["nlist"], r["hop"], r["h0"])
    out = []
    try:
        for staged in (0, 1):
            ctx.set_tuning(0, 0, grp, staged)
            out.append(ctx.lanczos(psi, 200, G.GBN_FP64))
    finally:
        ctx.set_tuning()
    for a, b in out:
        assert _rel(a[0], a0) <= 1e-10 and _rel(b[0], b0) <= 1e-10


def _cheb_setup(r, npol=100, dt=5.0):
    """Spectral bounds from a short recursion and the propagator coefficients (KuboInterval, KuboCn)."""
    n = r["geo"]["n"]
    a, b = orc.recursion(r["nb"], r["hop"], r["h0"], orc.init_wf(n, 3), 150, 0)
    ac, bc = orc.interval(a, b)
    c = orc.cheb_coef(dt, ac, bc, npol)
    return ac, bc, c


def _zstart(n, k):
    return np.stack([orc.init_wf(n, 40 + j) for j in range(k)])


@pytest.mark.parametrize("name", ["moire_field", "tbg", "graphene"])
def test_chebyshev_evolution_fp64(ctx, name):
    """KuboChebyshevEvolve: Chebyshev-evolved states within 1e-9 in norm of the oracle (complex
    hoppings with a field, real two-centre bilayer, graphene), three vectors at once."""
    r = built(name)
    n = r["geo"]["n"]
    ac, bc, c = _cheb_setup(r)
    z0 = _zstart(n, 3)
    ctx.load_hamiltonian(r["nb"]["nneigh"], r["nb"]["nlist"], r["hop"], r["h0"])
    z = ctx.cheb_evolve(c, ac, bc, z0, G.GBN_FP64)
    for k in range(3):
        ref = orc.cheb_evolve(r["nb"], r["hop"], r["h0"], c, ac, bc, z0[k])
        assert np.linalg.norm(z[k] - ref) <= 1e-9 * np.linalg.norm(ref)


@pytest.mark.parametrize("grp", [1, 2, 4])
def test_chebyshev_every_layout(ctx, grp):
    r = built("tbg")
    n = r["geo"]["n"]
    ac, bc, c = _cheb_setup(r)
    z0 = _zstart(n, 1)
    ref = orc.cheb_evolve(r["nb"], r["hop"], r["h0"], c, ac, bc, z0[0])
    ctx.load_hamiltonian(r["nb"]["nneigh"], r["nb"]["nlist"], r["hop"], r["h0"])
    try:
        ctx.set_tuning(0, 0, grp)
        z = ctx.cheb_evolve(c, ac, bc, z0, G.GBN_FP64)
    finally:
        ctx.set_tuning()
    assert np.linalg.norm(z[0] - ref) <= 1e-9 * np.linalg.norm(ref)


def test_chebyshev_mixed_precision(ctx):
    """Complex FP32 propagation with FP64 step arithmetic and accumulation: its error against the FP64
    oracle, 16 vectors of the bilayer (bound 2e-6 in norm, FP32 rounding of psi_n over 100 terms)."""
    r = built("tbg")
    n = r["geo"]["n"]
    ac, bc, c = _cheb_setup(r)
    z0 = _zstart(n, 16)
    ctx.load_hamiltonian(r["nb"]["nneigh"], r["nb"]["nlist"], r["hop"], r["h0"])
    z = ctx.cheb_evolve(c, ac, bc, z0, G.GBN_MIXED)
    for k in (0, 7, 15):
        ref = orc.cheb_evolve(r["nb"], r["hop"], r["h0"], c, ac, bc, z0[k])
        assert np.linalg.norm(z[k] - ref) <= 2e-6 * np.linalg.norm(ref)


@pytest.mark.parametrize("name,direction,zero_zu", [("moire_field", 1, False), ("tbg", 2, False), ("graphene", 1, True)])
def test_kubo_evol_fp64(ctx, name, direction, zero_zu):
    """KuboEvol: psi <- U psi and zupsi <- U zupsi + [U, X] psi within 1e-9 in norm of the oracle, along x
    and y, with complex (field) and real hoppings; zupsi = 0 isolates the commutator term."""
    r = built(name)
    n = r["geo"]["n"]
    ac, bc, c = _cheb_setup(r)
    psi = _zstart(n, 2)
    zu = np.zeros_like(psi) if zero_zu else np.stack([orc.init_wf(n, 70 + j) for j in range(2)])
    ctx.load_hamiltonian(r["nb"]["nneigh"], r["nb"]["nlist"], r["hop"], r["h0"])
    ctx.set_neighd(r["nb"]["neighd"])
    p, z = ctx.kubo_evol(c, ac, bc, psi, zu, direction, G.GBN_FP64)
    for k in range(2):
        pr, zr = orc.evol(r["nb"], r["hop"], r["h0"], c, ac, bc, psi[k], zu[k], direction)
        assert np.linalg.norm(p[k] - pr) <= 1e-9 * np.linalg.norm(pr)
        assert np.linalg.norm(z[k] - zr) <= 1e-9 * np.linalg.norm(zr)


def test_kubo_evol_mixed_precision(ctx):
    """The dual recurrence with complex FP32 vectors (FP64 step arithmetic and accumulations), 8 vectors
    of the bilayer: within 1e-5 in norm of the FP64 oracle."""
    r = built("tbg")
    n = r["geo"]["n"]
    ac, bc, c = _cheb_setup(r)
    psi = _zstart(n, 8)
    zu = np.zeros_like(psi)
    ctx.load_hamiltonian(r["nb"]["nneigh"], r["nb"]["nlist"], r["hop"], r["h0"])
    ctx.set_neighd(r["nb"]["neighd"])
    p, z = ctx.kubo_evol(c, ac, bc, psi, zu, 1, G.GBN_MIXED)
    for k in (0, 7):
        pr, zr = orc.evol(r["nb"], r["hop"], r["h0"], c, ac, bc, psi[k], zu[k], 1)
        assert np.linalg.norm(p[k] - pr) <= 1e-5 * np.linalg.norm(pr)
        assert np.linalg.norm(z[k] - zr) <= 1e-5 * np.linalg.norm(zr)
