"""Many fields in one batch (gbn_lanczos_fields): the Peierls phase of every entry applied from one
field-free matrix -- on the fly by every thread (the default), or through a table of each tile's
rotations built before its steps -- against the oracle's per-field Hamiltonian (HamPeierlsPeriodicGauge for each
field) and recursion."""
import numpy as np
import pytest

import refcases as R
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

G = pytest.importorskip("grabnes_b200")

MOIRE = dict(TypeOfSystem="Graphene", CellSize=11, SuperCell=8, LatticePercent=-1.0 / 11.0, MoirePotential=True,
             MoireJeil=True, MoireH0AndHZ=True, MoireOffDiag=True, MoireOffDiagMidpoint=True)
FIELDS = [0, 2, 5, -3, 16]
NVEC = 4


@pytest.fixture(scope="module")
def ctx():
    with G.Context(0) as c:
        yield c


@pytest.fixture(scope="module")
def base():
    return R.build(MOIRE)


def _field_free(ctx, r):
    geo = r["geo"]
    ctx.set_geometry(geo["rat"], geo["species"], geo["layer"], geo["ucell"])
    ctx.neighbours(r["cut2intra"], r["cut2inter"], r["second_layer"], tables=False)
    ctx.assemble(R.gpu_model(r["model"]), r["rat_on"], r["rat_hop"], None)


def _draws(n):
    return np.stack([np.stack([orc.rng_draws(1000 + 10 * f + v, n) for v in range(NVEC)]) for f in range(len(FIELDS))])


def _close(a, b, a0, b0, tol):
    scale = max(np.abs(a0).max(), np.abs(b0).max())
    return np.abs(a - a0).max() <= tol * scale and np.abs(b - b0).max() <= tol * scale


def test_fields_fp64_match_per_field_oracle(ctx, base):
    """FP64, uneven lengths: every vector of every field within 1e-10 of the oracle's recursion on that
    field's Hamiltonian."""
    n = base["geo"]["n"]
    u = _draws(n)
    ns = np.random.default_rng(5).integers(60, 121, (len(FIELDS), NVEC)).astype(np.int32)
    _field_free(ctx, base)
    a, b = ctx.lanczos_fields(FIELDS, u, ns, G.GBN_FP64)
    for f, m in enumerate(FIELDS):
        r = R.build(dict(MOIRE, MagFieldInteger=m)) if m else base
        for v in range(NVEC):
            psi = np.exp(2j * np.pi * u[f, v]) / np.sqrt(n)
            k = int(ns[f, v])
            a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], psi, k, 0)
            assert _close(a[f, v, :k], b[f, v, :k], a0, b0, 1e-10), (m, v)


@pytest.mark.parametrize("grp", [1, 2])
def test_fields_every_matrix_path(ctx, base, grp):
    """Records staged in shared memory or read in place, rows per group 1 or 2, the rotations from the
    tile table or on the fly: FP64 recursions of the batched fields agree to 1e-10 of the spectral scale."""
    n = base["geo"]["n"]
    u = _draws(n)
    _field_free(ctx, base)
    out = []
    try:
        for staged in (0, 1):
            for table in (1, 0):
                ctx.set_tuning(0, 0, grp, staged)
                ctx.set_kernel_variant(0, -1, 0, table)
                out.append(ctx.lanczos_fields(FIELDS, u, 80, G.GBN_FP64))
    finally:
        ctx.set_tuning()
        ctx.set_kernel_variant()
    for k in range(1, len(out)):
        assert _close(out[k][0], out[k][1], out[0][0], out[0][1], 1e-10), k


def test_fields_mixed_table_against_on_the_fly(ctx, base):
    """Mixed precision: the tile table's rotations (FP64 sincospi of the 32-bit turn fraction, rounded once)
    against the on-the-fly rotation (split-angle FP32, error below 2e-13): a_n, b_n within FP32 rounding."""
    n = base["geo"]["n"]
    u = _draws(n)
    _field_free(ctx, base)
    try:
        ctx.set_kernel_variant(0, -1, 0, 1)
        a1, b1 = ctx.lanczos_fields(FIELDS, u, 100, G.GBN_MIXED)
        ctx.set_kernel_variant(0, -1, 0, 0)
        a0, b0 = ctx.lanczos_fields(FIELDS, u, 100, G.GBN_MIXED)
    finally:
        ctx.set_kernel_variant()
    assert _close(a1, b1, a0, b0, 1e-5)


def test_fields_mixed_dos(ctx, base):
    """Mixed precision (FP32 vectors and field-free hoppings, phases from 32-bit turn fractions): the DOS
    of each field against the FP64 oracle's, and against the per-field mixed path (gbn_peierls)."""
    n, g0 = base["geo"]["n"], base["g0"]
    u = _draws(n)
    _field_free(ctx, base)
    a, b = ctx.lanczos_fields(FIELDS, u, 120, G.GBN_MIXED)
    eta, ne, lo, hi = 0.02 / g0, 600, -0.6 / g0, 0.6 / g0
    for f, m in enumerate(FIELDS):
        r = R.build(dict(MOIRE, MagFieldInteger=m)) if m else base
        d_ref = 0.0
        d_mix = 0.0
        d_fld = 0.0
        _field_free(ctx, base)
        if m:
            ctx.peierls(r["flux"])
        ap, bp = ctx.lanczos_phases(u[f], 120, G.GBN_MIXED)
        for v in range(NVEC):
            psi = np.exp(2j * np.pi * u[f, v]) / np.sqrt(n)
            a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], psi, 120, 0)
            d_ref = d_ref + orc.frac(a0, b0, eta, ne, lo, hi)[1]
            d_fld = d_fld + orc.frac(a[f, v], b[f, v], eta, ne, lo, hi)[1]
            d_mix = d_mix + orc.frac(ap[v], bp[v], eta, ne, lo, hi)[1]
        err_fld = np.abs(d_fld - d_ref).sum() / np.abs(d_ref).sum()
        err_mix = np.abs(d_mix - d_ref).sum() / np.abs(d_ref).sum()
        assert err_fld <= 1e-6, (m, err_fld, err_mix)


@pytest.mark.parametrize("mb", [1, 2])
def test_fields_fused_step(ctx, base, mb):
    """The fused step on the field-batched layout (gathers of v_k and u_{k-1} rotated per field, u_k formed
    in the gather, one launch per step): the DOS of each field within 1e-6 (normalised L1) of the FP64
    oracle's on that field's Hamiltonian, and at least one launch per step fewer than the two-launch step."""
    n, g0 = base["geo"]["n"], base["g0"]
    u = _draws(n)
    _field_free(ctx, base)
    try:
        ctx.set_kernel_variant(0, -1, 0, 0, -1, 0)
        l0 = ctx.launches
        ctx.lanczos_fields(FIELDS, u, 120, G.GBN_MIXED)
        two = ctx.launches - l0
        ctx.set_kernel_variant(0, -1, mb, 0, -1, 1)
        l0 = ctx.launches
        a, b = ctx.lanczos_fields(FIELDS, u, 120, G.GBN_MIXED)
        one = ctx.launches - l0
    finally:
        ctx.set_kernel_variant()
    assert two - one >= 120
    eta, ne, lo, hi = 0.02 / g0, 600, -0.6 / g0, 0.6 / g0
    for f, m in enumerate(FIELDS):
        r = R.build(dict(MOIRE, MagFieldInteger=m)) if m else base
        d_ref = 0.0
        d_fld = 0.0
        for v in range(NVEC):
            psi = np.exp(2j * np.pi * u[f, v]) / np.sqrt(n)
            a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], psi, 120, 0)
            d_ref = d_ref + orc.frac(a0, b0, eta, ne, lo, hi)[1]
            d_fld = d_fld + orc.frac(a[f, v], b[f, v], eta, ne, lo, hi)[1]
        err = np.abs(d_fld - d_ref).sum() / np.abs(d_ref).sum()
        assert err <= 1e-6, (m, err)


def test_fields_fused_step_fp64(ctx, base):
    """The fused step on the field-batched layout in FP64: every field's a_n, b_n within 1e-10 of the
    spectral scale of the oracle's recursion on that field's Hamiltonian, as the two-launch FP64 path."""
    n = base["geo"]["n"]
    u = _draws(n)
    ns = np.full((len(FIELDS), NVEC), 90, np.int32)
    _field_free(ctx, base)
    try:
        ctx.set_kernel_variant(0, -1, 2, 0, -1, 1)
        a, b = ctx.lanczos_fields(FIELDS, u, ns, G.GBN_FP64)
    finally:
        ctx.set_kernel_variant()
    for f, m in enumerate(FIELDS):
        r = R.build(dict(MOIRE, MagFieldInteger=m)) if m else base
        for v in range(NVEC):
            psi = np.exp(2j * np.pi * u[f, v]) / np.sqrt(n)
            a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], psi, 90, 0)
            assert _close(a[f, v], b[f, v], a0, b0, 1e-10), (m, v)


@pytest.mark.parametrize("prec", [G.GBN_FP64, G.GBN_MIXED])
def test_fields_fused_one_vector_per_field(ctx, base, prec):
    """One vector per field (the drop-in driver's DOS-only sweeps: one right-hand side per thread) with the
    fused step: FP64 within 1e-10 of the spectral scale of the oracle on each field's Hamiltonian; mixed
    precision, the DOS of each field within 1e-6 of the oracle's."""
    n, g0 = base["geo"]["n"], base["g0"]
    fields = FIELDS * 3   # 15 fields: a tile of 16
    u = np.stack([orc.rng_draws(2000 + f, n) for f in range(len(fields))])[:, None, :]
    _field_free(ctx, base)
    try:
        ctx.set_kernel_variant(0, -1, 2, 0, -1, 1)
        a, b = ctx.lanczos_fields(fields, u, 90, prec)
    finally:
        ctx.set_kernel_variant()
    eta, ne, lo, hi = 0.02 / g0, 600, -0.6 / g0, 0.6 / g0
    for f, m in enumerate(fields):
        r = R.build(dict(MOIRE, MagFieldInteger=m)) if m else base
        psi = np.exp(2j * np.pi * u[f, 0]) / np.sqrt(n)
        a0, b0 = orc.recursion(r["nb"], r["hop"], r["h0"], psi, 90, 0)
        if prec == G.GBN_FP64:
            assert _close(a[f, 0], b[f, 0], a0, b0, 1e-10), m
        else:
            d0 = orc.frac(a0, b0, eta, ne, lo, hi)[1]
            d1 = orc.frac(a[f, 0], b[f, 0], eta, ne, lo, hi)[1]
            assert np.abs(d1 - d0).sum() <= 1e-6 * np.abs(d0).sum(), m


def test_fields_reject_a_field_already_applied(ctx, base):
    _field_free(ctx, base)
    ctx.peierls(R.build(dict(MOIRE, MagFieldInteger=2))["flux"])
    u = _draws(base["geo"]["n"])
    with pytest.raises(G.GbnError):
        ctx.lanczos_fields(FIELDS, u, 20, G.GBN_FP64)


def test_fields_reject_repeated_images():
    """A 4x4 graphene cell with third neighbours: a row meets periodic images of one atom twice."""
    r = R.build(dict(TypeOfSystem="Graphene", CellSize=2, NeighLevels=3))
    n = r["geo"]["n"]
    assert any(len(set(row[:k])) < k for row, k in zip(r["nb"]["nlist"], r["nb"]["nneigh"]))
    with G.Context(0) as c:
        _field_free(c, r)
        with pytest.raises(G.GbnError):
            c.lanczos_fields([1, 2], np.zeros((2, 1, n)), 5, G.GBN_FP64)
