"""Errors at the C ABI: invalid arguments, calls out of order and numerical failures come back as negative
codes with a message, nothing aborts, and the context stays usable afterwards.  Host entry points on the
CPU; context entry points on the GPU.  Edge case: atoms without neighbours."""
import ctypes as C

import numpy as np
import pytest

import refcases as R
from oracle import oracle as orc

G = pytest.importorskip("grabnes_b200")
ARG, STATE, NUMERIC = -1, -3, -4


# ------------------------------------------------------------------------------------------ host (CPU)
def test_host_entry_points_reject_bad_arguments():
    L = G.lib()
    bad = G.Cell(7, 10, 1, (C.c_int32 * 4)(0, 0, 0, 0), 2.46, 40.0, 3.35)
    n = C.c_int64()
    assert L.gbn_cell_atoms(C.byref(bad), C.byref(n)) == ARG
    out = np.zeros(4)
    assert L.gbn_rng_uniform(1, -1, out) == ARG
    assert L.gbn_cheb_coef(1.0, 0.0, 1.0, 0, np.zeros(2, np.complex128)) != 0
    p = G.Pdos()
    p.mode = 99
    cell = G.build_cell(G.CELL_GRAPHENE, cell_size=4)
    with pytest.raises(G.GbnError):
        G.pdos_atoms(p, cell["rat"], cell["species"], cell["layer"], cell["ucell"])
    p.mode = G.PDOS_BY_NUMBER
    p.atom_number = cell["n"] + 1   # outside 1..N
    with pytest.raises(G.GbnError):
        G.pdos_atoms(p, cell["rat"], cell["species"], cell["layer"], cell["ucell"])
    p.mode = G.PDOS_LAYER
    p.number_of_layers = 0
    with pytest.raises(G.GbnError):
        G.pdos_sets(p, cell["species"], cell["layer"])


# ------------------------------------------------------------------------------------------ context (GPU)
@pytest.fixture(scope="module")
def graphene():
    return R.build(dict(TypeOfSystem="Graphene", CellSize=30, Hopping=2.7))


def _code(fn, *args, **kw):
    with pytest.raises(G.GbnError) as e:
        fn(*args, **kw)
    return e.value.code


@pytest.mark.gpu
def test_calls_out_of_order():
    with G.Context(0) as ctx:
        assert _code(ctx.lanczos, np.ones((1, 8), np.complex128), 5) == STATE
        assert _code(ctx.peierls, 1.0) == STATE


@pytest.mark.gpu
def test_invalid_arguments_leave_the_context_usable(graphene):
    r = graphene
    nb, n = r["nb"], r["geo"]["n"]
    psi = orc.init_wf(n, 1)
    with G.Context(0) as ctx:
        bad = nb["nlist"].copy()
        bad[3, 0] = n + 1
        assert _code(ctx.load_hamiltonian, nb["nneigh"], bad, r["hop"], r["h0"]) == ARG
        ctx.load_hamiltonian(nb["nneigh"], nb["nlist"], r["hop"], r["h0"])
        L = ctx._L
        a, b = np.zeros(10), np.zeros(10)
        assert L.gbn_lanczos(ctx._h, 7, 1, psi, None, 10, a, b) == ARG          # precision
        assert L.gbn_lanczos(ctx._h, 0, 1, psi, np.array([11], np.int32), 10, a, b) == ARG   # nsteps > nmax
        assert L.gbn_lanczos(ctx._h, 0, 0, psi, None, 10, a, b) == ARG          # no right-hand side
        assert b"nsteps" in L.gbn_last_error(ctx._h) or b"nrhs" in L.gbn_last_error(ctx._h)
        assert _code(ctx.cf_dos, np.ones(10), np.ones(10), 0.0, 10, -1.0, 1.0) == ARG   # eta <= 0
        assert _code(ctx.kubo_evol, np.ones(4, np.complex128), 0.0, 1.0, psi, psi) == STATE   # no NeighD
        assert _code(ctx.lanczos_sites, [0], 10) == ARG
        assert _code(ctx.lanczos_sets, np.full(n, 5, np.int32), np.zeros(n), [1.0], 10) == ARG
        # after all of these, a valid call still gives the oracle's coefficients
        a1, b1 = ctx.lanczos(psi, 100, G.GBN_FP64)
        a0, b0 = orc.recursion(nb, r["hop"], r["h0"], psi, 100, 0)
        assert np.abs(a1[0] - a0).max() <= 1e-10 * np.abs(b0).max() and np.abs(b1[0] - b0).max() <= 1e-10 * np.abs(b0).max()


@pytest.mark.gpu
def test_numerical_failures_are_reported(graphene):
    r = graphene
    nb, n = r["nb"], r["geo"]["n"]
    geo = r["geo"]
    with G.Context(0) as ctx:
        ctx.set_geometry(geo["rat"], geo["species"], geo["layer"], geo["ucell"])
        ctx.neighbours(r["cut2intra"], r["cut2inter"], r["second_layer"], tables=False)
        ctx.assemble(R.gpu_model(r["model"]), None, None, None)
        u = geo["ucell"]
        area = abs(u[0] * u[4] - u[1] * u[3])
        assert _code(ctx.peierls, 0.5 * np.pi * 1.0e20 / area) == NUMERIC   # half a flux quantum through the cell
        assert _code(ctx.lanczos, np.zeros((1, n), np.complex128), 20) == NUMERIC   # zero start vector: b = 0
        a, b = ctx.lanczos(orc.init_wf(n, 2), 50, G.GBN_FP64)
        assert np.all(np.isfinite(a)) and np.all(b > 0)


@pytest.mark.gpu
def test_atoms_without_neighbours(graphene):
    """Rows of isolated atoms (no entries, only H0) among connected ones: recursion against the oracle."""
    r = graphene
    nb = r["nb"]
    n = r["geo"]["n"]
    iso = [0, 17, n - 1]
    nn, nl = nb["nneigh"].copy(), nb["nlist"].copy()
    hop, h0 = r["hop"].copy(), r["h0"].copy()
    h0[iso] = [0.3, -0.2, 0.1]
    for i in range(n):   # drop every entry to or from an isolated atom, keeping the rest in order
        keep = [j for j in range(nn[i]) if i not in iso and nl[i, j] - 1 not in iso]
        row_l, row_h = nl[i, keep].copy(), hop[i, keep].copy()
        nn[i] = len(keep)
        nl[i, :] = 1
        hop[i, :] = 0
        nl[i, :len(keep)], hop[i, :len(keep)] = row_l, row_h
    tabs = dict(nb, nneigh=nn, nlist=nl)
    psi = orc.init_wf(n, 8)
    a0, b0 = orc.recursion(tabs, hop, h0, psi, 100, 0)
    with G.Context(0) as ctx:
        ctx.load_hamiltonian(nn, nl, hop, h0)
        for prec, tol in ((G.GBN_FP64, 1e-10), (G.GBN_MIXED, 1e-5)):
            a, b = ctx.lanczos(psi, 100, prec)
            assert np.abs(a[0] - a0).max() <= tol * np.abs(b0).max()
            assert np.abs(b[0] - b0).max() <= tol * np.abs(b0).max()
