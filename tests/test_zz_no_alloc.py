"""gbn_lanczos_noalloc against the context-based recursion, through the C ABI, on a B200.

gbn_lanczos_noalloc is for hosts that cannot allocate device memory (their pool allocator owns the
GPU, or cudaMalloc's device-wide synchronisation is not allowed while they have work in flight): the
caller passes the Hamiltonian, the start vector and a/b in its own device memory, and the recursion
vectors live in a fixed array inside the library.  Every call shares that array, so this test makes
two calls in a row with different start vectors and checks each against gbn_lanczos on a context
(the existing entry point), within the FP64 recursion tolerance of the other parity tests (1e-10
relative over 200 steps).  The file sorts last so that a run stopping at the first failure has run
every other test before it.
"""
import numpy as np
import pytest

import refcases as R
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

G = pytest.importorskip("grabnes_b200")
torch = pytest.importorskip("torch")

NSTEPS = 200
# 20 000-atom graphene: large enough that 200 FP64 steps stay clear of the recursion's sensitivity to
# summation order (the same case as the FP64 drop-in parity test)
GRAPHENE = dict(TypeOfSystem="Graphene", CellSize=100, Hopping=2.7, LatticeParameter=2.4595)


def _rel(x, y):
    return np.abs(x - y).max() / np.abs(y).max()


def test_noalloc_recursion_matches_context_recursion():
    r = R.build(GRAPHENE)
    nb = r["nb"]
    n, mn = r["geo"]["n"], nb["max_neigh"]
    psis = [orc.init_wf(n, 123456), orc.init_wf(n, 99)]
    refs = []
    with G.Context(0) as ctx:
        ctx.load_hamiltonian(nb["nneigh"], nb["nlist"], r["hop"], r["h0"])
        for psi in psis:
            refs.append(ctx.lanczos(psi, NSTEPS, G.GBN_FP64))

    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    nneigh = torch.from_numpy(np.ascontiguousarray(nb["nneigh"], np.int32)).to(dev)
    nlist = torch.from_numpy(np.ascontiguousarray(nb["nlist"], np.int32).reshape(-1)).to(dev)
    hopp = torch.from_numpy(np.ascontiguousarray(r["hop"], np.complex128).reshape(-1).view(np.float64)).to(dev)
    h0 = torch.from_numpy(np.ascontiguousarray(r["h0"], np.float64)).to(dev)
    stream = torch.cuda.current_stream(dev)
    L = G.lib()
    for psi, (a_ref, b_ref) in zip(psis, refs):
        d_psi = torch.from_numpy(np.ascontiguousarray(psi, np.complex128).view(np.float64)).to(dev)
        a = torch.full((NSTEPS,), float("nan"), dtype=torch.float64, device=dev)
        b = torch.full((NSTEPS,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        rc = L.gbn_lanczos_noalloc(n, mn, nneigh.data_ptr(), nlist.data_ptr(), hopp.data_ptr(), h0.data_ptr(),
                                   d_psi.data_ptr(), NSTEPS, a.data_ptr(), b.data_ptr(), stream.cuda_stream)
        assert rc == 0, G.ERRORS.get(rc, rc)
        a_np, b_np = a.cpu().numpy(), b.cpu().numpy()
        assert _rel(a_np, a_ref[0]) <= 1e-10 and _rel(b_np, b_ref[0]) <= 1e-10

    # one NList entry out of range: the kernel skips that access and reports it (GBN_ERR_ARG); the flag
    # lives in the shared array, so the next good call must find it cleared and repeat the good result
    bad = np.ascontiguousarray(nb["nlist"], np.int32).reshape(-1).copy()
    bad[5] = n + 7
    nlist_bad = torch.from_numpy(bad).to(dev)
    rc = L.gbn_lanczos_noalloc(n, mn, nneigh.data_ptr(), nlist_bad.data_ptr(), hopp.data_ptr(), h0.data_ptr(),
                               d_psi.data_ptr(), NSTEPS, a.data_ptr(), b.data_ptr(), stream.cuda_stream)
    assert rc == G.GBN_ERR_ARG
    a2 = torch.full((NSTEPS,), float("nan"), dtype=torch.float64, device=dev)
    b2 = torch.full((NSTEPS,), float("nan"), dtype=torch.float64, device=dev)
    rc = L.gbn_lanczos_noalloc(n, mn, nneigh.data_ptr(), nlist.data_ptr(), hopp.data_ptr(), h0.data_ptr(),
                               d_psi.data_ptr(), NSTEPS, a2.data_ptr(), b2.data_ptr(), stream.cuda_stream)
    assert rc == 0, G.ERRORS.get(rc, rc)
    assert np.array_equal(a2.cpu().numpy(), a_np) and np.array_equal(b2.cpu().numpy(), b_np)

    # beyond the stated maximum: rejected on the host before anything is launched
    rc = L.gbn_lanczos_noalloc(G.NOALLOC_MAX_ATOMS + 1, mn, nneigh.data_ptr(), nlist.data_ptr(), hopp.data_ptr(),
                               h0.data_ptr(), d_psi.data_ptr(), NSTEPS, a.data_ptr(), b.data_ptr(), stream.cuda_stream)
    assert rc == G.GBN_ERR_LIMIT
