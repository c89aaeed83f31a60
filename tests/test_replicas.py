"""Replicas over ranks (the multi-GPU path), run as two gloo processes on CPU.

Each rank draws its own random-phase vectors (seed_of), runs the recursion on them and contributes its
averaged DOS; mean_over_ranks must give the DOS of all the ranks' vectors together, and max_over_ranks
the slowest rank's time.  The per-rank recursion here is the oracle's (CPU); on GPUs the library runs
it, with the same host-side combination.
"""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GRAPHENE = dict(TypeOfSystem="Graphene", CellSize=24, Hopping=2.7, LatticeParameter=2.4595)
SEED, VECS, STEPS = 7, 2, 120


def _rank_dos(r, seed, nvec):
    from oracle import oracle as orc
    n = r["geo"]["n"]
    u = np.asarray(__import__("grabnes_b200").rng_uniform(seed, nvec * n)).reshape(nvec, n)
    dos = []
    for k in range(nvec):
        psi = np.exp(2j * np.pi * u[k]) / np.sqrt(n)
        a, b = orc.recursion(r["nb"], r["hop"], r["h0"], psi, STEPS, 1)
        e, d = orc.frac(a, b, 0.02, 400, -3.5, 3.5)
        dos.append(d)
    return e, np.mean(dos, axis=0)


def _worker(rank, ws, port, out):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from grabnes_b200 import replicas
    import refcases as R
    ws_, rank_, _ = replicas.init("gloo", timeout_s=60)
    assert (ws_, rank_) == (ws, rank)
    r = R.build(GRAPHENE)
    _, d = _rank_dos(r, replicas.seed_of(SEED, rank), VECS)
    mean = replicas.mean_over_ranks(d, ws)
    slowest = replicas.max_over_ranks(1.0 + rank, ws)
    replicas.barrier(ws)
    if rank == 0:
        np.save(out, np.concatenate([[slowest], mean]))
    replicas.finish(ws)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_replicas_combine_to_the_dos_of_all_vectors(tmp_path):
    import sys
    sys.path.insert(0, ROOT)
    import refcases as R
    from grabnes_b200 import replicas
    ws = 2
    out = str(tmp_path / "mean.npy")
    mp.start_processes(_worker, args=(ws, _free_port(), out), nprocs=ws, start_method="spawn", join=True)
    got = np.load(out)
    assert got[0] == 2.0   # the slowest rank's time
    r = R.build(GRAPHENE)
    parts = [_rank_dos(r, replicas.seed_of(SEED, k), VECS)[1] for k in range(ws)]
    assert np.allclose(got[1:], np.mean(parts, axis=0), rtol=0, atol=1e-14)
    # the ranks' streams differ: the replicas are independent samples
    assert np.abs(parts[0] - parts[1]).max() > 1e-3


def test_seeds_are_disjoint_per_rank():
    from grabnes_b200 import replicas
    seeds = {replicas.seed_of(SEED, k) for k in range(8)}
    assert len(seeds) == 8
