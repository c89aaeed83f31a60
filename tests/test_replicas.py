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


# ---------------------------------------------------------------------------- sharded driver sweeps
FAKE_DRIVER = """#!{python}
# Stands in for the driver on a machine without a GPU: the real driver's --print-job gives this rank's
# units (GRABNES_RANK / GRABNES_NRANKS, its sharding rule), and every unit writes its own folder.
import json, os, subprocess, sys
out = subprocess.run([{real!r}, "--print-job", sys.argv[1]], capture_output=True, text=True, check=True)
units = json.loads(out.stdout.splitlines()[0])["units"]
for mb, ph in units:
    d = "m%05d_p%d" % (mb, ph)
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "unit.txt"), "w") as f:
        f.write("%d %d\\n" % (mb, ph))
"""


def _launch(workdir, ws, driver):
    import subprocess
    import sys
    with open(os.path.join(workdir, "Gendata.in"), "w") as f:
        f.write("Run.TypeOfSystem Graphene\nStructure.CellSize 10\nMagField.InitialInteger 0\n"
                "MagField.FinalInteger 12\nMagField.IntegerStep 2\n")
    env = dict(os.environ, PYTHONPATH=ROOT)
    return subprocess.run([sys.executable, "-m", "grabnes_b200.launch", "--gpus", str(ws), "--driver", driver,
                           "Gendata.in"], cwd=workdir, env=env, capture_output=True, text=True, timeout=300)


def test_launcher_splits_a_sweep_over_two_gloo_ranks(tmp_path):
    """grabnes_b200.launch with two ranks (gloo on CPU): every field of a 7-field sweep is run by exactly
    one rank (the driver's own sharding rule, read from its --print-job), the folders of the two ranks
    together are those of a single-rank run, and rank 0 records both ranks' exit status."""
    import json
    real = os.path.join(ROOT, "grabnes_b200", "grabnes")
    if not os.path.exists(real):
        pytest.skip("driver not built")
    import sys
    fake = tmp_path / "fake_driver.py"
    fake.write_text(FAKE_DRIVER.format(python=sys.executable, real=real))
    fake.chmod(0o755)
    runs = {}
    for ws in (1, 2):
        wd = tmp_path / f"ws{ws}"
        wd.mkdir()
        p = _launch(str(wd), ws, str(fake))
        assert p.returncode == 0, p.stdout + p.stderr
        runs[ws] = {d: (wd / d / "unit.txt").read_text() for d in sorted(os.listdir(wd)) if d.startswith("m0")}
        st = json.loads((wd / "grabnes.shards.json").read_text())
        assert st["ranks"] == ws and [s["rc"] for s in st["statuses"]] == [0] * ws
    assert len(runs[1]) == 7 and runs[2] == runs[1]


def test_shard_units_cover_each_unit_once():
    from grabnes_b200 import replicas
    for ws in (1, 2, 3, 5):
        got = sorted(u for r in range(ws) for u in replicas.shard_units(11, r, ws))
        assert got == list(range(11))
