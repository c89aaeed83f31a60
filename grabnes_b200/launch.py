"""Run the drop-in driver (`grabnes Gendata.in`) over several GPUs: one process per GPU.

    python -m torch.distributed.run --nnodes 1 --nproc-per-node N --master-addr 127.0.0.1 \
        -m grabnes_b200.launch Gendata.in
    python -m grabnes_b200.launch --gpus N Gendata.in        # the same, processes started here

Every rank starts the driver on its GPU (GRABNES_DEVICE = local rank modulo the devices present) with
GRABNES_RANK / GRABNES_NRANKS, so that the driver runs its share of the sweep: unit u -- the u-th
(field, Haldane phase) pair of the reference's field loop (lanczosKuboCode/Src/calc.F90:82-114), or the
u-th field of a batched DOS-only sweep -- on rank u % N.  Each unit writes its own folder, exactly the
files a single process writes for it, so nothing is merged: the ranks exchange only their exit status,
wall time and log name (one all-gather over gloo, host objects), and rank 0 writes them to
grabnes.shards.json in the working directory.  A rank whose driver fails makes the launch fail.
The driver's output of rank r goes to grabnes.rank<r>.log.
"""
import argparse
import datetime
import json
import os
import socket
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER = os.path.join(HERE, "grabnes")


def run_rank(rank, ws, local, gendata, driver, timeout_s=86400):
    """One rank: the driver on its share of the sweep, then the status exchange (rank 0 writes it)."""
    import torch
    import torch.distributed as dist
    if ws > 1 and not dist.is_initialized():
        dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=timeout_s))
    ndev = torch.cuda.device_count() if torch.cuda.is_available() else 0
    env = dict(os.environ, GRABNES_RANK=str(rank), GRABNES_NRANKS=str(ws),
               GRABNES_DEVICE=str(local % ndev if ndev else 0))
    log = f"grabnes.rank{rank}.log"
    t0 = time.time()
    with open(log, "w") as f:
        rc = subprocess.run([driver, gendata], env=env, stdout=f, stderr=subprocess.STDOUT).returncode
    status = {"rank": rank, "rc": rc, "wall_s": time.time() - t0, "device": int(env["GRABNES_DEVICE"]),
              "host": socket.gethostname(), "log": log}
    statuses = [None] * ws
    if ws > 1:
        dist.all_gather_object(statuses, status)
    else:
        statuses = [status]
    worst = max(s["rc"] != 0 for s in statuses)
    if rank == 0:
        with open("grabnes.shards.json", "w") as f:
            json.dump({"ranks": ws, "gendata": gendata, "statuses": statuses}, f, indent=1)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 1 if worst else 0


def _spawned(local, ws, port, gendata, driver, rcs):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(local), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(local))
    rcs[local] = run_rank(local, ws, local, gendata, driver)


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    p.add_argument("gendata", nargs="?", default="Gendata.in")
    p.add_argument("--gpus", type=int, default=0, help="start this many ranks here (without torchrun)")
    p.add_argument("--driver", default=DRIVER, help="the driver executable (default: the package's grabnes)")
    a = p.parse_args(argv)
    if not os.path.exists(a.driver):
        sys.exit(f"driver not found: {a.driver} (build it with python -m grabnes_b200.build)")
    if "WORLD_SIZE" in os.environ and a.gpus == 0:   # under torchrun
        return run_rank(int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"]),
                        int(os.environ.get("LOCAL_RANK", "0")), a.gendata, a.driver)
    ws = max(1, a.gpus)
    if ws == 1:
        return run_rank(0, 1, 0, a.gendata, a.driver)
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    rcs = mp.Manager().dict()
    mp.spawn(_spawned, args=(ws, port, a.gendata, a.driver, rcs), nprocs=ws, join=True)
    return max(rcs.values()) if rcs else 1


if __name__ == "__main__":
    sys.exit(main())
