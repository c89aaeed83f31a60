#!/usr/bin/env python
"""Throughput of the batched Lanczos-recursion DOS on a B200.

Workload (one bench step = one complete recursion job): twisted-bilayer graphene at 1.08 degrees
(commensurate moire cell 31 30 30 31, 11 164 atoms) tiled 20 x 20 = 4 465 600 atoms, rigid,
intralayer nearest-neighbour t = -2.7 eV, two-centre interlayer hopping (Vpp_pi0 = 2.7, Vpp_sigma0 =
0.48 eV, decay 0.319 Ang, d = 3.35 Ang) to 5 Ang in-plane; 16 random-phase vectors (GNU Fortran
RNG, seed 7, vector r = draws r*N .. (r+1)*N-1); 2000 recursion steps each; complex FP32 vectors and
hoppings with FP64 a_n/b_n ("mixed").  Synthetic input of the reference's own model (no dataset).

Reported: value = atom-steps/s with the start vectors resident on the device (whole job, all
ranks); e2e = the same through gbn_lanczos_phases with host buffers (H2D of the draws, D2H of a, b);
roofline of the recursion-step kernel against measured HBM bandwidth; the plain FP64 paths (batched
and single vector) and the DOS error of the mixed path against the FP64 path; the oracle port timed
on the host cores as CPU baseline.  Further legs (each can be skipped or run alone): the 33-field
graphene/hBN sweep batched against field by field (fields_batch), the Chebyshev Kubo time evolution of
the 3.5M-atom graphene/hBN cell with its states on the device against on the host
(kubo_time_evolution), one DOS-loss gradient of a 964,548-atom twisted bilayer (dos_gradient), and the
batched mixed-precision DOS of the 3.5M-atom graphene/hBN cell with its roofline (moire_dos).  --impl reference times that CPU port alone (the reference is
Fortran + MPI and cannot be built in this image).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = {
    "Run.TypeOfSystem": "TwistedBilayerBasedOnMoireCell", "Structure.MoireCellParameters": (31, 30, 30, 31),
    "Structure.SuperCell": 20, "Structure.LatticeParameter": 2.4595, "Structure.InterlayerDistance": 3.35,
    "TB.Hopping": 2.7, "TB.NeighLevels": 1, "Interlayer.TypeOfBL": "Koshino", "Interlayer.Vpppi0": 2.7,
    "Interlayer.Vppsigma0": 0.48, "Interlayer.BLdelta": 0.319, "Neigh.LayerNeighbors": 100,
    "Neigh.LayerDistFactor": 3.2005,
}
NRHS, SEED, NSTEPS = 16, 7, 2000
METRIC = "Lanczos atom-steps/s & HBM GB/s: batched FP32 vs plain FP64 at DOS err<1e-6"
WORKLOAD_NAME = "tbg_1.08deg_20x20_4465600atoms_16vec_2000steps"
ETA_EV, NE, EMIN_EV, EMAX_EV = 0.01, 4000, -9.0, 9.0


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-i", str(self.index), "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [l.split(",") for l in open(self.f.name).read().splitlines() if l.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows if len(r) >= 9 for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_count():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def dist_init():
    from grabnes_b200 import replicas
    return replicas.init("nccl")


def dist_max(x, ws):
    from grabnes_b200 import replicas
    return replicas.max_over_ranks(x, ws)


def barrier(ws):
    from grabnes_b200 import replicas
    replicas.barrier(ws)


PROFILES = os.path.join(ROOT, "profiles")


def kernel_key(best):
    """Name of the sparse-product kernel a tuning selects, as the ncu summaries in profiles/ label their
    captures: rows per group, columns in flight, staged values or indices, register bound, prefetch."""
    staged = best.get("staged", -1) != 0
    unroll = best.get("unroll", 0) or 8              # library defaults in mixed precision
    sv = 0 if best.get("stage_values", -1) == 0 else 1
    g = best.get("rows_per_group", 0) or 2           # default rows per group for 16 vectors of ~33 entries
    mb = best.get("min_blocks", 0) or (3 if (unroll == 8 and g == 1 and staged) else 1)
    pf = best.get("prefetch", -1)
    pf = 6 if pf < 0 else pf
    rpt = best.get("rhs_per_thread", 0) or 4         # right-hand sides per thread (16 vectors: 4 threads a row)
    if not staged:
        return f"k_spmm_step<float, real, G={g}, RPT={rpt}, U={unroll}>"
    fused = ", FUSED" if best.get("fused", -1) == 1 else ""   # the update folded into the product
    return f"k_spmm_staged<float, real, G={g}, RPT={rpt}, U={unroll}, SV={sv}, MINB={mb}, prefetch={pf}{fused}>"


def traffic_from_profile(key, workload="bench_workload"):
    """DRAM bytes per sparse-product launch of the kernel `key` on a workload ("bench_workload": the TBG
    job, from captures of the same kernel on the 10 x 10 tiling scaled by the rows processed;
    "moire_dos": the 3.5M-atom graphene/hBN job, captured at full size), from the lines
    `dram_bytes_per_launch_<workload>[<key>] = <bytes>` of the committed ncu summaries; None when no
    summary covers that kernel."""
    import glob
    import re
    pat = re.compile(r"dram_bytes_per_launch_" + workload + r"\[(.+?)\]\s*=\s*([0-9.eE+]+)")
    for path in sorted(glob.glob(os.path.join(PROFILES, "*.md"))):
        with open(path) as f:
            for m in pat.finditer(f.read()):
                if m.group(1).strip() == key:
                    return float(m.group(2)), os.path.relpath(path, ROOT)
    return None, None


# ------------------------------------------------------------------------------------------- ours
def run_ours(args, ws, rank, local):
    import torch

    import grabnes_b200 as G
    from grabnes_b200 import model as M
    from grabnes_b200 import replicas

    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    if args.moire_dos_only:
        out = moire_dos_leg(G, M, local, stream, ws, nsteps=args.moire_steps, peak=peaks()[0], tuning=args.tuning)
        if rank == 0:
            print(json.dumps(out), flush=True)
        replicas.finish(ws)
        return
    if args.gradient_only:
        out = gradient_leg(G, M, local, stream, ws)
        if rank == 0:
            print(json.dumps(out), flush=True)
        replicas.finish(ws)
        return
    if args.tevol_only:   # the time evolution alone (profiling of its kernels)
        out = tevol_leg(G, M, local, stream, ws)
        if rank == 0:
            print(json.dumps(out), flush=True)
        replicas.finish(ws)
        return
    if args.fields_only:   # the batched-field sweep alone (profiling of its kernels)
        out = fields_leg(G, M, local, stream, ws, args.fields_scale)
        if rank == 0:
            print(json.dumps(out), flush=True)
        replicas.finish(ws)
        return
    ctx = G.Context(local)
    ctx.set_stream(stream.cuda_stream)
    job = M.job_from_keys(dict(WORKLOAD, **{"Structure.SuperCell": args.supercell}))
    nsteps = args.nsteps
    t0 = time.time()
    cell = M.setup(ctx, job)
    setup_s = time.time() - t0
    n = cell["n"]
    nnz = ctx.neighbours_total
    g0 = job["g0"]
    seed = replicas.seed_of(SEED, rank)   # every rank runs its own replica of the workload (weak scaling)
    u = G.rng_uniform(seed, NRHS * n).reshape(NRHS, n)

    # ---- autotuning of the recursion kernels on this Hamiltonian, then device-resident inputs: the start
    # vectors are staged once and every job rebuilds them on the device
    from grabnes_b200.tune import autotune
    if args.tuning:
        from grabnes_b200.tune import apply
        best = fixed_tuning(args.tuning)
        apply(ctx, best)
        tuning = []
    else:
        best, tuning = autotune(ctx, u, G.GBN_MIXED)
        best = dict(best, candidates_top5=sorted((r for r in tuning if "step_ms" in r),
                                                  key=lambda r: r["step_ms"])[:5],
                    best_of_each_step_form=best_of_each_form(tuning))
    ctx.stage_phases(u, G.GBN_MIXED)
    for _ in range(args.warmup):
        ctx.run_staged(nsteps)
    torch.cuda.synchronize()
    barrier(ws)
    clocks = Clocks(int(os.environ.get("GBN_SMI_INDEX", local)))
    clocks.start()
    launches0 = ctx.launches
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    kern_ms = 0.0
    kern_launches = 0
    for _ in range(args.steps):
        ctx.run_staged(nsteps)
        ms, nl = ctx.last_timing()
        kern_ms += ms
        kern_launches += nl
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = ctx.launches - launches0
    barrier(ws)
    clk = clocks.stop()
    ms_total = dist_max(ev0.elapsed_time(ev1), ws)
    atom_steps = float(n) * NRHS * nsteps
    value = ws * atom_steps * args.steps / (ms_total / 1e3)
    spmm_ms, update_ms = ctx.kernel_timing()
    if args.value_only:   # short runs for profiling: the timed loop only
        if rank == 0:
            print(json.dumps({"value": value, "unit": "atom-steps/s", "step_ms": kern_ms / kern_launches,
                              "spmm_ms": spmm_ms, "update_ms": update_ms, "atoms": n, "entries": nnz,
                              "tuning": best, "candidates": tuning}), flush=True)
        ctx.close()
        replicas.finish(ws)
        return

    # ---- roofline of the sparse-product kernel (the dominant one).  Its algorithmic bytes are those of a
    # recursion step: matrix (int32 column + FP32 hopping per entry), on-site FP32 and the three vector
    # streams (gather of x_k counted once, x_{k-1} read, v_{k+1} written); the update kernel's own stream
    # is extra traffic of the two-kernel design and is reported with the step time.
    b_alg = nnz * (4 + 4) + n * 4 + NRHS * n * 3 * 8
    achieved = b_alg / (spmm_ms / 1e3) / 1e9
    peak, peak_kind = peaks()
    kname = kernel_key(best)
    traffic, traffic_src = traffic_from_profile(kname)

    # ---- end to end through the C ABI with host buffers (pinned)
    u_pin = torch.from_numpy(u.copy()).pin_memory()
    u_np = u_pin.numpy()
    e2e_ms = []
    for it in range(max(1, min(args.steps, 2)) + 1):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        a_mix, b_mix = ctx.lanczos_phases(u_np, nsteps, G.GBN_MIXED)
        e1.record(stream)
        torch.cuda.synchronize()
        if it > 0:   # the first call also rebuilds the device layout
            e2e_ms.append(e0.elapsed_time(e1))
    e2e_ms = dist_max(statistics.median(e2e_ms), ws)
    e2e_value = ws * atom_steps / (e2e_ms / 1e3)

    # ---- plain FP64 paths and the DOS error of the mixed path, with the library's default tuning (the
    # autotuned values belong to the 16-vector mixed-precision tile; the default picks the rows per
    # group for the tile width: 2 for 16 vectors, 1 for a single vector)
    ctx.set_tuning()
    ctx.set_kernel_variant()
    torch.cuda.synchronize()
    f0 = time.perf_counter()
    a64, b64 = ctx.lanczos_phases(u_np, nsteps, G.GBN_FP64)
    fp64_batched_s = time.perf_counter() - f0
    fp64_batched_kernel_ms, nl64 = ctx.last_timing()
    f0 = time.perf_counter()
    ctx.lanczos_phases(u_np[:1], nsteps, G.GBN_FP64)
    fp64_single_s = time.perf_counter() - f0
    fp64_single_kernel_ms, _ = ctx.last_timing()
    e, d_mix = ctx.cf_dos(a_mix, b_mix, ETA_EV / g0, NE, EMIN_EV / g0, EMAX_EV / g0)
    _, d_64 = ctx.cf_dos(a64, b64, ETA_EV / g0, NE, EMIN_EV / g0, EMAX_EV / g0)
    dm, d6 = d_mix.mean(axis=0), d_64.mean(axis=0)
    dos_err = float(np.abs(dm - d6).sum() / np.abs(d6).sum())
    dos_err_per_vector = float(max(np.abs(d_mix[r] - d_64[r]).sum() / np.abs(d_64[r]).sum() for r in range(NRHS)))
    # the DOS of vector 0 against the FP64 oracle (the reference's three-pass recursion restated in C) on
    # the same Hamiltonian, the whole 2000 steps (rank 0, N=1; about a minute on the host cores)
    oracle_err = None
    if rank == 0 and ws == 1 and not args.no_cpu and not args.no_oracle_dos:
        oracle_err = oracle_dos_error(ctx, n, u[0], nsteps, a_mix[0], b_mix[0], a64[0], b64[0], g0)

    # ---- CPU baseline: the oracle's OpenMP port of KuboRecursion on the host cores (rank 0, N=1)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_baseline(ctx, n, u[0], args.cpu_steps)
    _HOST_TABLES.clear()

    # ---- the field sweep of the graphene/hBN moire model: all fields in one batch against field by field
    fields = None
    if not args.no_fields:
        fields = fields_leg(G, M, local, stream, ws)
    # ---- Chebyshev Kubo time evolution (graphene/hBN 0.61 degrees, Anderson disorder)
    tevol = None
    if not args.no_tevol:
        tevol = tevol_leg(G, M, local, stream, ws)
    grad = None
    if not args.no_gradient:
        grad = gradient_leg(G, M, local, stream, ws)
    mdos = None
    if not args.no_moire_dos:
        mdos = moire_dos_leg(G, M, local, stream, ws, peak=peak)

    out = {
        "metric": METRIC, "value": value, "unit": "atom-steps/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64 vectors/f32 hoppings, f64 a_n b_n", "data": "synthetic (reference model)",
        "config": {"workload": WORKLOAD_NAME, "atoms": n, "entries": nnz, "vectors": NRHS, "recursion_steps": nsteps,
                   "precision": "mixed", "parallelism": f"replicas x{ws}",
                   "l2_policy": "inputs larger than L2 (vectors 572 MB, matrix 1.2 GB per step)"},
        "e2e": {"value": e2e_value, "unit": "atom-steps/s", "h2d_bytes_per_step": int(u.nbytes),
                "d2h_bytes_per_step": int(a_mix.nbytes + b_mix.nbytes)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "traffic": traffic, "traffic_source": traffic_src,
                     "algorithmic_bytes_per_launch": b_alg,
                     "kernel": kname, "avg_launch_ms": spmm_ms, "update_kernel_ms": update_ms,
                     "step_ms": kern_ms / kern_launches,
                     "step_achieved": b_alg / (kern_ms / kern_launches / 1e3) / 1e9,
                     "step_frac": b_alg / (kern_ms / kern_launches / 1e3) / 1e9 / peak,
                     # the DRAM bytes the kernel actually moves (ncu) over its live launch time
                     "traffic_frac": (traffic / (spmm_ms / 1e3) / 1e9 / peak) if traffic else None},
        "tuning": best,
        "fp64": {"batched_atom_steps_per_s": atom_steps / (fp64_batched_kernel_ms / 1e3),
                 "single_vector_atom_steps_per_s": float(n) * nsteps / (fp64_single_kernel_ms / 1e3),
                 "batched_wall_s": fp64_batched_s, "single_wall_s": fp64_single_s},
        "dos_error_vs_fp64": {"l1_mean_dos": dos_err, "l1_worst_vector": dos_err_per_vector,
                              "eta_ev": ETA_EV, "energies": NE + 1},
        "dos_error_vs_oracle": oracle_err,
        "cpu_baseline": cpu, "clocks": clk, "gpu_launches": launches, "setup_s": setup_s,
        "fields_batch": fields, "kubo_time_evolution": tevol, "dos_gradient": grad,
        "moire_dos": mdos,
    }
    if rank == 0:
        print(json.dumps(out), flush=True)
    ctx.close()
    replicas.finish(ws)


FIELDS_KEYS = {"Run.TypeOfSystem": "Graphene", "Structure.CellSize": 55, "Structure.SuperCell": 8,
               "Moire.LatticePercent": -1.0 / 55.0, "Moire.Potential": True, "Moire.Jeil": True,
               "Moire.H0AndHZ": True, "Moire.OffDiag": True, "Moire.OffDiagMidpoint": True}


def fields_leg(G, M, local, stream, ws, scale=1.0):
    """Graphene on hBN, effective moire model (387,200 atoms; on-site and bond terms of the three first-shell
    harmonics, OffDiagMidpoint): 33 fields of m = 0, 2, .., 64 flux quanta (0-26 T), 8 random-phase
    vectors per field (264 right-hand sides, GNU RNG seed 11), recursion lengths uniform in [500, 3000]
    (numpy seed 11), mixed precision.  One call of gbn_lanczos_fields (host draws in, a and b out) against
    the field-by-field path (gbn_assemble + gbn_peierls + gbn_lanczos_phases per field); both timed on
    the device stream with the host work of each call inside.  The work counted is N x the sum of the
    lengths (the useful atom-steps); every rank runs the same sweep."""
    import torch
    job = M.job_from_keys(FIELDS_KEYS)
    ctx = G.Context(local)
    ctx.set_stream(stream.cuda_stream)
    cell = M.setup(ctx, job)
    n = cell["n"]
    rat_on = G.cart_roundtrip(cell["rat"], cell["ucell"])
    rat_hop = G.cart_roundtrip(rat_on, cell["ucell"])
    ms = np.arange(0, 65, 2, dtype=np.int32)
    nvec = 8
    ns = np.random.default_rng(11).integers(500, 3001, (len(ms), nvec))
    ns = np.maximum(1, np.rint(ns * scale)).astype(np.int32)   # scale < 1: shortened lengths (profiling)
    u = G.rng_uniform(11, len(ms) * nvec * n).reshape(len(ms), nvec, n)
    area = M.cell_area(cell["ucell"])
    work = float(n) * float(ns.sum())

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return r, dist_max(e0.elapsed_time(e1), ws) / 1e3

    def batched():
        ctx.assemble(job["model"], rat_on, rat_hop, None)
        return ctx.lanczos_fields(ms, u, ns, G.GBN_MIXED)

    def per_field():
        a = np.zeros((len(ms), nvec, int(ns.max())))
        for f, m in enumerate(ms):
            ctx.assemble(job["model"], rat_on, rat_hop, None)
            if m:
                ctx.peierls(M.flux_of(int(m), area))
            af, _ = ctx.lanczos_phases(u[f], ns[f], G.GBN_MIXED)
            a[f, :, :af.shape[1]] = af
        return a

    ctx.assemble(job["model"], rat_on, rat_hop, None)
    ctx.lanczos_fields(ms[:2], u[:2, :1], 60, G.GBN_MIXED)   # warm-up (layout, kernels)
    # the step form of the sweep, chosen on one tile of four fields x 8 vectors, 200 steps: two launches
    # (product + update) or the fused step with registers for one or two blocks per SM
    forms = {}
    for name, variant in (("two_launches", (0, -1, 0, 0, -1, 0)), ("fused_1_block", (0, -1, 1, 0, -1, 1)),
                          ("fused_2_blocks", (0, -1, 2, 0, -1, 1))):
        try:
            ctx.set_kernel_variant(*variant)
            ctx.lanczos_fields(ms[:4], u[:4], 200, G.GBN_MIXED)
            forms[name] = (ctx.last_timing()[0], variant)
        except Exception:
            pass
    form = min(forms, key=lambda k: forms[k][0])
    ctx.set_kernel_variant(*forms[form][1])
    (a, _), t_batch = timed(batched)
    loop_s = ctx.last_timing()[0] / 1e3
    launches = ctx.launches
    ctx.set_kernel_variant()
    _, t_field = timed(per_field)
    ctx.close()
    name = "graphene_hbn_moire_387200atoms_33fields_x8vec_500-3000steps" + ("" if scale == 1.0 else f"_x{scale:g}")
    return {"workload": name, "atoms": n,
            "fields": int(len(ms)), "vectors_per_field": nvec, "useful_atom_steps": work,
            "batched_s": t_batch, "batched_atom_steps_per_s": ws * work / t_batch, "batched_loop_s": loop_s,
            "per_field_s": t_field, "per_field_atom_steps_per_s": ws * work / t_field,
            "speedup_vs_per_field": t_field / t_batch, "precision": "mixed", "step_form": form,
            "step_form_probe_ms": {k: v[0] for k, v in forms.items()}}


TEVOL_KEYS = {"Run.TypeOfSystem": "Graphene", "Structure.CellSize": 83, "Structure.SuperCell": 16,
              "Moire.LatticePercent": -0.018016854251615, "Moire.Twisted": True, "Moire.TwistAngle": 0.608806541588,
              "Moire.Potential": True, "Moire.Jeil": True, "Moire.H0AndHZ": True, "Moire.OffDiag": True,
              "Moire.OffDiagMidpoint": True, "Disorder.Anderson": True, "Disorder.AndersonAmp": 1.0,
              "Kubo.SeedValue": 5}
HBAR_EV_S = 6.582119569e-16


def tevol_leg(G, M, local, stream, ws, nt=10, npol=100, nvec=8, nrecurs=100, nt_msd=100, nwr_msd=10):
    """Chebyshev Kubo time evolution of graphene on hBN at 0.61 degrees (example 07's cell, CellSize 83,
    SuperCell 16 = 3,527,168 atoms) with Anderson disorder W = 1 eV (seed 5): dt = 1 fs (g0 dt / hbar),
    KuboCn with the reference's default 100 polynomials, 8 random-phase vectors, mixed precision.
    (1) nt_msd = 100 of the workload's 1000 steps with the states on the device (gbn_kubo_tevol), the
    recursion of the commutator state every nwr_msd steps, and the mean-square displacement and
    diffusivity of the 8 vectors (gbn_kubo_msd); the whole workload is 10 x these steps (each step is the
    same work), which the line states.  (2) nt = 10 steps through gbn_kubo_tevol against the same steps
    through gbn_kubo_evol with the states on the host every step.  Work unit: an atom-polynomial step of
    the dual recurrence (N x vectors x (npol - 1) per time step); each time step also propagates zupsi by
    U (as many single products)."""
    import torch
    job = M.job_from_keys(TEVOL_KEYS)
    ctx = G.Context(local)
    ctx.set_stream(stream.cuda_stream)
    cell = M.setup(ctx, job)
    n = cell["n"]
    g0 = job["g0"]
    dt = 1.0e-15 * g0 / HBAR_EV_S
    u = G.rng_uniform(5, nvec * n).reshape(nvec, n)
    psi = np.exp(2j * np.pi * u) / np.sqrt(n)
    a, b = ctx.lanczos_phases(u[:1], 200, G.GBN_MIXED)
    ac, bc = G.cheb_interval(a[0], b[0])
    c = G.cheb_coef(dt, ac, bc, npol)
    zero = np.zeros_like(psi)
    ctx.kubo_tevol(c, ac, bc, psi, zero, 1, 1, 10, 1, G.GBN_MIXED)   # warm-up (layout, kernels)

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return r, dist_max(e0.elapsed_time(e1), ws) / 1e3

    (_, _, nrm_m, _, _), t_msd = timed(lambda: ctx.kubo_tevol(c, ac, bc, psi, zero, nt_msd, nwr_msd, nrecurs, 1,
                                                             G.GBN_MIXED))
    dt_fs = dt * HBAR_EV_S / g0 * 1e15
    t_fs, msd, d_ratio, d_slope = G.kubo_msd(nrm_m, nwr_msd, dt_fs)
    (p1, z1, nrm, _, _), t_dev = timed(lambda: ctx.kubo_tevol(c, ac, bc, psi, zero, nt, nt, nrecurs, 1, G.GBN_MIXED))

    def host_loop():
        p, z = psi, zero
        for _ in range(nt):
            p, z = ctx.kubo_evol(c, ac, bc, p, z, direction=1, precision=G.GBN_MIXED)
        nz = np.sum(np.abs(z) ** 2, axis=1)
        ctx.lanczos(z / np.sqrt(nz)[:, None], nrecurs, G.GBN_MIXED)
        return nz

    nz, t_host = timed(host_loop)
    ctx.close()
    work = float(n) * nvec * (npol - 1) * nt
    work_m = float(n) * nvec * (npol - 1) * nt_msd
    msd_out = {"time_steps": nt_msd, "write_every": nwr_msd, "device_resident_s": t_msd,
               "atom_poly_steps_per_s": ws * work_m / t_msd,
               "extrapolated_1000_steps_s": t_msd * 1000.0 / nt_msd,
               "extrapolation": "the workload's 1000 time steps are 10 x these 100 (each step the same work)",
               "t_fs": [float(x) for x in t_fs], "msd_ang2": [float(x) for x in msd],
               "msd_over_t_ang2_per_fs": [float(x) for x in d_ratio],
               "dmsd_dt_ang2_per_fs": [float(x) for x in d_slope],
               "accumulation": "FP64 (norms reduced in FP64, complex64 vectors, FP64 accumulators)"}
    return {"workload": "graphene_hbn_0.61deg_anderson_3527168atoms_8vec_dt1fs", "atoms": n, "vectors": nvec,
            "msd_diffusivity": msd_out,
            "npol": npol, "time_steps": nt, "dt_g0_over_hbar": dt, "atom_poly_steps": work,
            "device_resident_s": t_dev, "device_resident_atom_poly_steps_per_s": ws * work / t_dev,
            "host_states_s": t_host, "host_states_atom_poly_steps_per_s": ws * work / t_host,
            "speedup_vs_host_states": t_host / t_dev,
            "norm_rel_diff": float(np.abs(nrm[:, 0] - nz).max() / np.abs(nz).max()), "precision": "mixed"}


GRAD_KEYS = {"Run.TypeOfSystem": "TwistedBilayerBasedOnMoireCell", "Structure.MoireCellParameters": (32, 31, 31, 32),
             "Structure.SuperCell": 9, "Interlayer.TypeOfBL": "Koshino", "Interlayer.Vpppi0": 2.7,
             "Interlayer.Vppsigma0": 0.48, "Interlayer.BLdelta": 0.319, "Neigh.LayerNeighbors": 100,
             "Neigh.LayerDistFactor": 3.2005, "TB.Hopping": 2.7, "Kubo.SeedValue": 3}


def gradient_leg(G, M, local, stream, ws, nrecurs=600, checkpoint=32):
    """Gradient of a DOS loss of twisted bilayer graphene at 1.05 degrees (cell 32 31 31 32 tiled 9 x 9 =
    964,548 atoms, two-centre interlayer hopping with a smooth cutoff of width 0.5 Ang): L = sum_E (DOS -
    target)^2, eta = 5 meV, 2001 energies on [-1, 1] eV, target from parameters perturbed by 2 % (seed
    3), 600 recursion steps (FP64) with checkpoints every 32 steps.  One gbn_dos_gradient (forward sweep,
    loss and the reverse sweep for dL/d(t, Vpp_sigma0, delta, w)) against the assembly plus the forward
    recursion alone."""
    import torch
    from grabnes_b200 import autograd as AD
    ctx = G.Context(local)
    ctx.set_stream(stream.cuda_stream)
    job = M.job_from_keys(GRAD_KEYS)
    theta = np.array([2.7, 0.48, 0.319, 0.5])
    prob = AD.DosProblem(ctx, job, None, nrecurs, 0.005, 2000, -1.0, 1.0, checkpoint=checkpoint)
    rng = np.random.default_rng(3)
    _, _, target = prob.evaluate(theta * (1.0 + 0.02 * rng.uniform(-1, 1, 4)))
    prob.target = target

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return r, dist_max(e0.elapsed_time(e1), ws) / 1e3

    (loss, grad, _), t_grad = timed(lambda: prob.evaluate(theta))   # assembly, forward and reverse sweeps
    m = AD.model_with(prob.base, prob.g0, theta)

    def forward():   # the same assembly and an FP64 recursion of the same vector (its layout built anew)
        ctx.assemble(m, prob.rat_on, prob.rat_hop, None)
        return ctx.lanczos_phases(prob.u, nrecurs, G.GBN_FP64)

    _, t_fwd = timed(forward)
    n = prob.n
    ctx.close()
    return {"workload": "tbg_1.05deg_9x9_964548atoms_600steps_checkpoint32", "atoms": n, "recursion_steps": nrecurs,
            "checkpoint": checkpoint, "gradient_s": t_grad, "forward_recursion_s": t_fwd,
            "gradient_over_forward": t_grad / t_fwd, "loss": float(loss), "gradient": [float(x) for x in grad],
            "precision": "fp64"}


MOIRE_DOS_KEYS = {k: v for k, v in TEVOL_KEYS.items() if not k.startswith("Disorder.")}


def best_of_each_form(cands):
    """The autotuner's fastest candidate of each step form: two launches (product + update) and fused."""
    out = {}
    for form, sel in (("two_launches", lambda r: r.get("fused", -1) != 1), ("fused", lambda r: r.get("fused", -1) == 1)):
        ok = [r for r in cands if "step_ms" in r and sel(r)]
        if ok:
            out[form] = min(ok, key=lambda r: r["step_ms"])
    return out


def fixed_tuning(spec):
    """A tuning dictionary from 'rhs_per_thread,blocks_per_sm,rows_per_group,staged,prefetch[,unroll
    [,stage_values[,min_blocks[,fused]]]]'."""
    vals = [int(x) for x in spec.split(",")]
    names = ["rhs_per_thread", "blocks_per_sm", "rows_per_group", "staged", "prefetch", "unroll", "stage_values",
             "min_blocks", "fused"]
    best = dict(unroll=0, stage_values=-1, min_blocks=0, fused=-1, fixed=True)
    best.update(zip(names, vals))
    return best


def moire_dos_leg(G, M, local, stream, ws, nrhs=16, nsteps=2000, peak=None, tuning=""):
    """Batched mixed-precision Lanczos DOS of graphene on hBN at 0.61 degrees (example 07's cell, CellSize
    83, SuperCell 16 = 3,527,168 atoms, effective moire model with the midpoint bond term): 16 random-
    phase vectors (GNU RNG seed 123456 + k), 2000 steps, autotuned kernels, start vectors resident;
    against the plain FP64 single-vector path on the same cell, and the DOS of the two against each other
    (eta 5 meV, 1201 energies on [-0.6, 0.6] eV as in the example)."""
    import torch
    from grabnes_b200.tune import autotune
    job = M.job_from_keys(MOIRE_DOS_KEYS)
    ctx = G.Context(local)
    ctx.set_stream(stream.cuda_stream)
    cell = M.setup(ctx, job)
    n, nnz, g0 = cell["n"], ctx.neighbours_total, job["g0"]
    u = np.stack([G.rng_uniform(123456 + k, n) for k in range(nrhs)])
    if tuning:
        from grabnes_b200.tune import apply
        best = fixed_tuning(tuning)
        apply(ctx, best)
    else:
        best, cands = autotune(ctx, u, G.GBN_MIXED)
        best = dict(best, candidates_top5=sorted((r for r in cands if "step_ms" in r),
                                                  key=lambda r: r["step_ms"])[:5],
                    best_of_each_step_form=best_of_each_form(cands))
    ctx.stage_phases(u, G.GBN_MIXED)
    ctx.run_staged(200)
    torch.cuda.synchronize()
    ctx.run_staged(nsteps)
    ms, k = ctx.last_timing()
    spmm_ms, upd_ms = ctx.kernel_timing()
    a_mix = np.zeros((nrhs, nsteps))
    b_mix = np.zeros((nrhs, nsteps))
    ctx.run_staged(nsteps, a_mix, b_mix)
    ms2, _ = ctx.last_timing()
    ctx.set_tuning()
    ctx.set_kernel_variant()
    a64, b64 = ctx.lanczos_phases(u[:1], nsteps, G.GBN_FP64)
    ms64, _ = ctx.last_timing()
    _, d_mix = ctx.cf_dos(a_mix[:1], b_mix[:1], 0.005 / g0, 1200, -0.6 / g0, 0.6 / g0)
    _, d_64 = ctx.cf_dos(a64, b64, 0.005 / g0, 1200, -0.6 / g0, 0.6 / g0)
    ctx.close()
    b_alg = nnz * (4 + 4) + n * 4 + nrhs * n * 3 * 8
    ach = b_alg / (spmm_ms / 1e3) / 1e9
    step = min(ms, ms2) / nsteps
    kname = kernel_key(best)
    traffic, traffic_src = traffic_from_profile(kname, "moire_dos")
    return {"workload": "graphene_hbn_0.61deg_3527168atoms_16vec_2000steps", "atoms": n, "entries": nnz,
            "vectors": nrhs, "recursion_steps": nsteps, "tuning": best,
            "batched_mixed_atom_steps_per_s": ws * n * nrhs / (step / 1e3),
            "fp64_single_vector_atom_steps_per_s": ws * n / (ms64 / nsteps / 1e3),
            "step_ms": step, "spmm_ms": spmm_ms, "update_ms": upd_ms,
            "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": (ach / peak) if peak else None, "algorithmic_bytes_per_launch": b_alg,
                         "kernel": kname, "traffic": traffic, "traffic_source": traffic_src,
                         # the DRAM bytes the kernel actually moves (ncu) over its live launch time; the
                         # fused step's kernel is the whole step and moves 32 of every 24 algorithmic bytes
                         "traffic_frac": (traffic / (spmm_ms / 1e3) / 1e9 / peak) if (traffic and peak) else None,
                         "kernel_is_whole_step": best.get("fused", -1) == 1},
            "step_frac": (b_alg / (step / 1e3) / 1e9 / peak) if peak else None,
            "step_achieved_gbs": b_alg / (step / 1e3) / 1e9,
            "dos_error_vs_fp64_vector0": float(np.abs(d_mix[0] - d_64[0]).sum() / np.abs(d_64[0]).sum())}


_HOST_TABLES = {}


def host_tables(ctx):
    """The context's neighbour tables and Hamiltonian in the reference layout, copied to the host once."""
    if id(ctx) not in _HOST_TABLES:
        tabs = ctx.tables()
        h0, hop = ctx.hamiltonian()
        _HOST_TABLES.clear()
        _HOST_TABLES[id(ctx)] = (tabs, h0, hop)
    return _HOST_TABLES[id(ctx)]


def oracle_dos_error(ctx, n, u0, nsteps, a_mix, b_mix, a64, b64, g0):
    """Normalised L1 error of the DOS of one start vector, mixed precision and FP64 on the device, against
    the oracle's FP64 recursion of the same vector on the same Hamiltonian (reference layout, complex128)."""
    from oracle import oracle as orc
    tabs, h0, hop = host_tables(ctx)
    psi = np.exp(2j * np.pi * u0) / np.sqrt(n)
    t0 = time.perf_counter()
    a0, b0 = orc.recursion(tabs, hop, h0, psi, nsteps, cpu_count())
    dt = time.perf_counter() - t0
    args = (ETA_EV / g0, NE, EMIN_EV / g0, EMAX_EV / g0)
    _, d0 = orc.frac(a0, b0, *args)
    _, dm = ctx.cf_dos(a_mix[None, :], b_mix[None, :], *args)
    _, d6 = ctx.cf_dos(a64[None, :], b64[None, :], *args)
    l1 = lambda d: float(np.abs(d[0] - d0).sum() / np.abs(d0).sum())
    k = min(200, nsteps)
    return {"vector": 0, "recursion_steps": nsteps, "eta_ev": ETA_EV, "energies": NE + 1,
            "l1_mixed": l1(dm), "l1_fp64": l1(d6),
            "ab_rel_fp64_first200": float(max(np.abs(a64[:k] - a0[:k]).max(), np.abs(b64[:k] - b0[:k]).max())
                                          / np.abs(b0[:k]).max()),
            "oracle_s": dt, "oracle_cores": cpu_count()}


def cpu_baseline(ctx, n, u0, steps):
    """The oracle port of KuboRecursion (reference data layout, complex128, three passes per step)."""
    from oracle import oracle as orc
    tabs, h0, hop = host_tables(ctx)
    psi = np.exp(2j * np.pi * u0) / np.sqrt(n)
    cores = cpu_count()
    orc.recursion(tabs, hop, h0, psi, 1, cores)   # first touch
    t0 = time.perf_counter()
    orc.recursion(tabs, hop, h0, psi, steps, cores)
    dt = time.perf_counter() - t0
    return {"value": n * steps / dt, "unit": "atom-steps/s", "cores": cores, "kind": "port",
            "sample": f"1 vector x {steps} recursion steps on the full {n}-atom Hamiltonian (complex128, "
                      f"reference layout), {dt:.2f} s"}


# ------------------------------------------------------------------------------------- reference
def run_reference(args, ws, rank):
    """The reference's CPU algorithm (oracle port: Fortran + MPI are not available) on the host cores."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle import oracle as orc
    import refcases as R
    cores = cpu_count()
    keys = {k.split(".")[-1]: v for k, v in WORKLOAD.items()}
    keys["Hopping"] = WORKLOAD["TB.Hopping"]
    keys["NeighLevels"] = 1
    t0 = time.time()
    r = R.build(keys)
    setup_s = time.time() - t0
    n = r["geo"]["n"]
    psi = orc.init_wf(n, SEED)
    # one short first-touch run, which also sizes the samples to about 15 s of CPU work each (at most
    # --cpu-steps); the CPU needs no further warm-up, so W only bounds it
    t = time.perf_counter()
    probe = 20
    orc.recursion(r["nb"], r["hop"], r["h0"], psi, probe, cores)
    rate = probe / (time.perf_counter() - t)
    steps = int(max(20, min(args.cpu_steps, 15.0 * rate)))
    ts = []
    for _ in range(args.steps):
        t = time.perf_counter()
        orc.recursion(r["nb"], r["hop"], r["h0"], psi, steps, cores)
        ts.append(time.perf_counter() - t)
    per = statistics.median(ts)
    value = n * steps / per
    out = {"metric": METRIC, "value": value, "unit": "atom-steps/s", "n_gpus": ws, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": per * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "c128", "data": "synthetic (reference model)", "impl": "reference",
           "config": {"workload": WORKLOAD_NAME, "atoms": n, "sample_steps": steps, "vectors": 1,
                      "same_config": False,
                      "extrapolation": f"the workload is {NRHS} vectors x {NSTEPS} steps; each bench step times 1 "
                                       f"vector x {steps} steps of the same Hamiltonian, and the rate is per "
                                       f"atom-step, which the CPU recursion's cost is linear in (each step is "
                                       f"three passes over the same arrays)"},
           "cpu_baseline": {"value": value, "unit": "atom-steps/s", "cores": cores, "kind": "port",
                            "sample": f"1 vector x {steps} recursion steps of the full {n}-atom Hamiltonian per bench "
                                      f"step (complex128, reference layout; setup {setup_s:.0f} s untimed)"},
           "e2e": {"value": value, "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--cpu-steps", type=int, default=300, help="recursion steps of the CPU sample")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-oracle-dos", action="store_true", help="skip the oracle DOS check of vector 0")
    p.add_argument("--supercell", type=int, default=20, help="moire cells per side (20 = the workload)")
    p.add_argument("--nsteps", type=int, default=NSTEPS, help="recursion steps per job (2000 = the workload)")
    p.add_argument("--value-only", action="store_true", help="time the device-resident jobs only (profiling)")
    p.add_argument("--no-fields", action="store_true", help="skip the batched-field sweep (graphene/hBN, 33 fields)")
    p.add_argument("--fields-only", action="store_true", help="run the batched-field sweep alone")
    p.add_argument("--no-tevol", action="store_true", help="skip the Chebyshev Kubo time evolution leg")
    p.add_argument("--no-gradient", action="store_true", help="skip the DOS-gradient leg")
    p.add_argument("--no-moire-dos", action="store_true", help="skip the 3.5M-atom graphene/hBN DOS leg")
    p.add_argument("--moire-dos-only", action="store_true", help="run the 3.5M-atom graphene/hBN DOS leg alone")
    p.add_argument("--gradient-only", action="store_true", help="run the DOS-gradient leg alone")
    p.add_argument("--tevol-only", action="store_true", help="run the Chebyshev Kubo time evolution leg alone")
    p.add_argument("--fields-scale", type=float, default=1.0, help="scale of the sweep's recursion lengths (profiling)")
    p.add_argument("--tuning", default="", help="fixed kernel tuning 'rhs_per_thread,blocks_per_sm,rows_per_group,staged,prefetch"
                                                "[,unroll[,stage_values[,min_blocks]]]' instead of the autotuner")
    p.add_argument("--moire-steps", type=int, default=2000, help="recursion steps of the graphene/hBN DOS leg")
    args = p.parse_args()
    ws, rank, local = dist_init() if args.impl == "ours" else (int(os.environ.get("WORLD_SIZE", "1")),
                                                                 int(os.environ.get("RANK", "0")), 0)
    if args.impl == "reference":
        run_reference(args, ws, rank)
    else:
        run_ours(args, ws, rank, local)


if __name__ == "__main__":
    main()
