"""Autotuner of the recursion kernels.

Candidates: right-hand sides per thread (the width of each thread's vector loads, and with it the rows
a warp processes per slice), a cap on resident blocks per SM, and the sparse-product variant (matrix
chunks staged in shared memory by bulk asynchronous copies, or read from global memory).  Each
candidate runs a short recursion on the caller's own Hamiltonian and start vectors; the one with the
smallest device time per step (update + sparse product, CUDA events) is kept on the context.
"""
import itertools


def autotune(ctx, u, precision, nsteps=12, rhs_per_thread=(1, 2, 4), blocks_per_sm=(0, 3, 4), staged=(0, 1)):
    results = []
    for st, rpt, bps in itertools.product(staged, rhs_per_thread, blocks_per_sm):
        try:
            ctx.set_tuning(rpt, bps, st)
            ctx.stage_phases(u, precision)
            ctx.run_staged(nsteps)
            ctx.run_staged(nsteps)
        except Exception as exc:   # a candidate the library refuses is skipped
            results.append(dict(staged=st, rhs_per_thread=rpt, blocks_per_sm=bps, error=str(exc)))
            continue
        spmm, upd = ctx.kernel_timing()
        results.append(dict(staged=st, rhs_per_thread=rpt, blocks_per_sm=bps, spmm_ms=spmm, update_ms=upd,
                            step_ms=spmm + upd))
    ok = [r for r in results if "step_ms" in r]
    best = min(ok, key=lambda r: r["step_ms"])
    ctx.set_tuning(best["rhs_per_thread"], best["blocks_per_sm"], best["staged"])
    return best, results
