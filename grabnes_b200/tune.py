"""Autotuner of the recursion kernels.

Candidates: rows per group of the matrix layout (1 = plain sliced ELL; 2, 4 = neighbouring rows share
one gather per union column), right-hand sides per thread (the width of each thread's vector loads,
and with it the groups a warp processes per slice), the matrix path (slice records staged in shared
memory by per-warp bulk copies, or read from global memory), a prefetch (staged path only) of the
gather rows of each slice or of the rows its epilogue reads, and a cap on resident blocks per SM.
Each candidate runs a short recursion on the caller's own Hamiltonian and start vectors; the one with
the smallest device time per step (update + sparse product, CUDA events) is kept on the context.
"""
import itertools


def autotune(ctx, u, precision, nsteps=12, rhs_per_thread=(1, 2, 4), blocks_per_sm=(0,),
             rows_per_group=(1, 2, 4), staged=(0, 1), prefetch=(0, 1, 4)):
    results = []
    cands = [c for c in itertools.product(rows_per_group, staged, prefetch, rhs_per_thread, blocks_per_sm)
             if c[1] == 1 or c[2] == 0]   # the prefetch belongs to the staged path
    for grp, st, pf, rpt, bps in cands:
        try:
            ctx.set_tuning(rpt, bps, grp, st, pf)
            ctx.stage_phases(u, precision)
            ctx.run_staged(nsteps)
            ctx.run_staged(nsteps)
        except Exception as exc:   # a candidate the library refuses is skipped
            results.append(dict(rows_per_group=grp, staged=st, prefetch=pf, rhs_per_thread=rpt, blocks_per_sm=bps,
                                error=str(exc)))
            continue
        spmm, upd = ctx.kernel_timing()
        results.append(dict(rows_per_group=grp, staged=st, prefetch=pf, rhs_per_thread=rpt, blocks_per_sm=bps,
                            spmm_ms=spmm, update_ms=upd, step_ms=spmm + upd))
    ok = [r for r in results if "step_ms" in r]
    best = min(ok, key=lambda r: r["step_ms"])
    ctx.set_tuning(best["rhs_per_thread"], best["blocks_per_sm"], best["rows_per_group"], best["staged"],
                   best["prefetch"])
    return best, results
