"""Autotuner of the recursion kernels.

Candidates: rows per group of the matrix layout (1 = plain sliced ELL; 2, 4 = neighbouring rows share
one gather per union column), right-hand sides per thread (the width of each thread's vector loads,
and with it the groups a warp processes per slice), the matrix path (slice records staged in shared
memory by per-warp bulk copies, or read from global memory), the union columns whose gathers are in
flight together (4 or 8), a prefetch (staged path only) of the gather rows of each slice, of the rows
its epilogue reads, or of those and the rows of u_k one or more sweeps ahead, and a cap on resident
blocks per SM, and the fused step (the update folded into the product, one launch per step; real FP32
layouts at the widest loads).  The search runs in two stages on the caller's own Hamiltonian and start
vectors: the layout and path (rows per group, right-hand sides per thread, staged or not) at the default
variant, then, for the best layout of each rows-per-group value, the variant (unroll, prefetch, staged
values or indices, the register bound for 1, 2 or 3 blocks per SM, fused or two launches), and the same
for its staged layout at the widest vector loads.  Each candidate runs a short recursion; the one with
the smallest device time per step (update + sparse product, CUDA events) is kept on the context.
"""
import itertools


def _time(ctx, u, precision, nsteps, cand):
    grp, st, pf, rpt, bps, unroll, sv, mb, fu = cand
    what = dict(rows_per_group=grp, staged=st, prefetch=pf, rhs_per_thread=rpt, blocks_per_sm=bps, unroll=unroll,
                stage_values=sv, min_blocks=mb, fused=fu)
    try:
        ctx.set_tuning(rpt, bps, grp, st, pf)
        ctx.set_kernel_variant(unroll, sv, mb, -1, -1, fu)
        ctx.stage_phases(u, precision)
        ctx.run_staged(nsteps)
        ctx.run_staged(nsteps)
    except Exception as exc:   # a candidate the library refuses is skipped
        return dict(what, error=str(exc))
    spmm, upd = ctx.kernel_timing()
    return dict(what, spmm_ms=spmm, update_ms=upd, step_ms=spmm + upd)


def _key(r):
    return (r["rows_per_group"], r["staged"], r["prefetch"], r["rhs_per_thread"], r["blocks_per_sm"], r["unroll"],
            r["stage_values"], r["min_blocks"], r.get("fused", 0))


def apply(ctx, best):
    """Set a tuning dictionary (as returned by autotune) on the context."""
    ctx.set_tuning(best["rhs_per_thread"], best["blocks_per_sm"], best["rows_per_group"], best["staged"],
                   best["prefetch"])
    ctx.set_kernel_variant(best.get("unroll", 0), best.get("stage_values", -1), best.get("min_blocks", 0), -1, -1,
                           best.get("fused", -1))


def autotune(ctx, u, precision, nsteps=12, rhs_per_thread=(1, 2, 4), blocks_per_sm=(0,),
             rows_per_group=(1, 2, 4), staged=(0, 1), prefetch=(0, 4, 6), unroll=(4, 8)):
    results = []
    # stage 1: layout and matrix path at the library's default variant (-1/0: chosen by the library)
    for grp, st, rpt, bps in itertools.product(rows_per_group, staged, rhs_per_thread, blocks_per_sm):
        results.append(_time(ctx, u, precision, nsteps, (grp, st, -1, rpt, bps, 0, -1, 0, 0)))
    ok = [r for r in results if "step_ms" in r]
    # stage 2: for the best layout of every rows-per-group value, the unroll, prefetch, staged values or
    # indices only, and the register bound (1, 2 or 3 blocks per SM): the best variant differs between
    # layouts, so the layouts' defaults do not rank them
    seen = {_key(r) for r in results}
    layouts = []
    for grp in rows_per_group:
        mine = [r for r in ok if r["rows_per_group"] == grp]
        if not mine:
            continue
        layouts.append(min(mine, key=lambda r: r["step_ms"]))
        # and the staged layout at the widest loads (the variants often reorder the splits)
        wide = [r for r in mine if r["staged"] == 1 and r["rhs_per_thread"] == max(rhs_per_thread)]
        if wide and wide[0] is not layouts[-1]:
            layouts.append(wide[0])
    for lay in layouts:
        grp = lay["rows_per_group"]
        pfs = prefetch if lay["staged"] == 1 else (0,)
        for pf, un, sv, mb in itertools.product(pfs, unroll, (1, 0), (1, 2, 3)):
            if lay["staged"] != 1 and (sv == 0 or mb != 1):
                continue
            if mb > 1 and un != 8:
                continue
            if mb == 2 and sv == 0:
                continue
            cand = (grp, lay["staged"], pf, lay["rhs_per_thread"], lay["blocks_per_sm"], un, sv, mb, 0)
            if cand in seen:
                continue
            seen.add(cand)
            results.append(_time(ctx, u, precision, nsteps, cand))
        # the fused step: staged whole records, registers for one or two blocks per SM (the library refuses
        # shapes without it)
        if lay["staged"] == 1 and grp <= 2:
            uf = 4 if precision == 0 else 8   # the fused step's columns in flight: FP64 4, mixed 8
            for pf, mb in itertools.product(pfs, (1, 2)):
                cand = (grp, 1, pf, lay["rhs_per_thread"], lay["blocks_per_sm"], uf, 1, mb, 1)
                if cand in seen:
                    continue
                seen.add(cand)
                results.append(_time(ctx, u, precision, nsteps, cand))
    ok = [r for r in results if "step_ms" in r]
    best = min(ok, key=lambda r: r["step_ms"])
    apply(ctx, best)
    return best, results
