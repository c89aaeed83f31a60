// Batched Lanczos recursion on the B200: two launches per recursion step, or one with the fused step.
//
// The reference (lanczosKuboCode/Src/kubosubs.F90:26-138) makes three passes over the vectors per
// step: H psi with <psi, H psi>; w = H psi - a psi - b psi_prev with |w|; the scaling psi = w / b.
// Here the carried vectors are unnormalised: x_k = u_k / b_{k-1}, and a step is
//   k_update    u_k = v_k - (a_{k-1} / b_{k-2}) u_{k-1}  and  b_{k-1} = |u_k|
//               (v_k - a_{k-1} x_{k-1} is the reference's w, b_{k-1} its norm; stream: read v, u_{k-1},
//               write u_k; one FP64 sum per vector)
//   k_spmm_*    y = H u_k (one gather of u_k per union column of a row group),
//               v_{k+1} = y / b_{k-1} - (b_{k-1} / b_{k-2}) u_{k-1}   (= H x_k - b_{k-1} x_{k-1})
//               and a_k = Re<u_k, y> / b_{k-1}^2 (one FP64 sum per vector).
// The first update takes the start vector as given (b = 1 for it, as the reference's first step uses
// Psi unnormalised) and a run of n steps ends with one more update, which gives b_{n-1}.  Each kernel's
// block partial sums are reduced in a fixed order by its last block to finish (so the result does not
// depend on scheduling), which also writes a_k or b_{k-1} and the scalars of the next launch.
//
// Vectors of R right-hand sides are interleaved per row ([row][R] complex): TPR threads share a row
// group, each holding RPT right-hand sides (8-32 bytes per gather).  With 16 vectors a gathered row is
// one 128-byte line.  The product is bound by the latency of the chain column index -> gather: the
// grouped layout (struct Ell) gathers a column once for the G rows of a group, the staged kernel
// brings each warp's next slice record (column indices, and values unless they stream beside the
// gathers) into shared memory with one bulk asynchronous copy, and U columns' gathers are in flight
// together, so that only the gathers themselves wait on memory.
//
// The fused step (kernel variant fused = 1; real FP32 layouts) folds k_update into the product: product k
// gathers v_k and u_{k-1} at every union column and forms u_k = v_k - alpha u_{k-1} (alpha = a_{k-1} / b_{k-2}
// rounded to FP32) with one packed FMA wherever the column is gathered, writes u_k and v_{k+1}, and sums
// Re<u_k, H u_k>, |v_{k+1}|^2 and Re<v_{k+1}, u_k>; its last block derives a_k and b_k (reduce_and_finalize).
// v then alternates between vec[0] and vec[3], u between vec[1] and vec[2], and no closing pass is needed.
#include <algorithm>

#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include "gbn_step.cuh"

namespace gbn {

// ---------------------------------------------------------------------------- update kernel
// u_k = v_k - (a_{k-1} / b_{k-2}) u_{k-1} for all rows and right-hand sides (streaming), and
// b_{k-1} = |u_k| from the stored (rounded) elements.  The grid stride and the block size are multiples
// of R, so every thread keeps one right-hand side; the block's sums are reduced per right-hand side in
// thread order, then by the last block over the blocks in a fixed order.
template <typename VT>
__global__ void __launch_bounds__(256) k_update(const typename V2<VT>::t* __restrict__ v,
                                                const typename V2<VT>::t* __restrict__ xp,
                                                typename V2<VT>::t* __restrict__ xc, double* scal, double* partials,
                                                unsigned int* counter, double* b_out, int nmax, int64_t total, int R)
{
    const int r = (int)(threadIdx.x & (unsigned)(R - 1));
    const double c = scal[kScal * r] / scal[kScal * r + 1];
    using C2 = typename V2<VT>::t;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    double q = 0.0;
    auto one = [&](C2 vv, C2 xx, int64_t e) {   // FP64 arithmetic, one rounding to the storage type
        C2 o;
        o.x = (VT)((double)vv.x - c * (double)xx.x);
        o.y = (VT)((double)vv.y - c * (double)xx.y);
        xc[e] = o;
        q += (double)o.x * (double)o.x + (double)o.y * (double)o.y;
    };
    // four elements per thread in flight: all eight loads are issued before the first use
    constexpr int D = 4;
    int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (; e + (D - 1) * stride < total; e += D * stride) {
        C2 vv[D], xx[D];
#pragma unroll
        for (int i = 0; i < D; ++i) {
            vv[i] = __ldcs(v + e + i * stride);
            xx[i] = __ldcs(xp + e + i * stride);
        }
#pragma unroll
        for (int i = 0; i < D; ++i) one(vv[i], xx[i], e + i * stride);
    }
    for (; e < total; e += stride) one(__ldcs(v + e), __ldcs(xp + e), e);
    // block: the 256 / R threads of each right-hand side, combined in a fixed tree
    __shared__ double rs[256], rc[256];
    rs[threadIdx.x] = q;
    rc[threadIdx.x] = 0.0;
    tree_fixed_sum(rs, rc, (int)blockDim.x / R, R);
    if ((int)threadIdx.x < R) partials[(int64_t)blockIdx.x * R + threadIdx.x] = rs[threadIdx.x] + rc[threadIdx.x];
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    __shared__ double tot[32];
    grid_fixed_sum(partials, (int)gridDim.x, R, rs, rc, tot);
    if ((int)threadIdx.x < R) {
        const double b = sqrt(tot[threadIdx.x]);
        const unsigned int step = counter[1];   // products done so far: this is b_{step-1}
        if (step > 0) {
            if (!(b > 0.0) || !isfinite(b)) atomicOr(&counter[2], 1u);
            if ((int)step <= nmax) b_out[(int64_t)threadIdx.x * nmax + step - 1] = b;
        }
        scal[kScal * threadIdx.x + 2] = scal[kScal * threadIdx.x + 1];
        scal[kScal * threadIdx.x + 1] = step > 0 ? b : 1.0;   // the start vector is used as given
    }
    __syncthreads();
    if (threadIdx.x == 0) counter[0] = 0u;
}

// ---------------------------------------------------------------------------- sparse product
// ---------------------------------------------------------------------------- start vectors
// v <- psi (rows in the solver order), u_prev <- 0; then the first update gives u_0 = psi (a = 0, norm 1).
template <typename VT>
__global__ void k_start_from_phases(typename V2<VT>::t* v, typename V2<VT>::t* x, const double* u,
                                    const int32_t* perm, int64_t n, int64_t npad, int R, int nrhs_real,
                                    double inv_sqrt_n)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npad * R) return;
    const int64_t row = i / R;
    const int r = (int)(i % R);
    typename V2<VT>::t z;
    z.x = 0; z.y = 0;
    if (row < n) {
        const int rr = r < nrhs_real ? r : 0;  // padding vectors repeat the first one
        const double ph = 6.283185307179586 * u[(int64_t)rr * n + perm[row]];
        double sn, cs;
        sincos(ph, &sn, &cs);
        z.x = (VT)(cs * inv_sqrt_n);
        z.y = (VT)(sn * inv_sqrt_n);
    }
    v[i] = z;
    typename V2<VT>::t zero;
    zero.x = 0; zero.y = 0;
    x[i] = zero;
}

template <typename VT>
__global__ void k_start_from_psi(typename V2<VT>::t* v, typename V2<VT>::t* x, const double2* psi,
                                 const int32_t* perm, int64_t n, int64_t npad, int R, int nrhs_real)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npad * R) return;
    const int64_t row = i / R;
    const int r = (int)(i % R);
    typename V2<VT>::t z;
    z.x = 0; z.y = 0;
    if (row < n) {
        const int rr = r < nrhs_real ? r : 0;
        const double2 s = psi[(int64_t)rr * n + perm[row]];
        z.x = (VT)s.x;
        z.y = (VT)s.y;
    }
    v[i] = z;
    typename V2<VT>::t zero;
    zero.x = 0; zero.y = 0;
    x[i] = zero;
}

// Unit vectors on single atoms (KuboInitWFPDOS): vector r of the tile is 1 on atom site[r] (0-based).
template <typename VT>
__global__ void k_start_from_sites(typename V2<VT>::t* v, typename V2<VT>::t* x, const int64_t* site,
                                   const int32_t* perm, int64_t n, int64_t npad, int R, int nrhs_real)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npad * R) return;
    const int64_t row = i / R;
    const int r = (int)(i % R);
    typename V2<VT>::t z;
    z.x = 0; z.y = 0;
    if (row < n && perm[row] == site[r < nrhs_real ? r : 0]) z.x = (VT)1;
    v[i] = z;
    typename V2<VT>::t zero;
    zero.x = 0; zero.y = 0;
    x[i] = zero;
}

// Random phases on one set of atoms per vector (KuboInitWFLayerDOS): atom a of set s = set0 + r takes
// exp(2 pi i draw[a]) / den[s].x / den[s].y (den.x = sqrt of the assumed count, den.y = the norm
// correction, 1 when none is made).
template <typename VT>
__global__ void k_start_from_sets(typename V2<VT>::t* v, typename V2<VT>::t* x, const int32_t* set_of_atom,
                                  const double* draw, const double2* den, const int32_t* perm, int64_t n,
                                  int64_t npad, int R, int set0, int nrhs_real)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npad * R) return;
    const int64_t row = i / R;
    const int r = (int)(i % R);
    typename V2<VT>::t z;
    z.x = 0; z.y = 0;
    if (row < n) {
        const int32_t a = perm[row];
        const int s = set0 + (r < nrhs_real ? r : 0);
        if (set_of_atom[a] == s) {
            double sn, cs;
            sincos(6.283185307179586 * draw[a], &sn, &cs);
            const double2 d = den[s];
            z.x = (VT)(cs / d.x / d.y);
            z.y = (VT)(sn / d.x / d.y);
        }
    }
    v[i] = z;
    typename V2<VT>::t zero;
    zero.x = 0; zero.y = 0;
    x[i] = zero;
}

__global__ void k_init_scalars(double* scal, unsigned int* counter, int R)
{
    const int r = threadIdx.x;
    if (r < R) {
        scal[kScal * r] = 0.0;
        scal[kScal * r + 1] = 1.0;
        scal[kScal * r + 2] = 1.0;
        scal[kScal * r + 3] = 0.0;
    }
    if (r == 0) {
        counter[0] = 0u;
        counter[1] = 0u;
        counter[2] = 0u;
    }
}

// ---------------------------------------------------------------------------- host side
// right-hand sides per thread: the widest vector load (32 bytes) unless the tuning asks for fewer
void split_rhs(int prec, int R, int want, int* rpt, int* tpr)
{
    const int maxr = (prec == GBN_MIXED) ? 4 : 2;
    int r = R < maxr ? R : maxr;
    if (want > 0 && want < r && R % want == 0) r = want;
    if (R / r > 32) r = R / 32;
    *rpt = r;
    *tpr = R / r;
}


static StepFn step_kernel(int prec, bool cplx, int G, int R, int want_rpt, bool staged, StepVariant v)
{
    int rpt, tpr;
    split_rhs(prec, R, want_rpt, &rpt, &tpr);
    if (prec == GBN_MIXED) return step_kernel_mixed(cplx, G, rpt, tpr, staged, v);
    return step_kernel_fp64(cplx, G, rpt, tpr, staged, v);
}

// Launch shape of the sparse product.  Staged: warps per block such that two record buffers per warp
// fit the shared-memory budget.  cap: bytes of one buffer (whole records, or their column indices).
struct StepLaunch {
    StepFn fn = nullptr;
    int grid = 0, block = 256;
    size_t smem = 0;
    int64_t cap = 0;
    bool staged = false;
    const unsigned char* mat = nullptr;   // the records the kernel reads (the layout's, or its tile table)
    int64_t entry_bytes = 0;
    bool tiled = false;                   // the tile-local product (halo rows in shared memory)
    bool fused = false;                   // the update folded into the product (no update launches)
    int32_t pitch = 0, halo_off = 0;
};

constexpr size_t kStagedSmemBudget = 200 * 1024;
// blocks per SM of the streaming update kernel
constexpr int kUpdateBlocksPerSM = 8;

// The tile-local product (k_spmm_tiled), mixed precision and real values: 8 warps, two staging buffers
// per warp of the largest record percentile that leaves a halo buffer of at least 256 rows, with the
// blocks the registers allow (at most 2) per SM; the tiles are rebuilt when their halo limit changes.
// Returns false (and leaves L untouched) when the shape has no such kernel or nothing fits.
static int tiled_launch(gbn_ctx* c, int R, StepLaunch* L, bool* done)
{
    *done = false;
    Ell& E = c->ell;
    if (E.field || E.cplx || c->prec != GBN_MIXED) return GBN_OK;
    int rpt, tpr;
    split_rhs(c->prec, R, c->tune_rpt, &rpt, &tpr);
    StepFn fn = tiled_kernel_mixed(E.G, rpt, tpr, c->tune_min_blocks == 2 ? 2 : 1);
    if (!fn) return GBN_OK;
    int smem_sm = 0, resv = 0, optin = 0, reg_blocks = 0;
    GBN_CK(c, cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, c->device));
    GBN_CK(c, cudaDeviceGetAttribute(&resv, cudaDevAttrReservedSharedMemoryPerBlock, c->device));
    GBN_CK(c, cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
    cudaFuncAttributes fa;
    GBN_CK(c, cudaFuncGetAttributes(&fa, fn));
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&reg_blocks, fn, 256, 0) != cudaSuccess || reg_blocks < 1)
        reg_blocks = 1;
    const int target = reg_blocks < 2 ? reg_blocks : 2;
    int64_t budget = (int64_t)smem_sm / target - (int64_t)fa.sharedSizeBytes - resv;
    if (budget > optin - (int64_t)fa.sharedSizeBytes) budget = optin - (int64_t)fa.sharedSizeBytes;
    const int pitch = R * (int)sizeof(float2) + 16;
    constexpr int kMinHalo = 256;
    for (int i = 0; i < 4; ++i) {
        const int64_t cap = E.cap_pct[i];
        if (cap <= 0) continue;
        const int64_t stage = 128 + 8 * 2 * cap;
        const int64_t hmax = (budget - stage) / pitch;
        if (hmax < kMinHalo) continue;
        const int hm = (int)std::min<int64_t>(hmax, 4096);
        if (!E.tiles_valid || E.tile_hmax != hm) {
            const int rc = build_tiles(c, hm);
            if (rc) return rc;
        }
        L->fn = fn;
        L->tiled = true;
        L->staged = true;
        L->cap = cap;
        L->pitch = pitch;
        L->halo_off = (int32_t)stage;
        L->block = 256;
        L->smem = (size_t)stage + (size_t)hm * pitch;
        L->mat = E.tmat.as<unsigned char>();
        L->entry_bytes = E.entry_bytes;
        GBN_CK(c, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L->smem));
        *done = true;
        return GBN_OK;
    }
    return GBN_OK;
}

static int step_launch(gbn_ctx* c, int R, StepLaunch* L)
{
    const Ell& E = c->ell;
    if (E.nslices * E.gpw * E.G > E.npad)   // the epilogue and its prefetch address whole slices of rows
        return fail(c, GBN_ERR_ARG, "internal: matrix slices cover more rows than the vectors hold");
    // defaults (measured on the 4.47M-atom twisted bilayer and the 3.5M-atom graphene/hBN cell with 16
    // vectors, and on 80k/1.1M-atom cells with one vector): 8 columns in flight in mixed precision, 4 in
    // FP64; with 8 columns and one row per group, registers bounded for 3 blocks per SM
    StepVariant v;
    // FP64: 4 columns in flight, 8 for one vector on a low-degree cell (with auto_group's one row per group)
    const bool fp64_single_low = c->prec == GBN_FP64 && R == 1 && c->n > 0 && c->total < 8 * c->n;
    v.unroll = c->tune_unroll > 0 ? c->tune_unroll : (c->prec == GBN_MIXED || fp64_single_low ? 8 : 4);
    v.stage_values = c->tune_stage_values != 0;
    v.min_blocks = c->tune_min_blocks > 0 ? c->tune_min_blocks : (v.unroll == 8 && E.G == 1 && !E.cplx ? 3 : 1);
    // the update folded into the product (see k_spmm_staged), its registers bounded for two blocks per SM
    // unless another bound is asked for.  By default where rows hold at most 8 entries on average: one launch
    // per step there was 3-24 % faster in mixed precision and 10-95 % faster in FP64 on graphene and
    // graphene/hBN cells of 15k-3.5M atoms with 8-32 vectors, and the doubled gathers made it slower on the
    // twisted bilayer's 33 entries per row (mixed: 504 against 387 us per step, 1.1M atoms, 16 vectors).
    // One mixed vector: equal or faster (387k-atom graphene/hBN 18.5 against 23.4 us); one FP64 vector stays
    // on two launches (3.5M-atom graphene/hBN 121 against 110 us, 1.28M-atom graphene 53 against 50)
    const bool fp64_single = c->prec == GBN_FP64 && R == 1;
    const bool fused_default = c->tune_fused < 0 && c->n > 0 && c->total <= 8 * c->n && !fp64_single;
    const StepVariant v_two = v;
    v.fused = c->tune_fused == 1 || fused_default;
    if (v.fused && c->tune_min_blocks <= 0) v.min_blocks = 2;
    // batched fields rotate on the fly unless the tile table is asked for (measured slower on example 06's
    // sweep: 0.175 against 0.108 ms per product, the table's complex values per thread slot triple the
    // records' bytes)
    const bool use_table = E.field && c->tune_field_table == 1 && E.ftab_valid;
    L->mat = use_table ? E.ftab.as<unsigned char>() : E.mat.as<unsigned char>();
    L->entry_bytes = use_table ? E.ftab_entry_bytes : E.entry_bytes;
    // buffer bytes of a record of percentile i: whole records, or their index part (multiples of 16)
    auto cap_of = [&](int i) -> int64_t {
        const int64_t nent = E.cap_pct[i] / E.entry_bytes;
        return ((v.stage_values ? nent * L->entry_bytes : nent * 4) + 15) / 16 * 16;
    };
    const bool want_staged = c->tune_staged != 0 && cap_of(0) > 0;
    // the kernel of this variant; shapes without it take the base variant unless one was asked for
    const bool asked = c->tune_unroll > 0 || c->tune_stage_values >= 0 || c->tune_min_blocks > 0 || c->tune_fused == 1;
    auto pick = [&](bool staged) -> StepFn {
        int rpt, tpr;
        split_rhs(c->prec, R, c->tune_rpt, &rpt, &tpr);
        const StepVariant base;
        if (E.field) {
            if (v.fused)   // the fused step of the field layout: whole records staged, 4 columns in flight
                return (staged && !use_table && !(c->tune_unroll > 0 && c->tune_unroll != 4))
                           ? field_fused_kernel(c->prec, E.G, rpt, tpr, v.min_blocks == 2 ? 2 : 1) : nullptr;
            if (!((v.unroll == 4 && v.stage_values && v.min_blocks == 1) || !asked)) return nullptr;
            if (use_table)
                return E.ftab_slots == tpr ? field_table_kernel(c->prec, E.G, rpt, tpr, staged) : nullptr;
            return field_step_kernel(c->prec, E.G, rpt, tpr, staged);
        }
        StepFn f = step_kernel(c->prec, E.cplx, E.G, R, c->tune_rpt, staged, v);
        if (!f && v.fused && fused_default) return nullptr;   // the caller takes the two-launch step
        if (!f && !asked) f = step_kernel(c->prec, E.cplx, E.G, R, c->tune_rpt, staged, base);
        return f;
    };
    L->fn = pick(want_staged);
    if (!L->fn && fused_default) {   // no fused kernel for this shape: the two-launch step
        v = v_two;
        L->fn = pick(want_staged);
    }
    if (!L->fn) return fail(c, GBN_ERR_ARG, "no recursion kernel for this tile width and kernel variant");
    L->fused = v.fused;
    L->block = 256;
    L->smem = 0;
    L->staged = false;
    L->cap = 0;
    if (want_staged) {
        // Shared memory per block such that the blocks the registers allow (at most 3) fit on an SM with
        // their static shared memory: 8 warps with the largest record percentile whose two buffers per
        // warp fit (larger records are read in place), else fewer warps with the 99.5th percentile.
        int smem_sm = 0, resv = 0, optin = 0, reg_blocks = 0;
        GBN_CK(c, cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, c->device));
        GBN_CK(c, cudaDeviceGetAttribute(&resv, cudaDevAttrReservedSharedMemoryPerBlock, c->device));
        GBN_CK(c, cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
        cudaFuncAttributes fa;
        GBN_CK(c, cudaFuncGetAttributes(&fa, L->fn));
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&reg_blocks, L->fn, 256, 0) != cudaSuccess || reg_blocks < 1)
            reg_blocks = 1;
        int target = reg_blocks < 3 ? reg_blocks : 3;
        if (c->tune_blocks_per_sm > 0 && c->tune_blocks_per_sm < target) target = c->tune_blocks_per_sm;
        int64_t budget = (int64_t)smem_sm / target - (int64_t)fa.sharedSizeBytes - resv;
        if (budget > optin - (int64_t)fa.sharedSizeBytes) budget = optin - (int64_t)fa.sharedSizeBytes;
        int64_t cap = 0;
        int nw = 0;
        for (int i = 0; i < 4 && !cap; ++i)
            if (cap_of(i) > 0 && 128 + 8 * 2 * cap_of(i) <= budget) {
                cap = cap_of(i);
                nw = 8;
            }
        if (!cap && 128 + 2 * cap_of(0) <= budget) {
            cap = cap_of(0);
            nw = (int)((budget - 128) / (2 * cap));
            nw = nw > 8 ? 8 : nw;
        }
        if (cap) {
            L->staged = true;
            L->cap = cap;
            L->block = 32 * nw;   // >= 32 threads: R <= 32 threads read the step's scalars
            L->smem = 128 + (size_t)nw * 2 * cap;
            GBN_CK(c, cudaFuncSetAttribute(L->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L->smem));
        }
    }
    if (want_staged && !L->staged) {   // no buffer fits: the plain kernel
        if (fused_default && v.fused) {   // the fused step is staged only
            v = v_two;
            L->fused = false;
        }
        L->fn = pick(false);
        if (!L->fn) return fail(c, GBN_ERR_ARG, "no recursion kernel for this tile width and kernel variant");
    }
    if (c->tune_tiled == 1 && !L->fused) {   // the tile-local product where the shape has one
        bool done = false;
        const int rc = tiled_launch(c, R, L, &done);
        if (rc) return rc;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, L->fn, L->block, L->smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    if (c->tune_blocks_per_sm > 0 && c->tune_blocks_per_sm < per_sm) per_sm = c->tune_blocks_per_sm;
    L->grid = c->num_sms * per_sm;
    return GBN_OK;
}

int lanczos_prepare(gbn_ctx* c, int prec, int nrhs, bool field)
{
    if (nrhs != 1 && nrhs != 2 && nrhs != 4 && nrhs != 8 && nrhs != 16 && nrhs != 32)
        return fail(c, GBN_ERR_ARG, "internal: tile width must be 1, 2, 4, 8, 16 or 32");
    int rpt, tpr;
    split_rhs(prec, nrhs, c->tune_rpt, &rpt, &tpr);
    const int gpw = 32 / tpr;
    const int G = c->tune_group > 0 ? c->tune_group : auto_group(c, nrhs, prec);
    if (!c->ell.valid || c->ell.prec != prec || c->ell.gpw != gpw || c->ell.G != G || c->ell.field != field) {
        const int rc = build_ell(c, prec, G, gpw, field);
        if (rc) return rc;
    }
    c->prec = prec;
    c->nrhs = nrhs;
    const size_t esz = (prec == GBN_MIXED) ? sizeof(float2) : sizeof(double2);
    const size_t vbytes = (size_t)c->ell.npad * nrhs * esz;
    for (int i = 0; i < 3; ++i) GBN_CK(c, c->vec[i].ensure(vbytes));
    StepLaunch L;
    const int rc = step_launch(c, nrhs, &L);
    if (rc) return rc;
    if (L.fused) GBN_CK(c, c->vec[3].ensure(vbytes));   // the fused step keeps v_k and v_{k+1}
    const size_t blocks = (size_t)(L.grid > c->num_sms * kUpdateBlocksPerSM ? L.grid : c->num_sms * kUpdateBlocksPerSM);
    GBN_CK(c, c->partials.ensure(sizeof(double) * blocks * nrhs * (L.fused ? 3 : 1)));
    GBN_CK(c, c->scal.ensure(sizeof(double) * kScal * nrhs));
    GBN_CK(c, c->counter.ensure(sizeof(unsigned int) * 4));
    return GBN_OK;
}

int lanczos_start_from_phases(gbn_ctx* c, const double* d_u, int nrhs_real)
{
    const int64_t tot = c->ell.npad * c->nrhs;
    const int blk = 256;
    const int64_t grd = (tot + blk - 1) / blk;
    const double isn = 1.0 / sqrt((double)c->n);
    if (c->prec == GBN_MIXED)
        k_start_from_phases<float><<<grd, blk, 0, c->stream>>>(c->vec[0].as<float2>(), c->vec[1].as<float2>(), d_u,
                                                               c->ell.rperm.as<int32_t>(), c->n, c->ell.npad, c->nrhs,
                                                               nrhs_real, isn);
    else
        k_start_from_phases<double><<<grd, blk, 0, c->stream>>>(c->vec[0].as<double2>(), c->vec[1].as<double2>(),
                                                                d_u, c->ell.rperm.as<int32_t>(), c->n, c->ell.npad,
                                                                c->nrhs, nrhs_real, isn);
    GBN_CK_LAUNCH(c);
    return GBN_OK;
}

int lanczos_start_from_psi(gbn_ctx* c, const double* d_psi, int nrhs_real)
{
    const int64_t tot = c->ell.npad * c->nrhs;
    const int blk = 256;
    const int64_t grd = (tot + blk - 1) / blk;
    if (c->prec == GBN_MIXED)
        k_start_from_psi<float><<<grd, blk, 0, c->stream>>>(c->vec[0].as<float2>(), c->vec[1].as<float2>(),
                                                            reinterpret_cast<const double2*>(d_psi),
                                                            c->ell.rperm.as<int32_t>(), c->n, c->ell.npad, c->nrhs,
                                                            nrhs_real);
    else
        k_start_from_psi<double><<<grd, blk, 0, c->stream>>>(c->vec[0].as<double2>(), c->vec[1].as<double2>(),
                                                             reinterpret_cast<const double2*>(d_psi),
                                                             c->ell.rperm.as<int32_t>(), c->n, c->ell.npad, c->nrhs,
                                                             nrhs_real);
    GBN_CK_LAUNCH(c);
    return GBN_OK;
}

int lanczos_start_from_sites(gbn_ctx* c, const int64_t* d_site, int nrhs_real)
{
    const int64_t tot = c->ell.npad * c->nrhs;
    const int blk = 256;
    const int64_t grd = (tot + blk - 1) / blk;
    if (c->prec == GBN_MIXED)
        k_start_from_sites<float><<<grd, blk, 0, c->stream>>>(c->vec[0].as<float2>(), c->vec[1].as<float2>(), d_site,
                                                              c->ell.rperm.as<int32_t>(), c->n, c->ell.npad, c->nrhs,
                                                              nrhs_real);
    else
        k_start_from_sites<double><<<grd, blk, 0, c->stream>>>(c->vec[0].as<double2>(), c->vec[1].as<double2>(),
                                                               d_site, c->ell.rperm.as<int32_t>(), c->n, c->ell.npad,
                                                               c->nrhs, nrhs_real);
    GBN_CK_LAUNCH(c);
    return GBN_OK;
}

int lanczos_start_from_sets(gbn_ctx* c, const int32_t* d_set, const double* d_draw, const double* d_den, int set0,
                            int nrhs_real)
{
    const int64_t tot = c->ell.npad * c->nrhs;
    const int blk = 256;
    const int64_t grd = (tot + blk - 1) / blk;
    const double2* den = reinterpret_cast<const double2*>(d_den);
    if (c->prec == GBN_MIXED)
        k_start_from_sets<float><<<grd, blk, 0, c->stream>>>(c->vec[0].as<float2>(), c->vec[1].as<float2>(), d_set,
                                                             d_draw, den, c->ell.rperm.as<int32_t>(), c->n,
                                                             c->ell.npad, c->nrhs, set0, nrhs_real);
    else
        k_start_from_sets<double><<<grd, blk, 0, c->stream>>>(c->vec[0].as<double2>(), c->vec[1].as<double2>(),
                                                              d_set, d_draw, den, c->ell.rperm.as<int32_t>(), c->n,
                                                              c->ell.npad, c->nrhs, set0, nrhs_real);
    GBN_CK_LAUNCH(c);
    return GBN_OK;
}

// The captured graph of kGraphSteps recursion steps, rebuilt when the launch configuration changes.
// Capturing launches nothing; the launch counter is corrected for the captured kernels.
template <typename Step>
static int ensure_step_graph(gbn_ctx* c, const StepLaunch& L, const StepParams& p, int64_t total, int ublk,
                             int ugrid, Step& launch_step, int32_t k0)
{
    std::vector<unsigned char> key(sizeof(StepParams) + sizeof(StepLaunch) + 4 * sizeof(int64_t));
    StepParams q;
    memcpy(&q, &p, sizeof q);   // bytewise, padding included
    q.x_cur = q.x_prev = nullptr;
    q.v_out = q.u_out = nullptr;   // per step; the buffers they rotate over are in the key below
    const int64_t extra[4] = {total, ublk, ugrid, ((int64_t)c->prec << 32) | (int64_t)c->nrhs};
    memcpy(key.data(), &q, sizeof q);
    memcpy(key.data() + sizeof q, &L, sizeof L);
    memcpy(key.data() + sizeof q + sizeof L, extra, sizeof extra);
    const void* vp[4] = {c->vec[0].p, c->vec[1].p, c->vec[2].p, c->vec[3].p};
    key.insert(key.end(), (const unsigned char*)vp, (const unsigned char*)vp + sizeof vp);
    if (c->step_graph && key == c->step_graph_key) return GBN_OK;
    if (c->step_graph) {
        cudaGraphExecDestroy(c->step_graph);
        c->step_graph = nullptr;
    }
    const int64_t before = c->launches;
    GBN_CK(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int rc = GBN_OK;
    for (int32_t k = k0; k < k0 + kGraphSteps && rc == GBN_OK; ++k) rc = launch_step(k);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    c->launches = before;
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
    const cudaError_t e2 = cudaGraphInstantiate(&c->step_graph, g, 0);
    cudaGraphDestroy(g);
    if (e2 != cudaSuccess) {
        c->step_graph = nullptr;
        return cuda_fail(c, e2, "cudaGraphInstantiate");
    }
    c->step_graph_key = key;
    return GBN_OK;
}

int lanczos_run(gbn_ctx* c, int32_t nmax)
{
    const int R = c->nrhs;
    // the run synchronises at its end (timing, error flags), which a stream capture does not allow
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    GBN_CK(c, cudaStreamIsCapturing(c->stream, &cap));
    if (cap != cudaStreamCaptureStatusNone)
        return fail(c, GBN_ERR_ARG, "the recursion cannot run while its stream is being captured into a graph: "
                                    "it waits for its own kernels to read their timing and error flags");
    GBN_CK(c, c->ab.ensure(sizeof(double) * 2 * (size_t)R * nmax));
    k_init_scalars<<<1, 64, 0, c->stream>>>(c->scal.as<double>(), c->counter.as<unsigned int>(), R);
    GBN_CK_LAUNCH(c);
    StepLaunch L;
    memset(&L, 0, sizeof L);   // the graph key compares these structures bytewise, padding included
    const int rc = step_launch(c, R, &L);
    if (rc) return rc;
    c->last_staged = L.staged;
    // the block partials of this launch shape (it may differ from the one the buffers were sized for)
    GBN_CK(c, c->partials.ensure(sizeof(double) * (size_t)R * (L.fused ? 3 : 1) *
                                 (size_t)std::max(L.grid, c->num_sms * kUpdateBlocksPerSM)));
    if (L.fused)
        GBN_CK(c, c->vec[3].ensure((size_t)c->ell.npad * R * (c->prec == GBN_MIXED ? sizeof(float2) : sizeof(double2))));
    StepParams p;
    memset(&p, 0, sizeof p);
    p.slice_ptr = c->ell.slice_ptr.as<int64_t>();
    p.mat = L.mat;
    p.entry_bytes = L.entry_bytes;
    p.cap_record = L.cap;
    // default: the epilogue rows into L2, and in mixed precision the rows of u_k two sweeps ahead
    p.prefetch = c->tune_prefetch < 0 ? (c->prec == GBN_MIXED ? 6 : 4) : c->tune_prefetch;
    p.h0 = c->ell.h0.p;
    p.v_out = c->vec[0].p;
    p.scal = c->scal.as<double>();
    p.partials = c->partials.as<double>();
    p.counter = c->counter.as<unsigned int>();
    p.a_out = c->ab.as<double>();
    p.b_out = c->ab.as<double>() + (size_t)R * nmax;
    p.nslices = c->ell.nslices;
    p.nmax = nmax;
    p.field_m = c->field_m.as<int32_t>();
    if (L.tiled) {
        p.tile_slice = c->ell.tile_slice.as<int64_t>();
        p.halo_ptr = c->ell.halo_ptr.as<int64_t>();
        p.halo = c->ell.halo.as<int32_t>();
        p.ntiles = c->ell.ntiles;
        p.pitch = L.pitch;
        p.halo_off = L.halo_off;
    }
    const int64_t total = c->ell.npad * R;
    const int ublk = 256;   // a multiple of R (k_update keeps one right-hand side per thread)
    // at least 8 elements per thread, at most kUpdateBlocksPerSM blocks per SM
    const int ugrid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)c->num_sms * kUpdateBlocksPerSM,
                                                                   (total + ublk * 8 - 1) / (ublk * 8)));
    if (!c->ev0) {
        GBN_CK(c, cudaEventCreate(&c->ev0));
        GBN_CK(c, cudaEventCreate(&c->ev1));
    }
    // per-kernel durations of the first steps (three events per sampled step)
    const int nsample = nmax < kTimedSteps ? nmax : kTimedSteps;
    if (!c->kev[0]) {
        for (int i = 0; i < 3 * kTimedSteps; ++i) GBN_CK(c, cudaEventCreate(&c->kev[i]));
    }
    // step k (0-based): x_prev in vec[1 + k%2], x_cur written to vec[1 + (k+1)%2]; the step index of the
    // a_n, b_n outputs lives on the device (counter[1]), so a run of an even number of steps replays as is
    // the update of step k: u_k from v_k and u_{k-1}, and b_{k-1}
    auto launch_update = [&](int32_t k) -> int {
        void* xprev = c->vec[1 + (k & 1)].p;
        void* xcur = c->vec[1 + ((k + 1) & 1)].p;
        double* bo = c->ab.as<double>() + (size_t)R * nmax;
        if (c->prec == GBN_MIXED)
            k_update<float><<<ugrid, ublk, 0, c->stream>>>(c->vec[0].as<float2>(), static_cast<const float2*>(xprev),
                                                          static_cast<float2*>(xcur), c->scal.as<double>(),
                                                          c->partials.as<double>(), c->counter.as<unsigned int>(), bo,
                                                          nmax, total, R);
        else
            k_update<double><<<ugrid, ublk, 0, c->stream>>>(c->vec[0].as<double2>(), static_cast<const double2*>(xprev),
                                                           static_cast<double2*>(xcur), c->scal.as<double>(),
                                                           c->partials.as<double>(), c->counter.as<unsigned int>(), bo,
                                                           nmax, total, R);
        GBN_CK_LAUNCH(c);
        return GBN_OK;
    };
    // step k (0-based): u_{k-1} in vec[1 + k%2], u_k written to vec[1 + (k+1)%2]; the step index of the
    // a_n, b_n outputs lives on the device (counter[1]), so a run of an even number of steps replays as is
    auto launch_step = [&](int32_t k) -> int {
        void* xprev = c->vec[1 + (k & 1)].p;
        void* xcur = c->vec[1 + ((k + 1) & 1)].p;
        if (L.fused) {   // v_k in vec[0] / vec[3] by parity, u_{k-1} in vec[1 + k%2]; u_k, v_{k+1} written
            p.x_cur = (k & 1) ? c->vec[3].p : c->vec[0].p;
            p.v_out = (k & 1) ? c->vec[0].p : c->vec[3].p;
            p.x_prev = xprev;
            p.u_out = xcur;
            if (k < nsample) {
                GBN_CK(c, cudaEventRecord(c->kev[3 * k], c->stream));
                GBN_CK(c, cudaEventRecord(c->kev[3 * k + 1], c->stream));
            }
            L.fn<<<L.grid, L.block, L.smem, c->stream>>>(p);
            GBN_CK_LAUNCH(c);
            if (k < nsample) GBN_CK(c, cudaEventRecord(c->kev[3 * k + 2], c->stream));
            return GBN_OK;
        }
        if (k < nsample) GBN_CK(c, cudaEventRecord(c->kev[3 * k], c->stream));
        const int rcu = launch_update(k);
        if (rcu) return rcu;
        if (k < nsample) GBN_CK(c, cudaEventRecord(c->kev[3 * k + 1], c->stream));
        p.x_cur = xcur;
        p.x_prev = xprev;
        L.fn<<<L.grid, L.block, L.smem, c->stream>>>(p);
        GBN_CK_LAUNCH(c);
        if (k < nsample) GBN_CK(c, cudaEventRecord(c->kev[3 * k + 2], c->stream));
        return GBN_OK;
    };
    c->graph_replays = 0;
    GBN_CK(c, cudaEventRecord(c->ev0, c->stream));
    int32_t k = 0;
    for (; k < nsample; ++k) {
        const int rc2 = launch_step(k);
        if (rc2) return rc2;
    }
    // The remaining steps replay a captured graph of kGraphSteps steps (launch overhead is what limits
    // small cells).
    if (nmax - k >= 2 * kGraphSteps) {
        const int rc2 = ensure_step_graph(c, L, p, total, ublk, ugrid, launch_step, k);
        if (rc2) return rc2;
        for (; nmax - k >= kGraphSteps; k += kGraphSteps) {
            GBN_CK(c, cudaGraphLaunch(c->step_graph, c->stream));
            c->launches += (L.fused ? 1 : 2) * kGraphSteps;
            ++c->graph_replays;
        }
    }
    for (; k < nmax; ++k) {
        const int rc2 = launch_step(k);
        if (rc2) return rc2;
    }
    if (!L.fused) {   // the closing update gives b_{nmax-1} (the fused step's finish already did)
        const int rc2 = launch_update(nmax);
        if (rc2) return rc2;
    }
    GBN_CK(c, cudaEventRecord(c->ev1, c->stream));
    GBN_CK(c, cudaEventSynchronize(c->ev1));
    float ms = 0.f;
    GBN_CK(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->timing.step_ms = ms;
    c->timing.step_launches = nmax;
    double tu = 0.0, ts = 0.0;
    for (int k = 0; k < nsample; ++k) {
        float a = 0.f, b = 0.f;
        GBN_CK(c, cudaEventElapsedTime(&a, c->kev[3 * k], c->kev[3 * k + 1]));
        GBN_CK(c, cudaEventElapsedTime(&b, c->kev[3 * k + 1], c->kev[3 * k + 2]));
        tu += a;
        ts += b;
    }
    c->timing.update_ms_avg = nsample ? tu / nsample : 0.0;
    c->timing.spmm_ms_avg = nsample ? ts / nsample : 0.0;
    unsigned int flags[3];
    GBN_CK(c, cudaMemcpyAsync(flags, c->counter.p, sizeof(flags), cudaMemcpyDeviceToHost, c->stream));
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    if (flags[2] & 2u) return fail(c, GBN_ERR_TIMEOUT, "a staged matrix copy did not complete within its time limit");
    if (flags[2]) return fail(c, GBN_ERR_NUMERIC, "recursion produced a non-positive or non-finite b_n");
    return GBN_OK;
}

}  // namespace gbn
