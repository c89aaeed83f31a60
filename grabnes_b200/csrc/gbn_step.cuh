// The per-step pieces of the recursion's sparse product shared by its kernels (gbn_lanczos.cu: matrix
// records from global or shared memory; gbn_fields.cu: many fields from one field-free matrix): the
// launch parameters, the slice loop body with its FP64 epilogue, and the fixed-order reduction of the
// product's one dot product per right-hand side, which writes a_k.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "gbn_spmm.cuh"

namespace gbn {

// Scalars of the recursion per right-hand side r, scal[4 r + i]:
//   i = 0  a of the last product;  1  norm of the current carried vector u (x = u / norm);
//   2  norm of the previous carried vector;  3  the fused step's alpha (u_k = v_k - alpha u_{k-1}).
constexpr int kScal = 4;

struct StepParams {
    const int64_t* slice_ptr;
    const unsigned char* mat;  // slice records (column indices, then G values per union column)
    int64_t entry_bytes;       // 4 + G * value bytes
    int64_t cap_record;        // bytes of a staging buffer (larger records are read in place)
    int32_t prefetch;          // staged kernel: prefetch the gather rows of a slice (1 L2, 2 L1) or
                               // the rows of its epilogue (3 L1, 4 L2); 5..7: as 4, and the rows of
                               // u_k of the warp's slice 1, 2 or 4 sweeps ahead into L2 in one bulk prefetch
    const void* h0;
    const void* x_cur;   // u_k   [npad][R] (gathered; x_k = u_k / b_{k-1})
    const void* x_prev;  // u_{k-1}        (x_{k-1} = u_{k-1} / b_{k-2})
    void* v_out;         // v_{k+1} = H x_k - b_{k-1} x_{k-1}
    void* u_out;         // fused step: u_k, formed from v_k (x_cur) and u_{k-1} (x_prev) while gathering
    double* scal;        // [R][kScal]
    double* partials;    // [gridDim][R]
    unsigned int* counter;  // [0] block counter, [1] step index, [2] error flag
    double* a_out;       // [R][nmax]
    double* b_out;
    int64_t nslices;
    int32_t nmax;
    const int32_t* field_m;  // field-batched layout: flux quanta of each right-hand side [R] (else unused)
    // tile-local product (k_spmm_tiled): tiles of slices, their halo rows, the halo buffer in shared memory
    const int64_t* tile_slice;  // [ntiles + 1]
    const int64_t* halo_ptr;    // [ntiles + 1]
    const int32_t* halo;        // rows of u_k each tile gathers
    int64_t ntiles;
    int32_t pitch;              // bytes per halo row in shared memory (the row, padded by 16 bytes)
    int32_t halo_off;           // byte offset of the halo buffer in dynamic shared memory
};

using StepFn = void (*)(StepParams);
// the sparse-product kernel of the field-batched layout (gbn_fields.cu): rotations on the fly, or the
// tile table (complex values per thread slot)
StepFn field_step_kernel(int prec, int G, int rpt, int tpr, bool staged);
// the field-batched product with the update folded in (staged, the widest loads per thread), nullptr for
// other shapes
StepFn field_fused_kernel(int prec, int G, int rpt, int tpr, int min_blocks);
StepFn field_table_kernel(int prec, int G, int rpt, int tpr, bool staged);

// Variant of the product kernel: columns in flight per batch (4 or 8) and, for the staged kernel,
// whether the staged records carry the values or only the column indices.  Real-valued layouts at the
// widest loads per thread have every variant; other shapes use unroll 4 with whole records.
struct StepVariant {
    int unroll = 4;
    bool stage_values = true;
    int min_blocks = 1;   // staged, unroll 8: registers bounded for 2 (whole records) or 3 resident blocks per SM
    bool fused = false;   // the update folded into the product (staged, real FP32, 4 right-hand sides per thread)
};
// the product kernel of the real or complex layout (gbn_step_mixed.cu, gbn_step_fp64.cu)
StepFn step_kernel_mixed(bool cplx, int G, int rpt, int tpr, bool staged, StepVariant v);
StepFn step_kernel_fp64(bool cplx, int G, int rpt, int tpr, bool staged, StepVariant v);
// the tile-local product (mixed precision, real values; gbn_step_mixed.cu), nullptr for other shapes
StepFn tiled_kernel_mixed(int G, int rpt, int tpr, int min_blocks);

// Compensated summation (Neumaier's variant of Kahan's) for the block and grid reductions of the dot
// products: the running error term recovers the low-order bits that each addition loses.
struct NeumaierSum {
    double s = 0.0, c = 0.0;
    __device__ __forceinline__ void add(double x)
    {
        const double t = s + x;
        c += (fabs(s) >= fabs(x)) ? (s - t) + x : (x - t) + s;
        s = t;
    }
    __device__ __forceinline__ double value() const { return s + c; }
};

// Compensated pairwise combination of per-thread sums in shared memory, in a fixed order: entry
// j * R + r of (vs, vc) holds the sum and the error term of part j of right-hand side r (j < per); a
// tree of TwoSum steps over j leaves the total of r in vs[r] + vc[r].  Called by every thread of the
// block (it synchronises); per * R <= blockDim.x.
__device__ __forceinline__ void tree_fixed_sum(double* vs, double* vc, int per, int R)
{
    __syncthreads();
    int half = 1;
    while (half < per) half <<= 1;
    for (half >>= 1; half >= 1; half >>= 1) {
        const int j = (int)threadIdx.x / R, r = (int)threadIdx.x % R;
        if (j < half && j + half < per) {
            const int a = j * R + r, b = (j + half) * R + r;
            const double s = vs[a], x = vs[b];
            const double t = s + x;
            const double e = (fabs(s) >= fabs(x)) ? (s - t) + x : (x - t) + s;
            vs[a] = t;
            vc[a] = vc[a] + vc[b] + e;
        }
        __syncthreads();
    }
}

// Fixed-order total of the blocks' partial sums partials[nblk][R], computed by every thread of the calling
// (last) block: thread t takes right-hand side t % R and the blocks t / R, t / R + T / R, ... (T threads,
// a multiple of R), eight loads in flight, with Neumaier's compensation; then the T / R per-thread totals
// of each right-hand side are combined by tree_fixed_sum.  The assignment depends only on nblk, R and T,
// so the result does not depend on scheduling.  vs, vc: T doubles of shared memory each; tot[r] receives
// the totals.
__device__ __forceinline__ void grid_fixed_sum(const double* partials, int nblk, int R, double* vs, double* vc,
                                               double* tot)
{
    const int per = (int)blockDim.x / R;
    const int r = (int)threadIdx.x % R;
    constexpr int D = 8;
    NeumaierSum s;
    int j = (int)threadIdx.x / R;
    for (; j + (D - 1) * per < nblk; j += D * per) {
        double v[D];
#pragma unroll
        for (int i = 0; i < D; ++i) v[i] = __ldcg(partials + (int64_t)(j + i * per) * R + r);
#pragma unroll
        for (int i = 0; i < D; ++i) s.add(v[i]);
    }
    for (; j < nblk; j += per) s.add(__ldcg(partials + (int64_t)j * R + r));
    vs[threadIdx.x] = s.s;
    vc[threadIdx.x] = s.c;
    tree_fixed_sum(vs, vc, per, R);
    if ((int)threadIdx.x < R) tot[threadIdx.x] = vs[threadIdx.x] + vc[threadIdx.x];
    __syncthreads();
}

// Scalars of the step for the block's right-hand sides, in shared memory: 1 / b_{k-1} (x_k = u_k / b_{k-1})
// and b_{k-1} / b_{k-2} (the coefficient of u_{k-1} in v_{k+1}).  Read per epilogue row, so that they
// hold no registers across the column loop.  Needs at least R threads per block.
template <int R, int NSC = 2>
__device__ __forceinline__ void load_step_scalars(const StepParams& p, double (&sc)[NSC][R])
{
    if (threadIdx.x < R) {
        const double nb = p.scal[kScal * threadIdx.x + 1], nbp = p.scal[kScal * threadIdx.x + 2];
        sc[0][threadIdx.x] = 1.0 / nb;
        sc[1][threadIdx.x] = nb / nbp;
        if constexpr (NSC > 2) sc[2][threadIdx.x] = p.scal[kScal * threadIdx.x + 3];   // alpha (fused)
    }
    __syncthreads();
}

// Reduction of the sum Re<u_k, H u_k> over the block, then by the last block over all blocks in a fixed
// order; writes a_k = Re<u_k, H u_k> / b_{k-1}^2 and advances the step index.
// FUSED: three sums per right-hand side, S_a = Re<u_k, H u_k>, S_vv = |v_{k+1}|^2 and S_vu = Re<v_{k+1}, u_k>
// (acc_s[s * RPT + t], block partials in planes [s][block][R]).  With alpha = a_k / b_{k-1} (rounded to FP32
// for FP32 vectors, AL32: the value the next step forms u_{k+1} = v_{k+1} - alpha u_k with), b_k^2 =
// |u_{k+1}|^2 = S_vv - 2 alpha S_vu + alpha^2 b_{k-1}^2; the finish writes a_k and b_k and shifts the norms, as
// the update kernel does otherwise.
template <int RPT, int TPR, bool FUSED = false, bool AL32 = true>
__device__ __forceinline__ void reduce_and_finalize(const StepParams& p, double* acc_s)
{
    constexpr int R = RPT * TPR;
    constexpr int NS = FUSED ? 3 : 1;
    const int lane = threadIdx.x & 31;
    const int sub = lane / TPR;
    const int q = lane % TPR;
#pragma unroll
    for (int t = 0; t < NS * RPT; ++t) {
#pragma unroll
        for (int off = TPR; off < 32; off <<= 1) acc_s[t] += __shfl_xor_sync(0xffffffffu, acc_s[t], off);
    }
    __shared__ double red[NS][8][R];
    const int wib = threadIdx.x >> 5;
    if (sub == 0) {
#pragma unroll
        for (int k = 0; k < NS; ++k)
#pragma unroll
            for (int t = 0; t < RPT; ++t) red[k][wib][q * RPT + t] = acc_s[k * RPT + t];
    }
    __syncthreads();
    if ((int)threadIdx.x < NS * R) {
        const int k = (int)threadIdx.x / R, r = (int)threadIdx.x % R;
        NeumaierSum a;
        for (int wI = 0; wI < (int)(blockDim.x >> 5); ++wI) a.add(red[k][wI][r]);
        p.partials[((int64_t)k * gridDim.x + blockIdx.x) * R + r] = a.value();
    }
    // the last block to finish reduces all blocks in a fixed order
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(p.counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    __shared__ double fin_s[256], fin_c[256], tot[NS][R];
#pragma unroll
    for (int k = 0; k < NS; ++k)
        grid_fixed_sum(p.partials + (int64_t)k * gridDim.x * R, (int)gridDim.x, R, fin_s, fin_c, tot[k]);
    if (threadIdx.x < R) {
        const int r = threadIdx.x;
        const unsigned int step = p.counter[1];
        const double nb = p.scal[kScal * r + 1];
        const double a = tot[0][r] / (nb * nb);
        if (!isfinite(a)) atomicOr(&p.counter[2], 1u);
        if ((int)step < p.nmax) p.a_out[(int64_t)r * p.nmax + step] = a;
        p.scal[kScal * r] = a;
        if constexpr (FUSED) {
            const double al = AL32 ? (double)(float)(a / nb) : a / nb;
            const double b2 = tot[1][r] - 2.0 * al * tot[2][r] + al * al * (nb * nb);
            const double b = sqrt(b2);
            if (!(b > 0.0) || !isfinite(b)) atomicOr(&p.counter[2], 1u);
            if ((int)step < p.nmax) p.b_out[(int64_t)r * p.nmax + step] = b;
            p.scal[kScal * r + 2] = nb;
            p.scal[kScal * r + 1] = b;
            p.scal[kScal * r + 3] = al;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        p.counter[0] = 0u;
        p.counter[1] = p.counter[1] + 1u;
    }
}

// One slice of the grouped sliced ELL: GPW = 32/TPR groups; the TPR threads of a group each hold RPT
// right-hand sides of all G rows of the group.  Per union column a thread reads the column index and
// the G values (same address for the group's threads) and gathers RPT vector elements of that column
// once for all G rows: y = H u_k.  The epilogue per row adds the on-site term and is FP64 from there:
// v_{k+1} = y / b_{k-1} - (b_{k-1} / b_{k-2}) u_{k-1} rounded once, and the term of Re<u_k, y>.  cp/vp
// point at the thread's group in the slice record; the indices come from shared memory (SMEM) or global
// memory (streamed), the values likewise (SMEM_VAL).  U columns are in flight per batch.
// FIELD: field-batched values (FieldVal), the thread's field is that of its first right-hand side.
// FUSED: x_cur holds v_k and x_prev u_{k-1}; the gathers and the own rows use u_k = v_k - alpha u_{k-1} (one
// packed FP32 FMA, the same everywhere), u_k is written to u_out, and the three sums of reduce_and_finalize
// are accumulated (acc_s[3 RPT]).
template <typename VT, bool CPLX, int G, int RPT, int TPR, bool SMEM, bool FIELD, int U, bool SMEM_VAL, int VS = 1,
          bool FUSED = false, int NSC = 2>
__device__ __forceinline__ void group_slice(const StepParams& p, int64_t s, int w, const int32_t* __restrict__ cp,
                                            const typename StoredVal<VT, CPLX, FIELD>::t* __restrict__ vp,
                                            const double (&sc)[NSC][RPT * TPR], double* acc_s)
{
    if constexpr (FUSED) {
        using C2 = typename V2<VT>::t;
        constexpr int GPW = 32 / TPR;
        constexpr int R = RPT * TPR;
        const int lane = threadIdx.x & 31;
        const int sub = lane / TPR;
        const int q = lane % TPR;
        const C2* __restrict__ xv = static_cast<const C2*>(p.x_cur);
        const C2* __restrict__ xp = static_cast<const C2*>(p.x_prev);
        C2* __restrict__ vout = static_cast<C2*>(p.v_out);
        C2* __restrict__ uout = static_cast<C2*>(p.u_out);
        const VT* __restrict__ h0 = static_cast<const VT*>(p.h0);
        const int64_t row0 = (s * GPW + sub) * G;
        C2 al[RPT];
#pragma unroll
        for (int t = 0; t < RPT; ++t) {
            const VT a = (VT)(-sc[NSC - 1][q * RPT + t]);
            al[t].x = a;
            al[t].y = a;
        }
        C2 acc[G][RPT];
        typename FieldMult<VT>::t mf = 0;
        if constexpr (FIELD) mf = (typename FieldMult<VT>::t)(int64_t)p.field_m[q * RPT];
        group_columns<VT, CPLX, G, RPT, TPR, SMEM, FIELD, U, SMEM_VAL, VS, true>(xv, w, cp, vp, acc, mf, xp, al);
#pragma unroll
        for (int g = 0; g < G; ++g) {
            C2 xo[RPT], xm[RPT], vn[RPT];
            VecIO<VT, RPT>::load(xv + (row0 + g) * R + q * RPT, xo);
            VecIO<VT, RPT>::load(xp + (row0 + g) * R + q * RPT, xm);
            const VT d = h0[row0 + g];
#pragma unroll
            for (int t = 0; t < RPT; ++t) {
                xo[t] = fused_form(al[t], xm[t], xo[t]);   // u_k, as the gathers form it
                acc[g][t].x = fma(d, xo[t].x, acc[g][t].x);
                acc[g][t].y = fma(d, xo[t].y, acc[g][t].y);
                const double ib = sc[0][q * RPT + t], rb = sc[1][q * RPT + t];
                const double yr = acc[g][t].x, yi = acc[g][t].y;
                vn[t].x = (VT)(yr * ib - rb * (double)xm[t].x);
                vn[t].y = (VT)(yi * ib - rb * (double)xm[t].y);
                const double ur = xo[t].x, ui = xo[t].y, vr = vn[t].x, vi = vn[t].y;
                acc_s[t] += ur * yr + ui * yi;
                acc_s[RPT + t] += vr * vr + vi * vi;
                acc_s[2 * RPT + t] += vr * ur + vi * ui;
            }
            VecIO<VT, RPT>::store(vout + (row0 + g) * R + q * RPT, vn);
            VecIO<VT, RPT>::store(uout + (row0 + g) * R + q * RPT, xo);
        }
        return;
    }
    using C2 = typename V2<VT>::t;
    constexpr int GPW = 32 / TPR;
    constexpr int R = RPT * TPR;
    const int lane = threadIdx.x & 31;
    const int sub = lane / TPR;
    const int q = lane % TPR;
    const C2* __restrict__ xc = static_cast<const C2*>(p.x_cur);
    const C2* __restrict__ xp = static_cast<const C2*>(p.x_prev);
    C2* __restrict__ vout = static_cast<C2*>(p.v_out);
    const VT* __restrict__ h0 = static_cast<const VT*>(p.h0);
    const int64_t row0 = (s * GPW + sub) * G;
    C2 acc[G][RPT];
    typename FieldMult<VT>::t mf = 0;
    if constexpr (FIELD) mf = (typename FieldMult<VT>::t)(int64_t)p.field_m[q * RPT];
    group_columns<VT, CPLX, G, RPT, TPR, SMEM, FIELD, U, SMEM_VAL, VS>(xc, w, cp, vp, acc, mf);
    // epilogue per row: the on-site term (own u_k row, loaded here so that it holds no registers during
    // the column loop), then v_{k+1} and the dot-product term in FP64
#pragma unroll
    for (int g = 0; g < G; ++g) {
        C2 xo[RPT], xm[RPT], vn[RPT];
        VecIO<VT, RPT>::load(xc + (row0 + g) * R + q * RPT, xo);
        VecIO<VT, RPT>::load(xp + (row0 + g) * R + q * RPT, xm);
        const VT d = h0[row0 + g];
#pragma unroll
        for (int t = 0; t < RPT; ++t) {
            acc[g][t].x = fma(d, xo[t].x, acc[g][t].x);
            acc[g][t].y = fma(d, xo[t].y, acc[g][t].y);
            const double ib = sc[0][q * RPT + t], rb = sc[1][q * RPT + t];
            const double yr = acc[g][t].x, yi = acc[g][t].y;
            vn[t].x = (VT)(yr * ib - rb * (double)xm[t].x);
            vn[t].y = (VT)(yi * ib - rb * (double)xm[t].y);
            acc_s[t] += (double)xo[t].x * yr + (double)xo[t].y * yi;
        }
        VecIO<VT, RPT>::store(vout + (row0 + g) * R + q * RPT, vn);
    }
}

// Matrix records read from global memory.  Every block owns a contiguous range of slices (a compact
// region of the row order); its warps take neighbouring slices, so the rows they gather overlap in L1.
// FIELD: the field-batched layout (values FieldVal<VT>, fields p.field_m).
// SLOT: the field-batched tile table (complex values, one block per thread slot; thread q reads block q).
template <typename VT, bool CPLX, int G, int RPT, int TPR, bool FIELD = false, int U = kColUnroll, bool SLOT = false>
__global__ void __launch_bounds__(256) k_spmm_step(StepParams p)
{
    using HT = typename StoredVal<VT, CPLX, FIELD>::t;
    constexpr int GPW = 32 / TPR;
    constexpr int R = RPT * TPR;
    const int sub = (threadIdx.x & 31) / TPR;
    const int q = (threadIdx.x & 31) % TPR;
    __shared__ double sc[2][R];
    load_step_scalars<R>(p, sc);
    double acc_s[RPT];
#pragma unroll
    for (int t = 0; t < RPT; ++t) acc_s[t] = 0.0;
    const int nwb = (int)(blockDim.x >> 5);
    const int64_t per = (p.nslices + gridDim.x - 1) / gridDim.x;
    const int64_t s0 = (int64_t)blockIdx.x * per;
    const int64_t s1e = (s0 + per < p.nslices) ? s0 + per : p.nslices;
    for (int64_t s = s0 + (threadIdx.x >> 5); s < s1e; s += nwb) {
        const int64_t base = p.slice_ptr[s];
        const int w = (int)((p.slice_ptr[s + 1] - base) / GPW);
        const unsigned char* rec = p.mat + base * p.entry_bytes;
        constexpr int VS = SLOT ? TPR : 1;   // tile table: [column][group][slot][G]
        const int voff = val_thread_off<HT, G, TPR, VS>(sub, q);
        group_slice<VT, CPLX, G, RPT, TPR, false, FIELD, U, false, VS>(
            p, s, w, reinterpret_cast<const int32_t*>(rec) + sub * kColUnroll,
            reinterpret_cast<const HT*>(rec + (size_t)w * GPW * 4) + voff, sc, acc_s);
    }
    reduce_and_finalize<RPT, TPR>(p, acc_s);
}

// ---- bulk asynchronous copies (cp.async.bulk, the TMA engine) into shared memory, mbarrier completion
__device__ __forceinline__ uint32_t smem_u32(const void* ptr) { return (uint32_t)__cvta_generic_to_shared(ptr); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    uint64_t state;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 %0, [%1], %2;"
                 : "=l"(state) : "r"(smem_u32(bar)), "r"(bytes) : "memory");
    (void)state;
}

// global -> shared copy of `bytes` (multiple of 16, both addresses 16-byte aligned), no multicast
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return done != 0;
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// bounded wait: gives up after about one second (the caller records the failure)
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > 1000000000ull) return false;
    return true;
}

// Prefetch of the vector rows that the columns of a staged record will gather (x_k rows of R
// complex values, 128-byte lines), spread over the warp's lanes.  Prefetches do not block and hold
// no registers.
template <typename VT, int R>
__device__ __forceinline__ void prefetch_rows(const StepParams& p, const int32_t* cols, int ncols)
{
    constexpr int ROWB = R * (int)sizeof(typename V2<VT>::t);
    const char* x = static_cast<const char*>(p.x_cur);
    const int lane = threadIdx.x & 31;
    for (int i = lane; i < ncols; i += 32) {
        const char* a = x + (size_t)(uint32_t)cols[i] * ROWB;
#pragma unroll
        for (int off = 0; off < ROWB; off += 128) {
            if (p.prefetch == 2) asm volatile("prefetch.global.L1 [%0];" ::"l"(a + off));
            else asm volatile("prefetch.global.L2 [%0];" ::"l"(a + off));
        }
    }
}

// Prefetch of the rows a slice's epilogue reads (its own rows of x_k and x_{k-1}, contiguous in the
// row order, and their on-site values), issued before the column loop so that the epilogue's loads
// find them in L1 (mode 3) or L2 (mode 4) instead of waiting a DRAM round trip.
template <typename VT, int R, int G, int GPW>
__device__ __forceinline__ void prefetch_epilogue(const StepParams& p, int64_t s)
{
    constexpr int BLK = GPW * G * R * (int)sizeof(typename V2<VT>::t);   // bytes of one slice's rows
    const int lane = threadIdx.x & 31;
    const size_t off = (size_t)s * BLK;
    const char* a = static_cast<const char*>(p.x_prev) + off;
    const char* b = static_cast<const char*>(p.x_cur) + off;
    for (int i = lane * 128; i < BLK; i += 32 * 128) {
        if (p.prefetch == 3) {
            asm volatile("prefetch.global.L1 [%0];" ::"l"(a + i));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(b + i));
        } else {
            asm volatile("prefetch.global.L2 [%0];" ::"l"(a + i));
            asm volatile("prefetch.global.L2 [%0];" ::"l"(b + i));
        }
    }
    if (lane == 31) {
        const char* h = static_cast<const char*>(p.h0) + (size_t)s * GPW * G * sizeof(VT);
        asm volatile("prefetch.global.L1 [%0];" ::"l"(h));
    }
}

// Bulk prefetch of `bytes` contiguous bytes into L2 (one instruction; address and size multiples of 16).
__device__ __forceinline__ void bulk_prefetch_l2(const void* a, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(bytes) : "memory");
}

// The rows of u_k that slice s owns (contiguous in the row order; most of its neighbours' gathers of
// them come later in the block's sweep), prefetched into L2 by lane 0 of the warp.  s < nslices, so the
// range lies inside the vector (nslices * GPW * G <= npad rows).
template <typename VT, int R, int G, int GPW>
__device__ __forceinline__ void prefetch_ahead(const StepParams& p, int64_t s)
{
    constexpr int BLK = GPW * G * R * (int)sizeof(typename V2<VT>::t);   // multiple of 16 (R * 8 * GPW * G)
    if ((threadIdx.x & 31) == 0 && s < p.nslices)
        bulk_prefetch_l2(static_cast<const char*>(p.x_cur) + (size_t)s * BLK, (uint32_t)BLK);
}

// Matrix records staged in shared memory.  Each warp owns two record buffers and an mbarrier per
// buffer; its lane 0 copies the record of the warp's next-but-one slice with one bulk copy while the
// warp works on the current one, so the column indices that the gathers depend on come from shared
// memory instead of a DRAM round trip per unrolled column batch.  SV: the whole record (indices and
// values) is staged; otherwise only its column indices, and the values stream from global memory beside
// the gathers (their loads do not gate any address), which leaves more of the SM's memory to L1.
// Optionally the warp first prefetches all the vector rows a slice will gather.  Records larger than a
// buffer (the largest 0.5 %) are read in place.  No block-wide synchronisation in the loop; every wait
// is bounded (flag bit 2, GBN_ERR_TIMEOUT).
// FIELD: the field-batched layout (values FieldVal<VT>, fields p.field_m).
template <typename VT, bool CPLX, int G, int RPT, int TPR, bool FIELD = false, int U = kColUnroll, bool SV = true,
          int MINB = 1, bool SLOT = false, bool FUSED = false>
__global__ void __launch_bounds__(256, MINB) k_spmm_staged(StepParams p)
{
    using HT = typename StoredVal<VT, CPLX, FIELD>::t;
    constexpr int GPW = 32 / TPR;
    constexpr int R = RPT * TPR;
    extern __shared__ __align__(128) unsigned char dyn[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int sub = lane / TPR;
    const int q = lane % TPR;
    uint64_t* bar = reinterpret_cast<uint64_t*>(dyn) + 2 * wib;
    const int64_t cap = p.cap_record;   // bytes of one buffer: whole records (SV) or their index part
    unsigned char* buf = dyn + 128 + (size_t)wib * 2 * cap;
    constexpr int NSC = FUSED ? 3 : 2;
    constexpr int NS = FUSED ? 3 : 1;
    __shared__ double sc[NSC][R];
    load_step_scalars<R, NSC>(p, sc);
    double acc_s[NS * RPT];
#pragma unroll
    for (int t = 0; t < NS * RPT; ++t) acc_s[t] = 0.0;
    const int nwb = (int)(blockDim.x >> 5);
    const int64_t per = (p.nslices + gridDim.x - 1) / gridDim.x;
    const int64_t s0 = (int64_t)blockIdx.x * per;
    const int64_t s1e = (s0 + per < p.nslices) ? s0 + per : p.nslices;
    const int64_t eb = p.entry_bytes;

    // bytes copied for slice s: the record, or its column indices (the first 4 w GPW bytes)
    auto copy_bytes = [&](int64_t s) { return (p.slice_ptr[s + 1] - p.slice_ptr[s]) * (SV ? eb : 4); };
    // lane 0 only.  Records above the cap are not copied but prefetched into L2 whole, and so is the
    // value part of a record whose indices alone are staged, so that the loads read in place hit L2.
    auto issue = [&](int64_t s, int st) {
        const int64_t nent = p.slice_ptr[s + 1] - p.slice_ptr[s];
        const int64_t bytes = nent * (SV ? eb : 4);
        const unsigned char* src = p.mat + p.slice_ptr[s] * eb;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        const bool copy = bytes > 0 && bytes <= cap;
        mbar_expect_tx(&bar[st], copy ? (uint32_t)bytes : 0u);
        if (copy) bulk_g2s(buf + st * cap, src, (uint32_t)bytes, &bar[st]);
        if (nent > 0 && !copy) bulk_prefetch_l2(src, (uint32_t)(nent * eb));
        else if (nent > 0 && !SV) bulk_prefetch_l2(src + nent * 4, (uint32_t)(nent * (eb - 4)));
    };

    if (lane == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    int64_t s = s0 + wib;
    uint32_t pending = (s < s1e ? 1u : 0u) | (s + nwb < s1e ? 2u : 0u);   // bit st: a copy into buffer st
    if (lane == 0) {
        if (pending & 1u) issue(s, 0);
        if (pending & 2u) issue(s + nwb, 1);
    }
    uint32_t phase = 0u;   // bit st: parity of buffer st's next phase
    bool ok = true;
    for (int it = 0; s < s1e; s += nwb, ++it) {
        const int st = it & 1;
        // the record of this slice (copied while the previous one was processed)
        const bool got = mbar_wait_bounded(&bar[st], (phase >> st) & 1u);
        if (!__all_sync(0xffffffffu, got)) {   // uniform exit of the warp if a copy never completed
            ok = false;
            break;
        }
        phase ^= 1u << st;
        pending &= ~(1u << st);
        const int64_t base = p.slice_ptr[s];
        const int w = (int)((p.slice_ptr[s + 1] - base) / GPW);
        const unsigned char* grec = p.mat + base * eb;
        if (p.prefetch >= 3) prefetch_epilogue<VT, R, G, GPW>(p, s);
        if (p.prefetch >= 5) prefetch_ahead<VT, R, G, GPW>(p, s + (int64_t)(p.prefetch == 5 ? 1 : p.prefetch == 6 ? 2 : 4) * nwb);
        constexpr int VS = SLOT ? TPR : 1;   // tile table: [column][group][slot][G], the thread's own slot
        const int voff = val_thread_off<HT, G, TPR, VS>(sub, q);
        if (copy_bytes(s) <= cap) {
            const unsigned char* rec = buf + st * cap;
            if (p.prefetch == 1 || p.prefetch == 2)
                prefetch_rows<VT, R>(p, reinterpret_cast<const int32_t*>(rec), w * GPW);
            const HT* vp = reinterpret_cast<const HT*>((SV ? rec : grec) + (size_t)w * GPW * 4) + voff;
            group_slice<VT, CPLX, G, RPT, TPR, true, FIELD, U, SV, VS, FUSED, NSC>(
                p, s, w, reinterpret_cast<const int32_t*>(rec) + sub * kColUnroll, vp, sc, acc_s);
        } else {
            group_slice<VT, CPLX, G, RPT, TPR, false, FIELD, U, false, VS, FUSED, NSC>(
                p, s, w, reinterpret_cast<const int32_t*>(grec) + sub * kColUnroll,
                reinterpret_cast<const HT*>(grec + (size_t)w * GPW * 4) + voff, sc, acc_s);
        }
        __syncwarp();   // every lane is done with this buffer before it is refilled
        if (s + 2 * nwb < s1e) {
            pending |= 1u << st;
            if (lane == 0) issue(s + 2 * nwb, st);
        }
    }
    if (!ok) {
        if (lane == 0) atomicOr(&p.counter[2], 2u);
        // let copies still in flight land before the block's shared memory is released
        for (int st = 0; st < 2; ++st)
            if ((pending >> st) & 1u) mbar_wait_bounded(&bar[st], (phase >> st) & 1u);
        __syncwarp();
    }
    reduce_and_finalize<RPT, TPR, FUSED, sizeof(VT) == 4>(p, acc_s);
}

// ---------------------------------------------------------------------------- tile-local product
// A vector row (RPT right-hand sides of one thread) from the halo buffer in shared memory.
template <typename VT, int RPT> struct SmemRow;
template <> struct SmemRow<float, 4> {
    static __device__ __forceinline__ void load(const unsigned char* p, float2 o[4]) {
        const float4 a = *reinterpret_cast<const float4*>(p), b = *reinterpret_cast<const float4*>(p + 16);
        o[0] = make_float2(a.x, a.y); o[1] = make_float2(a.z, a.w); o[2] = make_float2(b.x, b.y); o[3] = make_float2(b.z, b.w);
    }
};
template <> struct SmemRow<float, 2> {
    static __device__ __forceinline__ void load(const unsigned char* p, float2 o[2]) {
        const float4 a = *reinterpret_cast<const float4*>(p);
        o[0] = make_float2(a.x, a.y); o[1] = make_float2(a.z, a.w);
    }
};
template <> struct SmemRow<float, 1> {
    static __device__ __forceinline__ void load(const unsigned char* p, float2 o[1]) { o[0] = *reinterpret_cast<const float2*>(p); }
};

// One batch of NB union columns of the tile-local product: the indices (tile-local) and values from the
// staged record (SMEM) or the record in global memory, the rows from the halo buffer.
template <typename VT, int G, int RPT, int TPR, bool SMEM, int NB>
__device__ __forceinline__ void tile_batch(const unsigned char* __restrict__ xs, int pitch,
                                           const int32_t* __restrict__ cp, const VT* __restrict__ vp,
                                           typename V2<VT>::t (&acc)[G][RPT])
{
    using C2 = typename V2<VT>::t;
    constexpr int GPW = 32 / TPR;
    int32_t c[NB];
    VT h[NB][G];
    C2 xg[NB][RPT];
    load_block_cols<GPW, NB, SMEM>(cp, c);
#pragma unroll
    for (int u = 0; u < NB; ++u) SmemRow<VT, RPT>::load(xs + (size_t)(uint32_t)c[u] * pitch, xg[u]);
    load_block_vals<VT, G, GPW, NB, SMEM, 1>(vp, h);
#pragma unroll
    for (int u = 0; u < NB; ++u)
#pragma unroll
        for (int g = 0; g < G; ++g)
#pragma unroll
            for (int t = 0; t < RPT; ++t) Hop<VT, false>::madd(acc[g][t], h[u][g], xg[u][t]);
}

// One slice of the tile-local product: the union-column loop over the halo buffer, then the same FP64
// epilogue as group_slice (own rows of u_k and u_{k-1} from global memory).
template <typename VT, int G, int RPT, int TPR, bool SMEM, int U>
__device__ __forceinline__ void tile_slice_step(const StepParams& p, int64_t s, int w, const unsigned char* xbuf,
                                           const int32_t* __restrict__ cp, const VT* __restrict__ vp,
                                           const double (&sc)[2][RPT * TPR], double* acc_s)
{
    using C2 = typename V2<VT>::t;
    constexpr int GPW = 32 / TPR;
    constexpr int R = RPT * TPR;
    const int lane = threadIdx.x & 31;
    const int sub = lane / TPR;
    const int q = lane % TPR;
    const C2* __restrict__ xc = static_cast<const C2*>(p.x_cur);
    const C2* __restrict__ xp = static_cast<const C2*>(p.x_prev);
    C2* __restrict__ vout = static_cast<C2*>(p.v_out);
    const VT* __restrict__ h0 = static_cast<const VT*>(p.h0);
    const int64_t row0 = (s * GPW + sub) * G;
    const unsigned char* xs = xbuf + q * RPT * (int)sizeof(C2);
    C2 acc[G][RPT];
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
        for (int t = 0; t < RPT; ++t) { acc[g][t].x = 0; acc[g][t].y = 0; }
    int k = 0;
    for (; k + U <= w; k += U) {
        tile_batch<VT, G, RPT, TPR, SMEM, U>(xs, p.pitch, cp, vp, acc);
        cp += U * GPW;
        vp += U * GPW * G;
    }
    if constexpr (U > kColUnroll) {
        for (; k < w; k += kColUnroll) {
            tile_batch<VT, G, RPT, TPR, SMEM, kColUnroll>(xs, p.pitch, cp, vp, acc);
            cp += kColUnroll * GPW;
            vp += kColUnroll * GPW * G;
        }
    }
#pragma unroll
    for (int g = 0; g < G; ++g) {
        C2 xo[RPT], xm[RPT], vn[RPT];
        VecIO<VT, RPT>::load(xc + (row0 + g) * R + q * RPT, xo);
        VecIO<VT, RPT>::load(xp + (row0 + g) * R + q * RPT, xm);
        const VT d = h0[row0 + g];
#pragma unroll
        for (int t = 0; t < RPT; ++t) {
            acc[g][t].x = fma(d, xo[t].x, acc[g][t].x);
            acc[g][t].y = fma(d, xo[t].y, acc[g][t].y);
            const double ib = sc[0][q * RPT + t], rb = sc[1][q * RPT + t];
            const double yr = acc[g][t].x, yi = acc[g][t].y;
            vn[t].x = (VT)(yr * ib - rb * (double)xm[t].x);
            vn[t].y = (VT)(yi * ib - rb * (double)xm[t].y);
            acc_s[t] += (double)xo[t].x * yr + (double)xo[t].y * yi;
        }
        VecIO<VT, RPT>::store(vout + (row0 + g) * R + q * RPT, vn);
    }
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

// The tile-local product.  Every block owns a contiguous range of tiles.  Per tile: the warps' first two
// slice records are copied into their staging buffers (bulk copies, as in k_spmm_staged), the block copies
// the tile's halo rows of u_k into shared memory (cp.async, 16 bytes per thread and request, rows padded
// to `pitch` so that the rows of one gather batch spread over the banks), and the warps then run the
// tile's slices with every gather read from shared memory: a gather batch waits a shared-memory latency
// instead of the slowest of its rows' L1 misses.  Waits are bounded as in k_spmm_staged; a warp that gives
// up marks the block, which stops at the next tile boundary (every thread still reaches every barrier).
// Measured slower than k_spmm_staged on both bench cells (4.47M-atom twisted bilayer: 1.60 against 1.19 ms;
// 3.5M-atom graphene/hBN: 0.58 against 0.30 ms): a halo that fits beside the staging buffers holds tiles
// of a few hundred rows, so each warp runs two or three slices between the block's barriers and the fill
// of every tile stalls the block.  It is an opt-in variant (gbn_set_kernel_variant), not a default.
template <typename VT, int G, int RPT, int TPR, int U, int MINB>
__global__ void __launch_bounds__(256, MINB) k_spmm_tiled(StepParams p)
{
    using C2 = typename V2<VT>::t;
    constexpr int GPW = 32 / TPR;
    constexpr int R = RPT * TPR;
    constexpr int ROWB = R * (int)sizeof(C2);
    constexpr int CH = ROWB / 16;
    static_assert(ROWB % 16 == 0, "halo rows are copied in 16-byte pieces");
    extern __shared__ __align__(128) unsigned char dyn[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int sub = lane / TPR;
    uint64_t* bar = reinterpret_cast<uint64_t*>(dyn) + 2 * wib;
    const int64_t cap = p.cap_record;
    unsigned char* buf = dyn + 128 + (size_t)wib * 2 * cap;
    unsigned char* xbuf = dyn + p.halo_off;
    __shared__ double sc[2][R];
    __shared__ int bad;
    if (threadIdx.x == 0) bad = 0;
    load_step_scalars<R>(p, sc);   // synchronises the block
    double acc_s[RPT];
#pragma unroll
    for (int t = 0; t < RPT; ++t) acc_s[t] = 0.0;
    const int nwb = (int)(blockDim.x >> 5);
    const int64_t per = (p.ntiles + gridDim.x - 1) / gridDim.x;
    const int64_t t0 = (int64_t)blockIdx.x * per;
    const int64_t t1 = (t0 + per < p.ntiles) ? t0 + per : p.ntiles;
    const int64_t eb = p.entry_bytes;
    const unsigned char* x = static_cast<const unsigned char*>(p.x_cur);

    auto copy_bytes = [&](int64_t s) { return (p.slice_ptr[s + 1] - p.slice_ptr[s]) * eb; };
    auto issue = [&](int64_t s, int st) {   // lane 0 only; records above the cap are read in place
        const int64_t bytes = copy_bytes(s);
        const unsigned char* src = p.mat + p.slice_ptr[s] * eb;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        const bool copy = bytes > 0 && bytes <= cap;
        mbar_expect_tx(&bar[st], copy ? (uint32_t)bytes : 0u);
        if (copy) bulk_g2s(buf + st * cap, src, (uint32_t)bytes, &bar[st]);
        else if (bytes > 0) bulk_prefetch_l2(src, (uint32_t)bytes);
    };
    if (lane == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    uint32_t phase = 0u, pending = 0u;
    for (int64_t t = t0; t < t1; ++t) {
        const int64_t sb = p.tile_slice[t], se = p.tile_slice[t + 1];
        int64_t s = sb + wib;
        if (!bad) {
            pending = (s < se ? 1u : 0u) | (s + nwb < se ? 2u : 0u);
            if (lane == 0) {
                if (pending & 1u) issue(s, 0);
                if (pending & 2u) issue(s + nwb, 1);
            }
        }
        // the tile's halo rows into shared memory
        const int64_t hb = p.halo_ptr[t];
        const int hn = (int)(p.halo_ptr[t + 1] - hb);
        for (int i = threadIdx.x; i < hn * CH; i += blockDim.x) {
            const int r = i / CH, ch = i - r * CH;
            cp_async16(xbuf + (size_t)r * p.pitch + ch * 16, x + (size_t)(uint32_t)p.halo[hb + r] * ROWB + ch * 16);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncthreads();
        for (int it = 0; s < se && !bad; s += nwb, ++it) {
            const int st = it & 1;
            const bool got = mbar_wait_bounded(&bar[st], (phase >> st) & 1u);
            if (!__all_sync(0xffffffffu, got)) {
                if (lane == 0) atomicOr(&bad, 1);
                break;
            }
            phase ^= 1u << st;
            pending &= ~(1u << st);
            const int64_t base = p.slice_ptr[s];
            const int w = (int)((p.slice_ptr[s + 1] - base) / GPW);
            if (p.prefetch >= 3) prefetch_epilogue<VT, R, G, GPW>(p, s);
            if (copy_bytes(s) <= cap) {
                const unsigned char* rec = buf + st * cap;
                tile_slice_step<VT, G, RPT, TPR, true, U>(p, s, w, xbuf,
                                                     reinterpret_cast<const int32_t*>(rec) + sub * kColUnroll,
                                                     reinterpret_cast<const VT*>(rec + (size_t)w * GPW * 4) + val_thread_off<VT, G, TPR, 1>(sub, 0),
                                                     sc, acc_s);
            } else {
                const unsigned char* rec = p.mat + base * eb;
                tile_slice_step<VT, G, RPT, TPR, false, U>(p, s, w, xbuf,
                                                      reinterpret_cast<const int32_t*>(rec) + sub * kColUnroll,
                                                      reinterpret_cast<const VT*>(rec + (size_t)w * GPW * 4) + val_thread_off<VT, G, TPR, 1>(sub, 0),
                                                      sc, acc_s);
            }
            __syncwarp();   // every lane is done with this buffer before it is refilled
            if (s + 2 * nwb < se) {
                pending |= 1u << st;
                if (lane == 0) issue(s + 2 * nwb, st);
            }
        }
        __syncthreads();   // the halo buffer is reused by the next tile
        if (bad) break;
    }
    if (bad) {
        if (lane == 0) atomicOr(&p.counter[2], 2u);
        for (int st = 0; st < 2; ++st)   // let copies still in flight land before shared memory is released
            if ((pending >> st) & 1u) mbar_wait_bounded(&bar[st], (phase >> st) & 1u);
        __syncwarp();
    }
    reduce_and_finalize<RPT, TPR>(p, acc_s);
}

template <typename VT, int G>
StepFn tiled_pick_g(int rpt, int tpr, int min_blocks)
{
    if constexpr (sizeof(VT) == 4) {
        if (rpt == 4 && tpr == 4) return min_blocks == 2 ? k_spmm_tiled<VT, G, 4, 4, 8, 2> : k_spmm_tiled<VT, G, 4, 4, 8, 1>;
        if (rpt == 4 && tpr == 2) return min_blocks == 2 ? k_spmm_tiled<VT, G, 4, 2, 8, 2> : k_spmm_tiled<VT, G, 4, 2, 8, 1>;
        if (rpt == 4 && tpr == 8) return min_blocks == 2 ? k_spmm_tiled<VT, G, 4, 8, 8, 2> : k_spmm_tiled<VT, G, 4, 8, 8, 1>;
    }
    return nullptr;
}

// ---------------------------------------------------------------------------- kernel selection
template <typename VT, bool CPLX, int G, int RP, int TP>
StepFn step_variant(bool staged, StepVariant v)
{
    constexpr int kWide = sizeof(VT) == 4 ? 4 : 2;   // right-hand sides of a 32-byte load
    constexpr bool kAll = !CPLX && (RP == kWide || TP == 1);
    if (v.fused) {   // staged, real values, the widest loads (or one vector), whole records; FP32 unroll 8, FP64 4
        if constexpr (!CPLX && ((RP == kWide && TP >= 2) || (RP == 1 && TP == 1)) && (sizeof(VT) == 4 || G <= 2)) {
            constexpr int UF = (sizeof(VT) == 4 || RP == 1) ? 8 : 4;   // one FP64 vector: 8 columns too
            if (!staged || v.unroll != UF || !v.stage_values) return nullptr;
            if (v.min_blocks == 2) return k_spmm_staged<VT, CPLX, G, RP, TP, false, UF, true, 2, false, true>;
            if (v.min_blocks == 1) return k_spmm_staged<VT, CPLX, G, RP, TP, false, UF, true, 1, false, true>;
        }
        return nullptr;
    }
    if constexpr (kAll) {
        if (!staged) {
            if (v.min_blocks != 1) return nullptr;
            return v.unroll == 8 ? k_spmm_step<VT, CPLX, G, RP, TP, false, 8> : k_spmm_step<VT, CPLX, G, RP, TP>;
        }
        if (v.unroll == 8 && v.min_blocks == 3)
            return v.stage_values ? k_spmm_staged<VT, CPLX, G, RP, TP, false, 8, true, 3>
                                  : k_spmm_staged<VT, CPLX, G, RP, TP, false, 8, false, 3>;
        if (v.unroll == 8 && v.min_blocks == 2 && v.stage_values) return k_spmm_staged<VT, CPLX, G, RP, TP, false, 8, true, 2>;
        if (v.min_blocks != 1) return nullptr;
        if (v.unroll == 8)
            return v.stage_values ? k_spmm_staged<VT, CPLX, G, RP, TP, false, 8, true>
                                  : k_spmm_staged<VT, CPLX, G, RP, TP, false, 8, false>;
        return v.stage_values ? k_spmm_staged<VT, CPLX, G, RP, TP, false, 4, true>
                              : k_spmm_staged<VT, CPLX, G, RP, TP, false, 4, false>;
    } else {
        if (v.unroll != 4 || !v.stage_values || v.min_blocks != 1) return nullptr;
        return staged ? k_spmm_staged<VT, CPLX, G, RP, TP> : k_spmm_step<VT, CPLX, G, RP, TP>;
    }
}

template <typename VT, bool CPLX, int G>
StepFn step_pick_g(int rpt, int tpr, bool staged, StepVariant v)
{
#define GBN_CASE(RP, TP) \
    if (rpt == RP && tpr == TP) return step_variant<VT, CPLX, G, RP, TP>(staged, v);
    GBN_CASE(1, 1) GBN_CASE(1, 2) GBN_CASE(1, 4) GBN_CASE(1, 8) GBN_CASE(1, 16) GBN_CASE(1, 32)
    GBN_CASE(2, 1) GBN_CASE(2, 2) GBN_CASE(2, 4) GBN_CASE(2, 8) GBN_CASE(2, 16)
    if constexpr (sizeof(VT) == 4) {
        GBN_CASE(4, 1) GBN_CASE(4, 2) GBN_CASE(4, 4) GBN_CASE(4, 8)
    }
#undef GBN_CASE
    return nullptr;
}

template <typename VT, bool CPLX>
StepFn step_pick(int G, int rpt, int tpr, bool staged, StepVariant v)
{
    if (G == 1) return step_pick_g<VT, CPLX, 1>(rpt, tpr, staged, v);
    if (G == 2) return step_pick_g<VT, CPLX, 2>(rpt, tpr, staged, v);
    if (G == 4) return step_pick_g<VT, CPLX, 4>(rpt, tpr, staged, v);
    return nullptr;
}

}  // namespace gbn
