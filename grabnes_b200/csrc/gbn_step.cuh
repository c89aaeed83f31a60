// The per-step pieces of the recursion's sparse product shared by its kernels (gbn_lanczos.cu: matrix
// records from global or shared memory; gbn_fields.cu: many fields from one field-free matrix): the
// launch parameters, the slice loop body with its FP64 epilogue, and the fixed-order reduction of the
// four dot products that writes a_k, b_k.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "gbn_spmm.cuh"

namespace gbn {

struct StepParams {
    const int64_t* slice_ptr;
    const unsigned char* mat;  // slice records (column indices, then G values per union column)
    int64_t entry_bytes;       // 4 + G * value bytes
    int64_t cap_record;        // bytes of a staging buffer (larger records are read in place)
    int32_t prefetch;          // staged kernel: prefetch the gather rows of a slice (1 L2, 2 L1) or
                               // the rows of its epilogue (3 L1, 4 L2)
    const void* h0;
    const void* x_cur;   // x_k   [npad][R] (gathered)
    const void* x_prev;  // x_{k-1}
    void* v_out;         // v_{k+1}
    double* scal;        // [R][2] a_{k-1}, b_{k-1}
    double* partials;    // [gridDim][R][4]
    unsigned int* counter;  // [0] block counter, [1] step index, [2] error flag
    double* a_out;       // [R][nmax]
    double* b_out;
    int64_t nslices;
    int32_t nmax;
    const int32_t* field_m;  // field-batched layout: flux quanta of each right-hand side [R] (else unused)
};

using StepFn = void (*)(StepParams);
// the sparse-product kernel of the field-batched layout (gbn_fields.cu)
StepFn field_step_kernel(int prec, int G, int rpt, int tpr, bool staged);

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

struct SliceSums {
    double s1, s2, s3, s4;
};

// Reduction of the four sums over the block, then by the last block over all blocks; writes a_k, b_k.
// Needs at least 4 R threads per block.
template <int RPT, int TPR>
__device__ __forceinline__ void reduce_and_finalize(const StepParams& p, SliceSums* acc_s)
{
    constexpr int R = RPT * TPR;
    const int lane = threadIdx.x & 31;
    const int sub = lane / TPR;
    const int q = lane % TPR;
#pragma unroll
    for (int t = 0; t < RPT; ++t) {
#pragma unroll
        for (int off = TPR; off < 32; off <<= 1) {
            acc_s[t].s1 += __shfl_xor_sync(0xffffffffu, acc_s[t].s1, off);
            acc_s[t].s2 += __shfl_xor_sync(0xffffffffu, acc_s[t].s2, off);
            acc_s[t].s3 += __shfl_xor_sync(0xffffffffu, acc_s[t].s3, off);
            acc_s[t].s4 += __shfl_xor_sync(0xffffffffu, acc_s[t].s4, off);
        }
    }
    __shared__ double red[8][R][4];
    const int wib = threadIdx.x >> 5;
    if (sub == 0) {
#pragma unroll
        for (int t = 0; t < RPT; ++t) {
            const int r = q * RPT + t;
            red[wib][r][0] = acc_s[t].s1; red[wib][r][1] = acc_s[t].s2;
            red[wib][r][2] = acc_s[t].s3; red[wib][r][3] = acc_s[t].s4;
        }
    }
    __syncthreads();
    if (threadIdx.x < R * 4) {
        const int r = threadIdx.x >> 2, k = threadIdx.x & 3;
        NeumaierSum a;
        for (int wI = 0; wI < (int)(blockDim.x >> 5); ++wI) a.add(red[wI][r][k]);
        p.partials[((int64_t)blockIdx.x * R + r) * 4 + k] = a.value();
    }
    // the last block to finish reduces all blocks in a fixed order
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = (atomicAdd(p.counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!last) return;
    __threadfence();
    __shared__ double tot[R][4];
    if (threadIdx.x < R * 4) {
        const int r = threadIdx.x >> 2, k = threadIdx.x & 3;
        NeumaierSum a;
        for (unsigned int bI = 0; bI < gridDim.x; ++bI) a.add(__ldcg(&p.partials[((int64_t)bI * R + r) * 4 + k]));
        tot[r][k] = a.value();
    }
    __syncthreads();
    if (threadIdx.x < R) {
        const int r = threadIdx.x;
        const unsigned int step = p.counter[1];
        const double a = tot[r][0];
        const double b2 = tot[r][1] - 2.0 * a * tot[r][2] + a * a * tot[r][3];
        const double b = sqrt(fabs(b2));
        if (!(b > 0.0) || !isfinite(a) || !isfinite(b)) atomicOr(&p.counter[2], 1u);
        if ((int)step < p.nmax) {
            p.a_out[(int64_t)r * p.nmax + step] = a;
            p.b_out[(int64_t)r * p.nmax + step] = b;
        }
        p.scal[2 * r] = a;
        p.scal[2 * r + 1] = b;
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
// once for all G rows.  The epilogue per row adds the on-site term and is FP64 from there:
// v_{k+1} = y - b_{k-1} x_{k-1} rounded once, and the four dot-product terms.  cp/vp point at the
// thread's group in the slice record, in global memory (streamed) or in shared memory (SMEM).
// FIELD: field-batched values (FieldVal), the thread's field is that of its first right-hand side.
template <typename VT, bool CPLX, int G, int RPT, int TPR, bool SMEM, bool FIELD = false>
__device__ __forceinline__ void group_slice(const StepParams& p, int64_t s, int w, const int32_t* __restrict__ cp,
                                            const typename StoredVal<VT, CPLX, FIELD>::t* __restrict__ vp,
                                            const double* cb, SliceSums* acc_s)
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
    C2 acc[G][RPT];
    typename FieldMult<VT>::t mf = 0;
    if constexpr (FIELD) mf = (typename FieldMult<VT>::t)(int64_t)p.field_m[q * RPT];
    group_columns<VT, CPLX, G, RPT, TPR, SMEM, FIELD>(xc, w, cp, vp, acc, mf);
    // epilogue per row: the on-site term (own x_k row, loaded here so that it holds no registers during
    // the column loop), then v_{k+1} and the dot-product terms in FP64
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
            vn[t].x = (VT)((double)acc[g][t].x - cb[t] * (double)xm[t].x);
            vn[t].y = (VT)((double)acc[g][t].y - cb[t] * (double)xm[t].y);
            const double xr = xo[t].x, xi = xo[t].y, yr = acc[g][t].x, yi = acc[g][t].y;
            const double vr = vn[t].x, vi = vn[t].y;
            acc_s[t].s1 += xr * yr + xi * yi;
            acc_s[t].s2 += vr * vr + vi * vi;
            acc_s[t].s3 += xr * vr + xi * vi;
            acc_s[t].s4 += xr * xr + xi * xi;
        }
        VecIO<VT, RPT>::store(vout + (row0 + g) * R + q * RPT, vn);
    }
}

// Matrix records read from global memory.  Every block owns a contiguous range of slices (a compact
// region of the row order); its warps take neighbouring slices, so the rows they gather overlap in L1.
// FIELD: the field-batched layout (values FieldVal<VT>, fields p.field_m).
template <typename VT, bool CPLX, int G, int RPT, int TPR, bool FIELD = false>
__global__ void __launch_bounds__(256) k_spmm_step(StepParams p)
{
    using HT = typename StoredVal<VT, CPLX, FIELD>::t;
    constexpr int GPW = 32 / TPR;
    const int q = (threadIdx.x & 31) % TPR;
    const int sub = (threadIdx.x & 31) / TPR;
    double cb[RPT];
    SliceSums acc_s[RPT];
#pragma unroll
    for (int t = 0; t < RPT; ++t) {
        cb[t] = p.scal[2 * (q * RPT + t) + 1];
        acc_s[t] = SliceSums{0.0, 0.0, 0.0, 0.0};
    }
    const int nwb = (int)(blockDim.x >> 5);
    const int64_t per = (p.nslices + gridDim.x - 1) / gridDim.x;
    const int64_t s0 = (int64_t)blockIdx.x * per;
    const int64_t s1e = (s0 + per < p.nslices) ? s0 + per : p.nslices;
    for (int64_t s = s0 + (threadIdx.x >> 5); s < s1e; s += nwb) {
        const int64_t base = p.slice_ptr[s];
        const int w = (int)((p.slice_ptr[s + 1] - base) / GPW);
        const unsigned char* rec = p.mat + base * p.entry_bytes;
        group_slice<VT, CPLX, G, RPT, TPR, false, FIELD>(p, s, w, reinterpret_cast<const int32_t*>(rec) + sub,
                                                  reinterpret_cast<const HT*>(rec + (size_t)w * GPW * 4) + sub * G,
                                                  cb, acc_s);
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

// Matrix records staged in shared memory.  Each warp owns two record buffers and an mbarrier per
// buffer; its lane 0 copies the record of the warp's next-but-one slice with one bulk copy while the
// warp works on the current one, so the column indices that the gathers depend on come from shared
// memory instead of a DRAM round trip per unrolled column batch.  Optionally the warp first
// prefetches all the vector rows a slice will gather.  Records larger than a buffer (the largest
// 0.5 %) are read in place.  No block-wide synchronisation in the loop; every wait is bounded (flag
// bit 2, GBN_ERR_TIMEOUT).
// FIELD: the field-batched layout (values FieldVal<VT>, fields p.field_m).
template <typename VT, bool CPLX, int G, int RPT, int TPR, bool FIELD = false>
__global__ void __launch_bounds__(256) k_spmm_staged(StepParams p)
{
    using HT = typename StoredVal<VT, CPLX, FIELD>::t;
    constexpr int GPW = 32 / TPR;
    constexpr int R = RPT * TPR;
    extern __shared__ __align__(128) unsigned char dyn[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int q = lane % TPR;
    const int sub = lane / TPR;
    uint64_t* bar = reinterpret_cast<uint64_t*>(dyn) + 2 * wib;
    unsigned char* buf = dyn + 128 + (size_t)wib * 2 * p.cap_record;
    double cb[RPT];
    SliceSums acc_s[RPT];
#pragma unroll
    for (int t = 0; t < RPT; ++t) {
        cb[t] = p.scal[2 * (q * RPT + t) + 1];
        acc_s[t] = SliceSums{0.0, 0.0, 0.0, 0.0};
    }
    const int nwb = (int)(blockDim.x >> 5);
    const int64_t per = (p.nslices + gridDim.x - 1) / gridDim.x;
    const int64_t s0 = (int64_t)blockIdx.x * per;
    const int64_t s1e = (s0 + per < p.nslices) ? s0 + per : p.nslices;
    const int64_t eb = p.entry_bytes;

    auto rec_bytes = [&](int64_t s) { return (p.slice_ptr[s + 1] - p.slice_ptr[s]) * eb; };
    auto issue = [&](int64_t s, int st) {   // lane 0 only; records above the cap are not copied
        const int64_t bytes = rec_bytes(s);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        const bool copy = bytes > 0 && bytes <= p.cap_record;
        mbar_expect_tx(&bar[st], copy ? (uint32_t)bytes : 0u);
        if (copy) bulk_g2s(buf + st * p.cap_record, p.mat + p.slice_ptr[s] * eb, (uint32_t)bytes, &bar[st]);
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
        const int64_t bytes = rec_bytes(s);
        if (p.prefetch >= 3) prefetch_epilogue<VT, R, G, GPW>(p, s);
        if (bytes <= p.cap_record) {
            const unsigned char* rec = buf + st * p.cap_record;
            if (p.prefetch == 1 || p.prefetch == 2)
                prefetch_rows<VT, R>(p, reinterpret_cast<const int32_t*>(rec), w * GPW);
            group_slice<VT, CPLX, G, RPT, TPR, true, FIELD>(p, s, w, reinterpret_cast<const int32_t*>(rec) + sub,
                                                     reinterpret_cast<const HT*>(rec + (size_t)w * GPW * 4) + sub * G,
                                                     cb, acc_s);
        } else {
            const unsigned char* rec = p.mat + base * eb;
            group_slice<VT, CPLX, G, RPT, TPR, false, FIELD>(p, s, w, reinterpret_cast<const int32_t*>(rec) + sub,
                                                      reinterpret_cast<const HT*>(rec + (size_t)w * GPW * 4) + sub * G,
                                                      cb, acc_s);
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
    reduce_and_finalize<RPT, TPR>(p, acc_s);
}

}  // namespace gbn
