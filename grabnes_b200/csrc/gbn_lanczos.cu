// Batched Lanczos recursion on the B200: two launches per recursion step.
//
// The reference (lanczosKuboCode/Src/kubosubs.F90:26-138) makes three passes over the vectors per
// step: H psi with <psi, H psi>; w = H psi - a psi - b psi_prev with |w|; the scaling psi = w / b.
// Here the carried state is the pair
//     v_k = H x_{k-1} - b_{k-2} x_{k-2}      and     x_{k-1},
// and a step is
//   k_update    x_k = (v_k - a_{k-1} x_{k-1}) / b_{k-1}             stream: read v, x_{k-1}; write x_k
//   k_spmm_step y = H x_k (one gather of x_k per matrix entry), v_{k+1} = y - b_{k-1} x_{k-1}, and
//               four FP64 dot products per vector
//                  S1 = Re<x_k, y>, S2 = |v_{k+1}|^2, S3 = Re<x_k, v_{k+1}>, S4 = |x_k|^2,
//               from which a_k = S1 and b_k^2 = |v_{k+1} - a_k x_k|^2 = S2 - 2 a_k S3 + a_k^2 S4.
// The partial sums of the blocks are reduced in a fixed order by the last block to finish (so the
// result does not depend on scheduling), which also writes a_k, b_k and the scalars of the next step.
// Each matrix entry is gathered once per step: for many right-hand sides the gathers, not the
// DRAM stream, bound the product (a row of R vectors is read once per neighbour that references it).
//
// Vectors of R right-hand sides are interleaved per row ([row][R] complex): TPR threads share a row,
// each holding RPT right-hand sides (16-32 bytes per gather); a warp processes a slice of
// SH = 32/TPR rows of the sliced-ELL matrix.
#include <cuda_runtime.h>
#include <math.h>

#include "gbn_internal.cuh"

namespace gbn {

template <typename VT> struct V2;
template <> struct V2<float> { using t = float2; };
template <> struct V2<double> { using t = double2; };

struct StepParams {
    const int64_t* slice_ptr;
    const int32_t* col;
    const void* val;
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
    int64_t max_chunk;   // entries of the largest chunk (staged kernel)
    int32_t nmax;
};

// ---------------------------------------------------------------------------- vector loads
template <typename VT, int RPT> struct VecIO;
template <> struct VecIO<float, 4> {
    static __device__ __forceinline__ void load(const float2* p, float2 o[4]) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(p));
        const float4 b = __ldg(reinterpret_cast<const float4*>(p) + 1);
        o[0] = make_float2(a.x, a.y); o[1] = make_float2(a.z, a.w);
        o[2] = make_float2(b.x, b.y); o[3] = make_float2(b.z, b.w);
    }
    static __device__ __forceinline__ void store(float2* p, const float2 o[4]) {
        reinterpret_cast<float4*>(p)[0] = make_float4(o[0].x, o[0].y, o[1].x, o[1].y);
        reinterpret_cast<float4*>(p)[1] = make_float4(o[2].x, o[2].y, o[3].x, o[3].y);
    }
};
template <> struct VecIO<float, 2> {
    static __device__ __forceinline__ void load(const float2* p, float2 o[2]) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(p));
        o[0] = make_float2(a.x, a.y); o[1] = make_float2(a.z, a.w);
    }
    static __device__ __forceinline__ void store(float2* p, const float2 o[2]) {
        reinterpret_cast<float4*>(p)[0] = make_float4(o[0].x, o[0].y, o[1].x, o[1].y);
    }
};
template <> struct VecIO<float, 1> {
    static __device__ __forceinline__ void load(const float2* p, float2 o[1]) { o[0] = __ldg(p); }
    static __device__ __forceinline__ void store(float2* p, const float2 o[1]) { p[0] = o[0]; }
};
template <> struct VecIO<double, 2> {
    static __device__ __forceinline__ void load(const double2* p, double2 o[2]) { o[0] = __ldg(p); o[1] = __ldg(p + 1); }
    static __device__ __forceinline__ void store(double2* p, const double2 o[2]) { p[0] = o[0]; p[1] = o[1]; }
};
template <> struct VecIO<double, 1> {
    static __device__ __forceinline__ void load(const double2* p, double2 o[1]) { o[0] = __ldg(p); }
    static __device__ __forceinline__ void store(double2* p, const double2 o[1]) { p[0] = o[0]; }
};

// hopping value types: real VT or complex V2<VT>
template <typename VT, bool CPLX> struct Hop;
template <typename VT> struct Hop<VT, false> {
    using t = VT;
    static __device__ __forceinline__ void msub(typename V2<VT>::t& acc, VT h, typename V2<VT>::t x) {
        acc.x = fma(-h, x.x, acc.x);
        acc.y = fma(-h, x.y, acc.y);
    }
    static __device__ __forceinline__ VT load(const VT* p) { return __ldcs(p); }
};
template <typename VT> struct Hop<VT, true> {
    using t = typename V2<VT>::t;
    static __device__ __forceinline__ void msub(typename V2<VT>::t& acc, t h, typename V2<VT>::t x) {
        acc.x = fma(-h.x, x.x, acc.x);
        acc.x = fma(h.y, x.y, acc.x);
        acc.y = fma(-h.x, x.y, acc.y);
        acc.y = fma(-h.y, x.x, acc.y);
    }
    static __device__ __forceinline__ t load(const t* p) { return __ldcs(p); }
};

// ---------------------------------------------------------------------------- update kernel
// x_k = (v_k - a x_{k-1}) * (1/b) for all rows and right-hand sides (streaming, 16 B per thread).
template <typename VT>
__global__ void __launch_bounds__(256) k_update(const typename V2<VT>::t* __restrict__ v,
                                                const typename V2<VT>::t* __restrict__ xp,
                                                typename V2<VT>::t* __restrict__ xc, const double* __restrict__ scal,
                                                int64_t total, int R)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += stride) {
        const int r = (int)(e % R);
        const double a = scal[2 * r], b = scal[2 * r + 1];
        const typename V2<VT>::t vv = __ldcs(v + e), xx = __ldcs(xp + e);
        typename V2<VT>::t o;   // FP64 arithmetic, one rounding to the storage type
        o.x = (VT)(((double)vv.x - a * (double)xx.x) / b);
        o.y = (VT)(((double)vv.y - a * (double)xx.y) / b);
        xc[e] = o;
    }
}

// ---------------------------------------------------------------------------- SpMM kernels
// matrix entries are read either from global memory (streamed, evict-first) or from shared memory
struct FromGlobal {
    template <typename T> static __device__ __forceinline__ T ld(const T* p) { return __ldcs(p); }
};
struct FromShared {
    template <typename T> static __device__ __forceinline__ T ld(const T* p) { return *p; }
};

struct SliceSums {
    double s1, s2, s3, s4;
};

// One slice of SH rows: y = H x_k for the thread's row and right-hand sides, v_{k+1} = y - b x_{k-1},
// and the four dot-product terms of the row.
template <typename VT, bool CPLX, int RPT, int TPR, typename SRC>
__device__ __forceinline__ void spmm_slice(const StepParams& p, int64_t s, int w, const int32_t* __restrict__ cp,
                                           const typename Hop<VT, CPLX>::t* __restrict__ hp, const double* cb,
                                           SliceSums* acc_s)
{
    using C2 = typename V2<VT>::t;
    using HT = typename Hop<VT, CPLX>::t;
    constexpr int SH = 32 / TPR;
    constexpr int R = RPT * TPR;
    const int lane = threadIdx.x & 31;
    const int sub = lane / TPR;
    const int q = lane % TPR;
    const C2* __restrict__ xc = static_cast<const C2*>(p.x_cur);
    const C2* __restrict__ xp = static_cast<const C2*>(p.x_prev);
    C2* __restrict__ vout = static_cast<C2*>(p.v_out);
    const VT* __restrict__ h0 = static_cast<const VT*>(p.h0);
    const int64_t row = s * SH + sub;
    C2 xo[RPT], acc[RPT];
    VecIO<VT, RPT>::load(xc + row * R + q * RPT, xo);
    const VT d = h0[row];
#pragma unroll
    for (int t = 0; t < RPT; ++t) { acc[t].x = d * xo[t].x; acc[t].y = d * xo[t].y; }
    // batches of KB entries: all column indices first, then all gathers, then the products, so that KB
    // independent gathers are in flight per thread
    constexpr int KB = (RPT * sizeof(VT) >= 16) ? 8 : 16;
    for (int k0 = 0; k0 < w; k0 += KB) {
        int32_t c[KB];
        HT h[KB];
#pragma unroll
        for (int j = 0; j < KB; ++j) {
            if (k0 + j < w) {
                c[j] = SRC::ld(cp + (int64_t)(k0 + j) * SH);
                h[j] = SRC::ld(hp + (int64_t)(k0 + j) * SH);
            } else {
                c[j] = (int32_t)row;
                h[j] = HT{};
            }
        }
        C2 xg[KB][RPT];
#pragma unroll
        for (int j = 0; j < KB; ++j) VecIO<VT, RPT>::load(xc + (int64_t)c[j] * R + q * RPT, xg[j]);
#pragma unroll
        for (int j = 0; j < KB; ++j)
#pragma unroll
            for (int t = 0; t < RPT; ++t) Hop<VT, CPLX>::msub(acc[t], h[j], xg[j][t]);
    }
    C2 xm[RPT], vn[RPT];
    VecIO<VT, RPT>::load(xp + row * R + q * RPT, xm);
#pragma unroll
    for (int t = 0; t < RPT; ++t) {
        // epilogue in FP64: v_{k+1} = y - b_{k-1} x_{k-1}, rounded once to the storage type
        vn[t].x = (VT)((double)acc[t].x - cb[t] * (double)xm[t].x);
        vn[t].y = (VT)((double)acc[t].y - cb[t] * (double)xm[t].y);
        const double xr = xo[t].x, xi = xo[t].y, yr = acc[t].x, yi = acc[t].y, vr = vn[t].x, vi = vn[t].y;
        acc_s[t].s1 += xr * yr + xi * yi;
        acc_s[t].s2 += vr * vr + vi * vi;
        acc_s[t].s3 += xr * vr + xi * vi;
        acc_s[t].s4 += xr * xr + xi * xi;
    }
    VecIO<VT, RPT>::store(vout + row * R + q * RPT, vn);
}

// Reduction of the four sums over the block, then by the last block over all blocks; writes a_k, b_k.
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
        double a = 0.0;
        for (int wI = 0; wI < (int)(blockDim.x >> 5); ++wI) a += red[wI][r][k];
        p.partials[((int64_t)blockIdx.x * R + r) * 4 + k] = a;
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
        double a = 0.0;
        for (unsigned int bI = 0; bI < gridDim.x; ++bI) a += __ldcg(&p.partials[((int64_t)bI * R + r) * 4 + k]);
        tot[r][k] = a;
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

// Matrix read from global memory.  Every block owns a contiguous range of slices (a compact region of
// the Morton order); its warps take neighbouring slices, so the rows they gather overlap in L1.
template <typename VT, bool CPLX, int RPT, int TPR>
__global__ void __launch_bounds__(256) k_spmm_step(StepParams p)
{
    using HT = typename Hop<VT, CPLX>::t;
    constexpr int SH = 32 / TPR;
    const int q = (threadIdx.x & 31) % TPR;
    const int sub = (threadIdx.x & 31) / TPR;
    double cb[RPT];
    SliceSums acc_s[RPT];
#pragma unroll
    for (int t = 0; t < RPT; ++t) {
        cb[t] = p.scal[2 * (q * RPT + t) + 1];
        acc_s[t] = SliceSums{0.0, 0.0, 0.0, 0.0};
    }
    const HT* __restrict__ val = static_cast<const HT*>(p.val);
    const int nwb = (int)(blockDim.x >> 5);
    const int64_t per = (p.nslices + gridDim.x - 1) / gridDim.x;
    const int64_t s0 = (int64_t)blockIdx.x * per;
    const int64_t s1e = (s0 + per < p.nslices) ? s0 + per : p.nslices;
    for (int64_t s = s0 + (threadIdx.x >> 5); s < s1e; s += nwb) {
        const int64_t base = p.slice_ptr[s];
        const int w = (int)((p.slice_ptr[s + 1] - base) / SH);
        spmm_slice<VT, CPLX, RPT, TPR, FromGlobal>(p, s, w, p.col + base + sub, val + base + sub, cb, acc_s);
    }
    reduce_and_finalize<RPT, TPR>(p, acc_s);
}

// ---- bulk asynchronous copies (TMA, cp.async.bulk) into shared memory with mbarrier completion
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

// Matrix staged in shared memory: the block's slices are processed in chunks of kChunkSlices
// consecutive slices (one per warp); thread 0 copies chunk i+2 while the warps work on chunk i
// (double buffering, completion by mbarrier transaction counts).  Chunks start on 16-byte boundaries
// and hold a multiple of 16 bytes (slices hold a multiple of 4 entries).
template <typename VT, bool CPLX, int RPT, int TPR>
__global__ void __launch_bounds__(256) k_spmm_staged(StepParams p)
{
    using HT = typename Hop<VT, CPLX>::t;
    constexpr int SH = 32 / TPR;
    extern __shared__ __align__(128) unsigned char dyn[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(dyn);               // 2 barriers
    int32_t* scol[2];
    HT* sval[2];
    {
        unsigned char* b = dyn + 128;
        const size_t ccol = (size_t)p.max_chunk * sizeof(int32_t), cval = (size_t)p.max_chunk * sizeof(HT);
        scol[0] = reinterpret_cast<int32_t*>(b);
        sval[0] = reinterpret_cast<HT*>(b + ccol);
        scol[1] = reinterpret_cast<int32_t*>(b + ccol + cval);
        sval[1] = reinterpret_cast<HT*>(b + 2 * ccol + cval);
    }
    const int q = (threadIdx.x & 31) % TPR;
    const int sub = (threadIdx.x & 31) / TPR;
    const int wib = threadIdx.x >> 5;
    double cb[RPT];
    SliceSums acc_s[RPT];
#pragma unroll
    for (int t = 0; t < RPT; ++t) {
        cb[t] = p.scal[2 * (q * RPT + t) + 1];
        acc_s[t] = SliceSums{0.0, 0.0, 0.0, 0.0};
    }
    const int32_t* __restrict__ gcol = p.col;
    const HT* __restrict__ gval = static_cast<const HT*>(p.val);
    const int64_t nchunks = (p.nslices + kChunkSlices - 1) / kChunkSlices;
    const int64_t per = (nchunks + gridDim.x - 1) / gridDim.x;
    const int64_t c0 = (int64_t)blockIdx.x * per;
    const int64_t c1 = (c0 + per < nchunks) ? c0 + per : nchunks;

    auto issue = [&](int64_t ci, int buf) {
        const int64_t sa = ci * kChunkSlices;
        const int64_t sb = (sa + kChunkSlices < p.nslices) ? sa + kChunkSlices : p.nslices;
        const int64_t e0 = p.slice_ptr[sa], e1 = p.slice_ptr[sb];
        const uint32_t ne = (uint32_t)(e1 - e0);
        const uint32_t bc = ne * (uint32_t)sizeof(int32_t), bv = ne * (uint32_t)sizeof(HT);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&bar[buf], bc + bv);
        if (ne) {
            bulk_g2s(scol[buf], gcol + e0, bc, &bar[buf]);
            bulk_g2s(sval[buf], gval + e0, bv, &bar[buf]);
        }
    };

    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (c0 < c1) issue(c0, 0);
        if (c0 + 1 < c1) issue(c0 + 1, 1);
    }
    uint32_t phase[2] = {0u, 0u};
    bool ok = true;
    for (int64_t ci = c0; ci < c1; ++ci) {
        const int buf = (int)((ci - c0) & 1);
        const bool got = mbar_wait_bounded(&bar[buf], phase[buf]);
        phase[buf] ^= 1u;
        if (!__syncthreads_and(got)) {   // uniform exit of the block if a copy never completed
            ok = false;
            break;
        }
        const int64_t s = ci * kChunkSlices + wib;
        if (s < p.nslices && wib < kChunkSlices) {
            const int64_t ebase = p.slice_ptr[ci * kChunkSlices];
            const int64_t base = p.slice_ptr[s];
            const int w = (int)((p.slice_ptr[s + 1] - base) / SH);
            spmm_slice<VT, CPLX, RPT, TPR, FromShared>(p, s, w, scol[buf] + (base - ebase) + sub,
                                                       sval[buf] + (base - ebase) + sub, cb, acc_s);
        }
        __syncthreads();
        if (threadIdx.x == 0 && ci + 2 < c1) issue(ci + 2, buf);
    }
    if (!ok) {
        if (threadIdx.x == 0) atomicOr(&p.counter[2], 2u);
        // let copies still in flight land before the block's shared memory is released
        mbar_wait_bounded(&bar[0], phase[0]);
        mbar_wait_bounded(&bar[1], phase[1]);
        __syncthreads();
    }
    reduce_and_finalize<RPT, TPR>(p, acc_s);
}

// ---------------------------------------------------------------------------- start vectors
// v <- psi (permuted rows), x_prev <- 0; then the first update gives x_1 = psi (a_0 = 0, b_0 = 1).
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

__global__ void k_init_scalars(double* scal, unsigned int* counter, int R)
{
    const int r = threadIdx.x;
    if (r < R) {
        scal[2 * r] = 0.0;
        scal[2 * r + 1] = 1.0;
    }
    if (r == 0) {
        counter[0] = 0u;
        counter[1] = 0u;
        counter[2] = 0u;
    }
}

// ---------------------------------------------------------------------------- host side
// right-hand sides per thread: the widest vector load (32 bytes) unless the tuning asks for fewer
static void split_rhs(int prec, int R, int want, int* rpt, int* tpr)
{
    const int maxr = (prec == GBN_MIXED) ? 4 : 2;
    int r = R < maxr ? R : maxr;
    if (want > 0 && want < r && R % want == 0) r = want;
    if (R / r > 32) r = R / 32;
    *rpt = r;
    *tpr = R / r;
}

int rows_per_slice(int prec, int nrhs, int want_rpt)
{
    int rpt, tpr;
    split_rhs(prec, nrhs, want_rpt, &rpt, &tpr);
    return 32 / tpr;
}

using StepFn = void (*)(StepParams);

template <typename VT, bool CPLX>
static StepFn pick(int rpt, int tpr, bool staged)
{
#define GBN_CASE(RP, TP) \
    if (rpt == RP && tpr == TP) return staged ? k_spmm_staged<VT, CPLX, RP, TP> : k_spmm_step<VT, CPLX, RP, TP>;
    GBN_CASE(1, 1) GBN_CASE(1, 2) GBN_CASE(1, 4) GBN_CASE(1, 8) GBN_CASE(1, 16) GBN_CASE(1, 32)
    GBN_CASE(2, 1) GBN_CASE(2, 2) GBN_CASE(2, 4) GBN_CASE(2, 8) GBN_CASE(2, 16)
    if constexpr (sizeof(VT) == 4) {
        GBN_CASE(4, 1) GBN_CASE(4, 2) GBN_CASE(4, 4) GBN_CASE(4, 8)
    }
#undef GBN_CASE
    return nullptr;
}

static StepFn step_kernel(int prec, bool cplx, int R, int want_rpt, bool staged)
{
    int rpt, tpr;
    split_rhs(prec, R, want_rpt, &rpt, &tpr);
    if (prec == GBN_MIXED) return cplx ? pick<float, true>(rpt, tpr, staged) : pick<float, false>(rpt, tpr, staged);
    return cplx ? pick<double, true>(rpt, tpr, staged) : pick<double, false>(rpt, tpr, staged);
}

// dynamic shared memory of the staged kernel: two chunk buffers of column indices and values
static size_t staged_smem(const gbn_ctx* c)
{
    return 128 + 2 * (size_t)c->ell.max_chunk_entries * (sizeof(int32_t) + (size_t)c->ell.val_size);
}

static bool use_staged(const gbn_ctx* c)
{
    if (c->tune_staged == 0) return false;
    return staged_smem(c) <= 160 * 1024;
}

static int step_grid(gbn_ctx* c, StepFn fn, size_t smem)
{
    int per_sm = 0;
    if (smem > 0) cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, smem) != cudaSuccess || per_sm < 1) per_sm = 1;
    if (c->tune_blocks_per_sm > 0 && c->tune_blocks_per_sm < per_sm) per_sm = c->tune_blocks_per_sm;
    return c->num_sms * per_sm;
}

int lanczos_prepare(gbn_ctx* c, int prec, int nrhs)
{
    if (nrhs != 1 && nrhs != 2 && nrhs != 4 && nrhs != 8 && nrhs != 16 && nrhs != 32)
        return fail(c, GBN_ERR_ARG, "internal: tile width must be 1, 2, 4, 8, 16 or 32");
    const int sh = rows_per_slice(prec, nrhs, c->tune_rpt);
    if (!c->ell.valid || c->ell.prec != prec || c->ell.sh != sh) {
        const int rc = build_ell(c, prec, sh);
        if (rc) return rc;
    }
    c->prec = prec;
    c->nrhs = nrhs;
    const size_t esz = (prec == GBN_MIXED) ? sizeof(float2) : sizeof(double2);
    const size_t vbytes = (size_t)c->ell.npad * nrhs * esz;
    for (int i = 0; i < 3; ++i) GBN_CK(c, c->vec[i].ensure(vbytes));
    const bool staged = use_staged(c);
    StepFn fn = step_kernel(prec, c->ell.cplx, nrhs, c->tune_rpt, staged);
    if (!fn) return fail(c, GBN_ERR_ARG, "no recursion kernel for this tile width");
    const int grid = step_grid(c, fn, staged ? staged_smem(c) : 0);
    GBN_CK(c, c->partials.ensure(sizeof(double) * (size_t)grid * nrhs * 4));
    GBN_CK(c, c->scal.ensure(sizeof(double) * 2 * nrhs));
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
                                                               c->perm.as<int32_t>(), c->n, c->ell.npad, c->nrhs,
                                                               nrhs_real, isn);
    else
        k_start_from_phases<double><<<grd, blk, 0, c->stream>>>(c->vec[0].as<double2>(), c->vec[1].as<double2>(),
                                                                d_u, c->perm.as<int32_t>(), c->n, c->ell.npad,
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
                                                            c->perm.as<int32_t>(), c->n, c->ell.npad, c->nrhs, nrhs_real);
    else
        k_start_from_psi<double><<<grd, blk, 0, c->stream>>>(c->vec[0].as<double2>(), c->vec[1].as<double2>(),
                                                             reinterpret_cast<const double2*>(d_psi),
                                                             c->perm.as<int32_t>(), c->n, c->ell.npad, c->nrhs,
                                                             nrhs_real);
    GBN_CK_LAUNCH(c);
    return GBN_OK;
}

int lanczos_run(gbn_ctx* c, int32_t nmax)
{
    const int R = c->nrhs;
    GBN_CK(c, c->ab.ensure(sizeof(double) * 2 * (size_t)R * nmax));
    k_init_scalars<<<1, 64, 0, c->stream>>>(c->scal.as<double>(), c->counter.as<unsigned int>(), R);
    GBN_CK_LAUNCH(c);
    const bool staged = use_staged(c);
    const size_t smem = staged ? staged_smem(c) : 0;
    StepFn fn = step_kernel(c->prec, c->ell.cplx, R, c->tune_rpt, staged);
    if (!fn) return fail(c, GBN_ERR_ARG, "no recursion kernel for this tile width");
    const int grid = step_grid(c, fn, smem);
    c->last_staged = staged;
    StepParams p;
    p.slice_ptr = c->ell.slice_ptr.as<int64_t>();
    p.col = c->ell.col.as<int32_t>();
    p.val = c->ell.val.p;
    p.h0 = c->ell.h0.p;
    p.v_out = c->vec[0].p;
    p.scal = c->scal.as<double>();
    p.partials = c->partials.as<double>();
    p.counter = c->counter.as<unsigned int>();
    p.a_out = c->ab.as<double>();
    p.b_out = c->ab.as<double>() + (size_t)R * nmax;
    p.nslices = c->ell.nslices;
    p.max_chunk = c->ell.max_chunk_entries;
    p.nmax = nmax;
    const int64_t total = c->ell.npad * R;
    const int ublk = 256;
    const int ugrid = c->num_sms * 8;
    if (!c->ev0) {
        GBN_CK(c, cudaEventCreate(&c->ev0));
        GBN_CK(c, cudaEventCreate(&c->ev1));
    }
    // per-kernel durations of the first steps (three events per sampled step)
    const int nsample = nmax < kTimedSteps ? nmax : kTimedSteps;
    if (!c->kev[0]) {
        for (int i = 0; i < 3 * kTimedSteps; ++i) GBN_CK(c, cudaEventCreate(&c->kev[i]));
    }
    GBN_CK(c, cudaEventRecord(c->ev0, c->stream));
    for (int32_t k = 0; k < nmax; ++k) {
        // step k (0-based): x_prev in vec[1 + k%2], x_cur written to vec[1 + (k+1)%2]
        void* xprev = c->vec[1 + (k & 1)].p;
        void* xcur = c->vec[1 + ((k + 1) & 1)].p;
        if (k < nsample) GBN_CK(c, cudaEventRecord(c->kev[3 * k], c->stream));
        if (c->prec == GBN_MIXED)
            k_update<float><<<ugrid, ublk, 0, c->stream>>>(c->vec[0].as<float2>(), static_cast<const float2*>(xprev),
                                                          static_cast<float2*>(xcur), c->scal.as<double>(), total, R);
        else
            k_update<double><<<ugrid, ublk, 0, c->stream>>>(c->vec[0].as<double2>(), static_cast<const double2*>(xprev),
                                                           static_cast<double2*>(xcur), c->scal.as<double>(), total, R);
        GBN_CK_LAUNCH(c);
        if (k < nsample) GBN_CK(c, cudaEventRecord(c->kev[3 * k + 1], c->stream));
        p.x_cur = xcur;
        p.x_prev = xprev;
        fn<<<grid, 256, smem, c->stream>>>(p);
        GBN_CK_LAUNCH(c);
        if (k < nsample) GBN_CK(c, cudaEventRecord(c->kev[3 * k + 2], c->stream));
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
