// Device building blocks shared by the recursion and the Chebyshev kernels: vector loads, the product
// of a stored hopping with a gathered vector element, and the union-column loop of the grouped sliced
// ELL (struct Ell): y[g][t] = sum over the group's union columns of val[g] * x[col][t].
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "gbn_internal.cuh"

namespace gbn {

template <typename VT> struct V2;
template <> struct V2<float> { using t = float2; };
template <> struct V2<double> { using t = double2; };

// ---------------------------------------------------------------------------- vector loads
template <typename VT, int RPT> struct VecIO;
// 32-byte loads are single 256-bit instructions (ld.global.v8 / v4.f64, sm_100): the TPR threads of a
// row group then read a whole 128-byte row in one instruction, one L1 wavefront per row
template <> struct VecIO<float, 4> {
    static __device__ __forceinline__ void load(const float2* p, float2 o[4]) {
        asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
            : "=f"(o[0].x), "=f"(o[0].y), "=f"(o[1].x), "=f"(o[1].y), "=f"(o[2].x), "=f"(o[2].y), "=f"(o[3].x),
              "=f"(o[3].y)
            : "l"(p));
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
    static __device__ __forceinline__ void load(const double2* p, double2 o[2]) {
        asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
            : "=d"(o[0].x), "=d"(o[0].y), "=d"(o[1].x), "=d"(o[1].y)
            : "l"(p));
    }
    static __device__ __forceinline__ void store(double2* p, const double2 o[2]) { p[0] = o[0]; p[1] = o[1]; }
};
template <> struct VecIO<double, 1> {
    static __device__ __forceinline__ void load(const double2* p, double2 o[1]) { o[0] = __ldg(p); }
    static __device__ __forceinline__ void store(double2* p, const double2 o[1]) { p[0] = o[0]; }
};

// hopping value types: real VT or complex V2<VT>; values are stored negated, so products are added
template <typename VT, bool CPLX> struct Hop;
template <> struct Hop<float, false> {
    using t = float;
    // packed FP32 (one FFMA2 for the real and imaginary parts)
    static __device__ __forceinline__ void madd(float2& acc, float h, float2 x) {
        acc = __ffma2_rn(make_float2(h, h), x, acc);
    }
};
template <> struct Hop<double, false> {
    using t = double;
    static __device__ __forceinline__ void madd(double2& acc, double h, double2 x) {
        acc.x = fma(h, x.x, acc.x);
        acc.y = fma(h, x.y, acc.y);
    }
};
template <typename VT> struct Hop<VT, true> {
    using t = typename V2<VT>::t;
    static __device__ __forceinline__ void madd(typename V2<VT>::t& acc, t h, typename V2<VT>::t x) {
        acc.x = fma(h.x, x.x, acc.x);
        acc.x = fma(-h.y, x.y, acc.x);
        acc.y = fma(h.x, x.y, acc.y);
        acc.y = fma(h.y, x.x, acc.y);
    }
};

// Values of the field-batched layout: the field-free (negated) hopping h and the Peierls phase per flux
// quantum t as a fixed-point fraction of a turn (2^-32 turn resolution in FP32, 2^-64 in FP64).  For m
// flux quanta the entry is h * exp(2 pi i frac(m t)); the product m t wraps exactly in integer arithmetic.
template <typename VT> struct FieldVal;
template <> struct FieldVal<float> { float h; uint32_t t; };
template <> struct FieldVal<double> { double h; uint64_t t; };

// h exp(i 2 pi u / 2^32): the top 16 bits of the turn fraction u by sincospif (exact argument), the low
// bits by the second-order expansion of exp(i pi s_lo), |pi s_lo| < 1e-4 (error below 2e-13)
__device__ __forceinline__ float2 field_rotate(FieldVal<float> v, uint32_t m)
{
    const uint32_t u = v.t * m;
    const float s_hi = (float)(int32_t)(u & 0xffff0000u) * 4.656612873077393e-10f;   // 2^-31
    const float s_lo = (float)(u & 0xffffu) * 4.656612873077393e-10f;
    float sn, cs;
    sincospif(s_hi, &sn, &cs);
    const float e = 3.14159265358979f * s_lo;
    const float er = fmaf(-0.5f * e, e, 1.0f);   // cos(e)
    const float ei = e;                          // sin(e)
    const float c2 = cs * er - sn * ei, s2 = sn * er + cs * ei;
    return make_float2(v.h * c2, v.h * s2);
}
__device__ __forceinline__ double2 field_rotate(FieldVal<double> v, uint64_t m)
{
    const uint64_t u = v.t * m;
    double sn, cs;
    sincospi((double)(int64_t)u * 1.0842021724855044e-19, &sn, &cs);   // 2^-63
    return make_double2(v.h * cs, v.h * sn);
}

// G consecutive values of one union column (G * sizeof(HT) = 4..64 bytes, naturally aligned), read
// with the widest loads: from global memory once and evicted first (the matrix is streamed every
// step), or from shared memory
template <typename HT, int G, bool SMEM>
__device__ __forceinline__ void load_group_vals(const HT* p, HT (&h)[G])
{
    constexpr int B = G * (int)sizeof(HT);
    if constexpr (B % 16 == 0) {
        uint4 t[B / 16];
#pragma unroll
        for (int i = 0; i < B / 16; ++i) {
            if constexpr (SMEM) t[i] = reinterpret_cast<const uint4*>(p)[i];
            else t[i] = __ldcs(reinterpret_cast<const uint4*>(p) + i);
        }
        memcpy(h, t, B);
    } else if constexpr (B == 8) {
        uint2 t;
        if constexpr (SMEM) t = *reinterpret_cast<const uint2*>(p);
        else t = __ldcs(reinterpret_cast<const uint2*>(p));
        memcpy(h, &t, B);
    } else {
        static_assert(B == 4, "value group of 4, 8 or a multiple of 16 bytes");
        unsigned int t;
        if constexpr (SMEM) t = *reinterpret_cast<const unsigned int*>(p);
        else t = __ldcs(reinterpret_cast<const unsigned int*>(p));
        memcpy(h, &t, B);
    }
}

// The column indices of NB union columns (whole blocks of kColUnroll, rec_slot's order) of the group whose
// first index of the current block cp points at, from shared memory (SMEM) or streamed from global memory:
// per block one 16-byte load (IB = 16), two 8-byte loads (IB = 8) or one 4-byte load per column (IB = 4).
// The narrower loads hold register pairs or single registers instead of an aligned quad; the fused step at
// two or more rows per group keeps its 128 registers without spilling only with them.  A warp's groups
// read distinct banks with 4-byte loads up to 8 groups, and with 8-byte loads pay 2-way conflicts at 16
// groups (4 wavefronts per block, as many as 4-byte loads of a column-major record).
template <int GPW, int NB, bool SMEM, int IB = 16>
__device__ __forceinline__ void load_block_cols(const int32_t* cp, int32_t (&c)[NB])
{
    static_assert(kColUnroll == 4 && NB % kColUnroll == 0, "whole blocks of four columns");
    static_assert(IB == 16 || IB == 8 || IB == 4, "16-, 8- or 4-byte index loads");
#pragma unroll
    for (int b = 0; b < NB / kColUnroll; ++b) {
        if constexpr (IB == 16) {
            const int4* p = reinterpret_cast<const int4*>(cp + b * kColUnroll * GPW);
            int4 t;
            if constexpr (SMEM) t = *p;
            else t = __ldcs(p);
            c[4 * b] = t.x;
            c[4 * b + 1] = t.y;
            c[4 * b + 2] = t.z;
            c[4 * b + 3] = t.w;
        } else if constexpr (IB == 8) {
            const int2* p = reinterpret_cast<const int2*>(cp + b * kColUnroll * GPW);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                int2 t;
                if constexpr (SMEM) t = p[h];
                else t = __ldcs(p + h);
                c[4 * b + 2 * h] = t.x;
                c[4 * b + 2 * h + 1] = t.y;
            }
        } else {
#pragma unroll
            for (int i = 0; i < kColUnroll; ++i) {
                if constexpr (SMEM) c[4 * b + i] = cp[b * kColUnroll * GPW + i];
                else c[4 * b + i] = __ldcs(cp + b * kColUnroll * GPW + i);
            }
        }
    }
}

// index-load width of the union-column loop: 16 bytes, except the fused step at two or more rows per group
template <bool FUSED, int G, int GPW>
constexpr int kIndexLoad = !(FUSED && G > 1) ? 16 : GPW <= 8 ? 4 : GPW <= 16 ? 8 : 16;

// Offset of a thread's first value in a slice record's values (VS > 1: the field tile table, one value
// block per thread slot q of the group).
template <typename HT, int G, int TPR, int VS>
__device__ __forceinline__ int val_thread_off(int sub, int q)
{
    if constexpr (VS == 1 && block_vals(G, (int)sizeof(HT))) return sub * kColUnroll;
    else if constexpr (VS > 1) return (sub * TPR + q) * G;
    else return sub * G;
}

// The G values of each of NB union columns (whole blocks, val_slot's order) from the thread's pointer
// into the current block.  One FP32 value per column: a block's four values with one 16-byte load, which
// a warp's groups serve from distinct banks.  Otherwise one load of G values per column, column-major.
template <typename HT, int G, int GPW, int NB, bool SMEM, int VS>
__device__ __forceinline__ void load_block_vals(const HT* vp, HT (&h)[NB][G])
{
#pragma unroll
    for (int b = 0; b < NB / kColUnroll; ++b) {
        if constexpr (VS == 1 && block_vals(G, (int)sizeof(HT))) {
            HT hb[kColUnroll];
            load_group_vals<HT, kColUnroll, SMEM>(vp + b * kColUnroll * GPW, hb);
#pragma unroll
            for (int i = 0; i < kColUnroll; ++i) h[kColUnroll * b + i][0] = hb[i];
        } else {
#pragma unroll
            for (int i = 0; i < kColUnroll; ++i)
                load_group_vals<HT, G, SMEM>(vp + (b * kColUnroll + i) * GPW * G * VS, h[kColUnroll * b + i]);
        }
    }
}

// The union-column loop of one group: GPW = 32/TPR groups per slice; the TPR threads of a group each
// hold RPT right-hand sides of all G rows of the group.  Per union column a thread reads the column
// index and the G values (same address for the group's threads) and gathers RPT vector elements of that
// column once for all G rows.  cp/vp point at the thread's group in the slice record (its first
// column of the current block, rec_slot's order); the indices come
// from shared memory (SMEM) or global memory (streamed, evict-first), the values likewise (SMEM_VAL).
// w is the slice width (a multiple of kColUnroll).  U columns are in flight per batch: their indices,
// gathers and values are all issued before the first product, so U gathers wait on memory together.
// FIELD: the values are FieldVal<VT> and every thread rotates them by its right-hand sides' field mf
// (mf flux quanta, the same for the thread's RPT right-hand sides) before the complex products.
template <typename VT, bool CPLX, bool FIELD> struct StoredVal { using t = typename Hop<VT, CPLX>::t; };
template <typename VT, bool CPLX> struct StoredVal<VT, CPLX, true> { using t = FieldVal<VT>; };
template <typename VT> struct FieldMult;
template <> struct FieldMult<float> { using t = uint32_t; };
template <> struct FieldMult<double> { using t = uint64_t; };

// x = v + a u per element, the same instruction wherever it is formed (packed FP32 FMA, or two FP64 FMAs)
__device__ __forceinline__ float2 fused_form(float2 a, float2 u, float2 v) { return __ffma2_rn(a, u, v); }
__device__ __forceinline__ double2 fused_form(double2 a, double2 u, double2 v)
{
    return make_double2(fma(a.x, u.x, v.x), fma(a.y, u.y, v.y));
}

// FUSED (real or field-batched values): the gathered vector is formed from two stored ones,
// x = v + (-alpha) u, by one
// packed FMA per element from the same two loads wherever the column is gathered (xq: v, xu: u, al: the
// thread's -alpha pairs), so every row sees the same rounded x.
template <typename VT, bool CPLX, int G, int RPT, int TPR, bool SMEM, bool SMEM_VAL, bool FIELD, int NB, int VS = 1,
          bool FUSED = false>
__device__ __forceinline__ void column_batch(const typename V2<VT>::t* __restrict__ xq,
                                             const int32_t* __restrict__ cp,
                                             const typename StoredVal<VT, CPLX, FIELD>::t* __restrict__ vp,
                                             typename V2<VT>::t (&acc)[G][RPT], typename FieldMult<VT>::t mf,
                                             const typename V2<VT>::t* __restrict__ xu = nullptr,
                                             const typename V2<VT>::t* al = nullptr)
{
    using C2 = typename V2<VT>::t;
    using HT = typename StoredVal<VT, CPLX, FIELD>::t;
    constexpr int GPW = 32 / TPR;
    constexpr int R = RPT * TPR;
    int32_t c[NB];
    HT h[NB][G];
    C2 xg[NB][RPT];
    load_block_cols<GPW, NB, SMEM, kIndexLoad<FUSED, G, GPW>>(cp, c);
#pragma unroll
    for (int u = 0; u < NB; ++u) VecIO<VT, RPT>::load(xq + (size_t)(uint32_t)c[u] * R, xg[u]);
    if constexpr (FUSED) {
        static_assert(!CPLX, "the fused gather is for layouts of real or field-batched values");
        C2 xh[NB][RPT];
#pragma unroll
        for (int u = 0; u < NB; ++u) VecIO<VT, RPT>::load(xu + (size_t)(uint32_t)c[u] * R, xh[u]);
#pragma unroll
        for (int u = 0; u < NB; ++u)
#pragma unroll
            for (int t = 0; t < RPT; ++t) xg[u][t] = fused_form(al[t], xh[u][t], xg[u][t]);
    }
    load_block_vals<HT, G, GPW, NB, SMEM_VAL, VS>(vp, h);
    if constexpr (FIELD) {
#pragma unroll
        for (int u = 0; u < NB; ++u)
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const C2 hr = field_rotate(h[u][g], mf);
#pragma unroll
                for (int t = 0; t < RPT; ++t) Hop<VT, true>::madd(acc[g][t], hr, xg[u][t]);
            }
    } else {
#pragma unroll
        for (int u = 0; u < NB; ++u)
#pragma unroll
            for (int g = 0; g < G; ++g)
#pragma unroll
                for (int t = 0; t < RPT; ++t) Hop<VT, CPLX>::madd(acc[g][t], h[u][g], xg[u][t]);
    }
}

// VS: value blocks per union column and group (the field tile table holds one per thread slot, VS = TPR,
// interleaved [column][group][slot][G]); the caller's vp includes the thread's own slot.
template <typename VT, bool CPLX, int G, int RPT, int TPR, bool SMEM, bool FIELD = false, int U = kColUnroll,
          bool SMEM_VAL = SMEM, int VS = 1, bool FUSED = false>
__device__ __forceinline__ void group_columns(const typename V2<VT>::t* __restrict__ x, int w,
                                              const int32_t* __restrict__ cp,
                                              const typename StoredVal<VT, CPLX, FIELD>::t* __restrict__ vp,
                                              typename V2<VT>::t (&acc)[G][RPT],
                                              typename FieldMult<VT>::t mf = 0,
                                              const typename V2<VT>::t* __restrict__ xu = nullptr,
                                              const typename V2<VT>::t* al = nullptr)
{
    using C2 = typename V2<VT>::t;
    constexpr int GPW = 32 / TPR;
    static_assert(U % kColUnroll == 0, "the unroll is a multiple of the slice-width granule");
    const int q = (threadIdx.x & 31) % TPR;
    const C2* __restrict__ xq = x + q * RPT;
    const C2* __restrict__ xuq = FUSED ? xu + q * RPT : nullptr;
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
        for (int t = 0; t < RPT; ++t) { acc[g][t].x = 0; acc[g][t].y = 0; }
    int k = 0;
    for (; k + U <= w; k += U) {
        column_batch<VT, CPLX, G, RPT, TPR, SMEM, SMEM_VAL, FIELD, U, VS, FUSED>(xq, cp, vp, acc, mf, xuq, al);
        cp += U * GPW;
        vp += U * GPW * G * VS;
    }
    if constexpr (U > kColUnroll) {
        for (; k < w; k += kColUnroll) {
            column_batch<VT, CPLX, G, RPT, TPR, SMEM, SMEM_VAL, FIELD, kColUnroll, VS, FUSED>(xq, cp, vp, acc, mf,
                                                                                              xuq, al);
            cp += kColUnroll * GPW;
            vp += kColUnroll * GPW * G * VS;
        }
    }
}

}  // namespace gbn
