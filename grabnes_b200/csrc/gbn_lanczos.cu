// Batched Lanczos recursion on the B200: one fused kernel per recursion step.
//
// The reference (lanczosKuboCode/Src/kubosubs.F90:26-138) makes three passes over the vectors per
// step (H psi with <psi,H psi>; w = H psi - a psi - b psi_prev with |w|; scaling).  Here a step is one
// pass.  The state carried between steps is the pair
//     v_k = H x_{k-1} - b_{k-2} x_{k-2}      and     x_{k-1}
// from which x_k = (v_k - a_{k-1} x_{k-1}) / b_{k-1} is formed wherever it is needed (own row and every
// gathered neighbour).  By linearity H x_k = (H v_k - a_{k-1} H x_{k-1}) / b_{k-1}, so the sparse
// product accumulates H v and H x separately and combines them once per row.  The step writes the next
// pair (v_{k+1} = H x_k - b_{k-1} x_{k-1}, x_k) and four FP64 dot products per vector,
//     S1 = Re<x_k, H x_k>, S2 = |v_{k+1}|^2, S3 = Re<x_k, v_{k+1}>, S4 = |x_k|^2,
// from which a_k = S1 and b_k^2 = |v_{k+1} - a_k x_k|^2 = S2 - 2 a_k S3 + a_k^2 S4 follow exactly.
// Memory traffic per step: matrix + 2 vector reads + 2 vector writes (the reference's loop structure
// needs matrix + 7).  The block partial sums are reduced in a fixed order by the last block to finish
// (deterministic), which also writes a_k, b_k and the scalars of the next step.
//
// Vectors of R right-hand sides are interleaved per row ([row][R] complex), so a row of R vectors is
// one contiguous segment: TPR threads share a row, each holding RPT right-hand sides (16-32 bytes of
// vector loads per gather).  Rows are processed in slices of SH = 32/TPR rows by one warp.
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
    const void* v_in;   // [npad][R]
    const void* x_in;
    void* v_out;
    void* x_out;
    double* scal;       // [R][2] a_{k-1}, b_{k-1}
    double* partials;   // [gridDim][R][4]
    unsigned int* counter;  // [0] block counter, [1] step index, [2] error flag
    double* a_out;      // [R][nmax]
    double* b_out;
    int64_t nslices;
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
    // acc -= h * x
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

// ---------------------------------------------------------------------------- step kernel
template <typename VT, bool CPLX, int RPT, int TPR>
__global__ void __launch_bounds__(256) k_lanczos_step(StepParams p)
{
    using C2 = typename V2<VT>::t;
    using HT = typename Hop<VT, CPLX>::t;
    constexpr int SH = 32 / TPR;
    constexpr int R = RPT * TPR;
    const int lane = threadIdx.x & 31;
    const int sub = lane / TPR;
    const int q = lane % TPR;

    const C2* __restrict__ vin = static_cast<const C2*>(p.v_in);
    const C2* __restrict__ xin = static_cast<const C2*>(p.x_in);
    C2* __restrict__ vout = static_cast<C2*>(p.v_out);
    C2* __restrict__ xout = static_cast<C2*>(p.x_out);
    const HT* __restrict__ val = static_cast<const HT*>(p.val);
    const VT* __restrict__ h0 = static_cast<const VT*>(p.h0);

    VT ca[RPT], cib[RPT], cb[RPT];
    double s1[RPT], s2[RPT], s3[RPT], s4[RPT];
#pragma unroll
    for (int t = 0; t < RPT; ++t) {
        const int r = q * RPT + t;
        const double a = p.scal[2 * r], b = p.scal[2 * r + 1];
        ca[t] = (VT)a;
        cb[t] = (VT)b;
        cib[t] = (VT)(1.0 / b);
        s1[t] = s2[t] = s3[t] = s4[t] = 0.0;
    }

    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t s = warp; s < p.nslices; s += nwarps) {
        const int64_t row = s * SH + sub;
        const int64_t base = p.slice_ptr[s];
        const int w = (int)((p.slice_ptr[s + 1] - base) / SH);
        C2 vo[RPT], xo[RPT], accV[RPT], accX[RPT];
        VecIO<VT, RPT>::load(vin + row * R + q * RPT, vo);
        VecIO<VT, RPT>::load(xin + row * R + q * RPT, xo);
        const VT d = h0[row];
#pragma unroll
        for (int t = 0; t < RPT; ++t) {
            accV[t].x = d * vo[t].x; accV[t].y = d * vo[t].y;
            accX[t].x = d * xo[t].x; accX[t].y = d * xo[t].y;
        }
        const int32_t* __restrict__ cp = p.col + base + sub;
        const HT* __restrict__ hp = val + base + sub;
#pragma unroll 4
        for (int k = 0; k < w; ++k) {
            const int32_t c = __ldcs(cp + (int64_t)k * SH);
            const HT h = Hop<VT, CPLX>::load(hp + (int64_t)k * SH);
            C2 vg[RPT], xg[RPT];
            VecIO<VT, RPT>::load(vin + (int64_t)c * R + q * RPT, vg);
            VecIO<VT, RPT>::load(xin + (int64_t)c * R + q * RPT, xg);
#pragma unroll
            for (int t = 0; t < RPT; ++t) {
                Hop<VT, CPLX>::msub(accV[t], h, vg[t]);
                Hop<VT, CPLX>::msub(accX[t], h, xg[t]);
            }
        }
        C2 vn[RPT], xk[RPT];
#pragma unroll
        for (int t = 0; t < RPT; ++t) {
            // x_k = (v - a x) / b ; y = H x_k = (Hv - a Hx) / b ; v_next = y - b x
            xk[t].x = (vo[t].x - ca[t] * xo[t].x) * cib[t];
            xk[t].y = (vo[t].y - ca[t] * xo[t].y) * cib[t];
            C2 y;
            y.x = (accV[t].x - ca[t] * accX[t].x) * cib[t];
            y.y = (accV[t].y - ca[t] * accX[t].y) * cib[t];
            vn[t].x = y.x - cb[t] * xo[t].x;
            vn[t].y = y.y - cb[t] * xo[t].y;
            const double xr = xk[t].x, xi = xk[t].y, yr = y.x, yi = y.y, vr = vn[t].x, vi = vn[t].y;
            s1[t] += xr * yr + xi * yi;
            s2[t] += vr * vr + vi * vi;
            s3[t] += xr * vr + xi * vi;
            s4[t] += xr * xr + xi * xi;
        }
        VecIO<VT, RPT>::store(vout + row * R + q * RPT, vn);
        VecIO<VT, RPT>::store(xout + row * R + q * RPT, xk);
    }

    // reduce over the rows of the warp (lanes with the same q)
#pragma unroll
    for (int t = 0; t < RPT; ++t) {
#pragma unroll
        for (int off = TPR; off < 32; off <<= 1) {
            s1[t] += __shfl_xor_sync(0xffffffffu, s1[t], off);
            s2[t] += __shfl_xor_sync(0xffffffffu, s2[t], off);
            s3[t] += __shfl_xor_sync(0xffffffffu, s3[t], off);
            s4[t] += __shfl_xor_sync(0xffffffffu, s4[t], off);
        }
    }
    __shared__ double red[8][R][4];
    const int wib = threadIdx.x >> 5;
    if (sub == 0) {
#pragma unroll
        for (int t = 0; t < RPT; ++t) {
            const int r = q * RPT + t;
            red[wib][r][0] = s1[t]; red[wib][r][1] = s2[t]; red[wib][r][2] = s3[t]; red[wib][r][3] = s4[t];
        }
    }
    __syncthreads();
    if (threadIdx.x < R * 4) {
        const int r = threadIdx.x >> 2, k = threadIdx.x & 3;
        double acc = 0.0;
        for (int wI = 0; wI < (int)(blockDim.x >> 5); ++wI) acc += red[wI][r][k];
        p.partials[((int64_t)blockIdx.x * R + r) * 4 + k] = acc;
    }
    // last block to finish reduces all blocks in a fixed order
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int prev = atomicAdd(p.counter, 1u);
        last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    __shared__ double tot[R][4];
    if (threadIdx.x < R * 4) {
        const int r = threadIdx.x >> 2, k = threadIdx.x & 3;
        double acc = 0.0;
        for (unsigned int bI = 0; bI < gridDim.x; ++bI) acc += __ldcg(&p.partials[((int64_t)bI * R + r) * 4 + k]);
        tot[r][k] = acc;
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

// ---------------------------------------------------------------------------- start vectors
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
static void split_rhs(int prec, int R, int* rpt, int* tpr)
{
    const int maxr = (prec == GBN_MIXED) ? 4 : 2;
    *rpt = R < maxr ? R : maxr;
    *tpr = R / *rpt;
}

int rows_per_slice(int prec, int nrhs)
{
    int rpt, tpr;
    split_rhs(prec, nrhs, &rpt, &tpr);
    return 32 / tpr;
}

using StepFn = void (*)(StepParams);

template <typename VT, bool CPLX>
static StepFn pick(int rpt, int tpr)
{
#define GBN_CASE(RP, TP) \
    if (rpt == RP && tpr == TP) return k_lanczos_step<VT, CPLX, RP, TP>;
    GBN_CASE(1, 1) GBN_CASE(2, 1)
    if constexpr (sizeof(VT) == 4) {
        GBN_CASE(4, 1) GBN_CASE(4, 2) GBN_CASE(4, 4) GBN_CASE(4, 8)
    } else {
        GBN_CASE(2, 2) GBN_CASE(2, 4) GBN_CASE(2, 8) GBN_CASE(2, 16)
    }
#undef GBN_CASE
    return nullptr;
}

static StepFn step_kernel(int prec, bool cplx, int R)
{
    int rpt, tpr;
    split_rhs(prec, R, &rpt, &tpr);
    if (prec == GBN_MIXED) return cplx ? pick<float, true>(rpt, tpr) : pick<float, false>(rpt, tpr);
    return cplx ? pick<double, true>(rpt, tpr) : pick<double, false>(rpt, tpr);
}

static int step_grid(gbn_ctx* c, StepFn fn)
{
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, 0) != cudaSuccess || per_sm < 1) per_sm = 1;
    return c->num_sms * per_sm;
}

int lanczos_prepare(gbn_ctx* c, int prec, int nrhs)
{
    if (nrhs != 1 && nrhs != 2 && nrhs != 4 && nrhs != 8 && nrhs != 16 && nrhs != 32)
        return fail(c, GBN_ERR_ARG, "internal: tile width must be 1, 2, 4, 8, 16 or 32");
    const int sh = rows_per_slice(prec, nrhs);
    if (!c->ell.valid || c->ell.prec != prec || c->ell.sh != sh) {
        const int rc = build_ell(c, prec, sh);
        if (rc) return rc;
    }
    c->prec = prec;
    c->nrhs = nrhs;
    const size_t esz = (prec == GBN_MIXED) ? sizeof(float2) : sizeof(double2);
    const size_t vbytes = (size_t)c->ell.npad * nrhs * esz;
    for (int i = 0; i < 4; ++i) GBN_CK(c, c->vec[i].ensure(vbytes));
    StepFn fn = step_kernel(prec, c->ell.cplx, nrhs);
    if (!fn) return fail(c, GBN_ERR_ARG, "no recursion kernel for this tile width");
    const int grid = step_grid(c, fn);
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
    StepFn fn = step_kernel(c->prec, c->ell.cplx, R);
    if (!fn) return fail(c, GBN_ERR_ARG, "no recursion kernel for this tile width");
    const int grid = step_grid(c, fn);
    StepParams p;
    p.slice_ptr = c->ell.slice_ptr.as<int64_t>();
    p.col = c->ell.col.as<int32_t>();
    p.val = c->ell.val.p;
    p.h0 = c->ell.h0.p;
    p.scal = c->scal.as<double>();
    p.partials = c->partials.as<double>();
    p.counter = c->counter.as<unsigned int>();
    p.a_out = c->ab.as<double>();
    p.b_out = c->ab.as<double>() + (size_t)R * nmax;
    p.nslices = c->ell.nslices;
    p.nmax = nmax;
    if (!c->ev0) {
        GBN_CK(c, cudaEventCreate(&c->ev0));
        GBN_CK(c, cudaEventCreate(&c->ev1));
    }
    GBN_CK(c, cudaEventRecord(c->ev0, c->stream));
    for (int32_t k = 0; k < nmax; ++k) {
        const int in = (k & 1) ? 2 : 0, out = (k & 1) ? 0 : 2;
        p.v_in = c->vec[in].p;
        p.x_in = c->vec[in + 1].p;
        p.v_out = c->vec[out].p;
        p.x_out = c->vec[out + 1].p;
        fn<<<grid, 256, 0, c->stream>>>(p);
        GBN_CK_LAUNCH(c);
    }
    GBN_CK(c, cudaEventRecord(c->ev1, c->stream));
    GBN_CK(c, cudaEventSynchronize(c->ev1));
    float ms = 0.f;
    GBN_CK(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->timing.step_ms = ms;
    c->timing.step_launches = nmax;
    unsigned int flags[3];
    GBN_CK(c, cudaMemcpyAsync(flags, c->counter.p, sizeof(flags), cudaMemcpyDeviceToHost, c->stream));
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    if (flags[2]) return fail(c, GBN_ERR_NUMERIC, "recursion produced a non-positive or non-finite b_n");
    return GBN_OK;
}

}  // namespace gbn
