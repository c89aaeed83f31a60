// Chebyshev time evolution (KuboChebyshevEvolve, lanczosKuboCode/Src/kubosubs.F90:557-619) on the
// grouped sliced ELL of the recursion.
//
// With x = (H - ac) / (2 bc) the reference propagates
//     psi_0 = sqrt(2) z,   psi_1 = x psi_0 (= (H - ac) psi_0 / (2 bc)),
//     psi_{n+1} = ((H - ac) psi_n - bc psi_{n-1}) / bc          (= 2 x psi_n - psi_{n-1})
// and returns z <- c_0 z + sum_{n >= 1} c_n psi_n, i.e. c_0 z + sqrt(2) sum c_n T_n(x) z.  One launch per
// polynomial: psi_n is gathered once per union column, psi_{n+1} overwrites psi_{n-1} in place (each
// row is read and written only by its own thread), and the accumulation into z is FP64 for both
// precisions.  Mixed precision keeps psi_n in complex FP32 with the step's arithmetic in FP64.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <vector>

#include "gbn_spmm.cuh"

namespace gbn {

struct ChebParams {
    const int64_t* slice_ptr;
    const unsigned char* mat;
    int64_t entry_bytes;
    const void* h0;
    const void* psi_n;   // gathered
    void* psi_out;       // psi_{n-1} on entry, psi_{n+1} on exit
    double2* z;          // [npad][R] FP64 accumulator
    double cr, ci;       // c_{n+1}
    double ac, alpha, beta;   // psi_{n+1} = (H psi_n - ac psi_n) * alpha - beta * psi_{n-1}
    int64_t nslices;
};

template <typename VT, bool CPLX, int G, int RPT, int TPR>
__global__ void __launch_bounds__(256) k_cheb_step(ChebParams p)
{
    using C2 = typename V2<VT>::t;
    using HT = typename Hop<VT, CPLX>::t;
    constexpr int GPW = 32 / TPR;
    constexpr int R = RPT * TPR;
    const int lane = threadIdx.x & 31;
    const int sub = lane / TPR;
    const int q = lane % TPR;
    const C2* __restrict__ xn = static_cast<const C2*>(p.psi_n);
    C2* __restrict__ xo = static_cast<C2*>(p.psi_out);
    const VT* __restrict__ h0 = static_cast<const VT*>(p.h0);
    const int nwb = (int)(blockDim.x >> 5);
    const int64_t per = (p.nslices + gridDim.x - 1) / gridDim.x;
    const int64_t s0 = (int64_t)blockIdx.x * per;
    const int64_t s1e = (s0 + per < p.nslices) ? s0 + per : p.nslices;
    for (int64_t s = s0 + (threadIdx.x >> 5); s < s1e; s += nwb) {
        const int64_t base = p.slice_ptr[s];
        const int w = (int)((p.slice_ptr[s + 1] - base) / GPW);
        const unsigned char* rec = p.mat + base * p.entry_bytes;
        C2 acc[G][RPT];
        group_columns<VT, CPLX, G, RPT, TPR, false>(xn, w, reinterpret_cast<const int32_t*>(rec) + sub,
                                                    reinterpret_cast<const HT*>(rec + (size_t)w * GPW * 4) + sub * G,
                                                    acc);
        const int64_t row0 = (s * GPW + sub) * G;
#pragma unroll
        for (int g = 0; g < G; ++g) {
            const int64_t e0 = (row0 + g) * R + q * RPT;
            C2 own[RPT], prev[RPT], nxt[RPT];
            VecIO<VT, RPT>::load(xn + e0, own);
#pragma unroll
            for (int t = 0; t < RPT; ++t) prev[t] = xo[e0 + t];   // read before the in-place write below
            const VT d = h0[row0 + g];
#pragma unroll
            for (int t = 0; t < RPT; ++t) {
                C2 y = acc[g][t];
                y.x = fma(d, own[t].x, y.x);
                y.y = fma(d, own[t].y, y.y);
                const double nr = ((double)y.x - p.ac * (double)own[t].x) * p.alpha - p.beta * (double)prev[t].x;
                const double ni = ((double)y.y - p.ac * (double)own[t].y) * p.alpha - p.beta * (double)prev[t].y;
                nxt[t].x = (VT)nr;
                nxt[t].y = (VT)ni;
                // z += c_{n+1} psi_{n+1}, with psi_{n+1} as stored (what the next step gathers)
                double2 zz = p.z[e0 + t];
                const double sr = (double)nxt[t].x, si = (double)nxt[t].y;
                zz.x += p.cr * sr - p.ci * si;
                zz.y += p.cr * si + p.ci * sr;
                p.z[e0 + t] = zz;
            }
            VecIO<VT, RPT>::store(xo + e0, nxt);
        }
    }
}

// psi_0 = sqrt(2) z, psi_{-1} = 0 (the first step reads it with weight 0) and z <- c_0 z, rows in the
// solver order; padding rows and vectors are zero
template <typename VT>
__global__ void k_cheb_start(typename V2<VT>::t* psi0, typename V2<VT>::t* psim1, double2* z, const double2* zin,
                             const int32_t* rperm, int64_t n, int64_t npad, int R, int nrhs_real, double c0r,
                             double c0i)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npad * R) return;
    const int64_t row = i / R;
    const int r = (int)(i % R);
    double2 v = make_double2(0.0, 0.0);
    if (row < n && r < nrhs_real) v = zin[(int64_t)r * n + rperm[row]];
    typename V2<VT>::t p0;
    p0.x = (VT)(1.4142135623730951 * v.x);
    p0.y = (VT)(1.4142135623730951 * v.y);
    psi0[i] = p0;
    p0.x = 0;
    p0.y = 0;
    psim1[i] = p0;
    z[i] = make_double2(c0r * v.x - c0i * v.y, c0r * v.y + c0i * v.x);
}

// z back to the reference atom order, [rhs][n]
__global__ void k_cheb_finish(const double2* z, double2* zout, const int32_t* rperm, int64_t n, int R, int nrhs_real)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * R) return;
    const int64_t row = i / R;
    const int r = (int)(i % R);
    if (r < nrhs_real) zout[(int64_t)r * n + rperm[row]] = z[i];
}

using ChebFn = void (*)(ChebParams);

template <typename VT, bool CPLX, int G>
static ChebFn pick_cheb_g(int rpt, int tpr)
{
#define GBN_CASE(RP, TP) \
    if (rpt == RP && tpr == TP) return k_cheb_step<VT, CPLX, G, RP, TP>;
    GBN_CASE(1, 1) GBN_CASE(1, 2) GBN_CASE(1, 4) GBN_CASE(1, 8) GBN_CASE(1, 16) GBN_CASE(1, 32)
    GBN_CASE(2, 1) GBN_CASE(2, 2) GBN_CASE(2, 4) GBN_CASE(2, 8) GBN_CASE(2, 16)
    if constexpr (sizeof(VT) == 4) {
        GBN_CASE(4, 1) GBN_CASE(4, 2) GBN_CASE(4, 4) GBN_CASE(4, 8)
    }
#undef GBN_CASE
    return nullptr;
}

template <typename VT, bool CPLX>
static ChebFn pick_cheb(int G, int rpt, int tpr)
{
    if (G == 1) return pick_cheb_g<VT, CPLX, 1>(rpt, tpr);
    if (G == 2) return pick_cheb_g<VT, CPLX, 2>(rpt, tpr);
    if (G == 4) return pick_cheb_g<VT, CPLX, 4>(rpt, tpr);
    return nullptr;
}

static int tile_width(int nrhs)
{
    int t = 1;
    while (t < nrhs && t < 32) t <<= 1;
    return t;
}

int cheb_evolve(gbn_ctx* c, int32_t prec, int32_t nrhs, const double* c_host, int32_t npol, double ac, double bc,
                double* z_host)
{
    if (!c->have_ham) return fail(c, GBN_ERR_STATE, "no Hamiltonian: call gbn_load_hamiltonian or gbn_assemble first");
    if (prec != GBN_FP64 && prec != GBN_MIXED) return fail(c, GBN_ERR_ARG, "precision must be GBN_FP64 or GBN_MIXED");
    if (nrhs < 1 || npol < 1 || !c_host || !z_host) return fail(c, GBN_ERR_ARG, "bad Chebyshev arguments");
    if (!(bc > 0.0) || !isfinite(bc) || !isfinite(ac)) return fail(c, GBN_ERR_ARG, "bc must be positive and finite");
    const int T = tile_width(nrhs);
    int rc = lanczos_prepare(c, prec, T);   // layout and vectors for a tile of T right-hand sides
    if (rc) return rc;
    int rpt, tpr;
    split_rhs(prec, T, c->tune_rpt, &rpt, &tpr);
    ChebFn fn;
    if (prec == GBN_MIXED) fn = c->ell.cplx ? pick_cheb<float, true>(c->ell.G, rpt, tpr)
                                            : pick_cheb<float, false>(c->ell.G, rpt, tpr);
    else fn = c->ell.cplx ? pick_cheb<double, true>(c->ell.G, rpt, tpr) : pick_cheb<double, false>(c->ell.G, rpt, tpr);
    if (!fn) return fail(c, GBN_ERR_ARG, "no Chebyshev kernel for this tile width");
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, 0) != cudaSuccess || per_sm < 1) per_sm = 1;
    const int grid = c->num_sms * per_sm;
    const int64_t n = c->n, npad = c->ell.npad;
    GBN_CK(c, c->cheb[0].ensure(sizeof(double2) * (size_t)npad * T));
    GBN_CK(c, c->cheb[1].ensure(sizeof(double2) * (size_t)n * T));
    c->staged = false;   // the recursion's staged start vectors were laid out for another tile
    double2* z = c->cheb[0].as<double2>();
    const int32_t* rp = c->ell.rperm.as<int32_t>();
    const int blk = 256;
    const unsigned sgrid = (unsigned)((npad * T + blk - 1) / blk);
    const unsigned fgrid = (unsigned)((n * T + blk - 1) / blk);
    int64_t launches = 0;
    float ms_total = 0.f;
    for (int r0 = 0; r0 < nrhs; r0 += T) {
        const int cnt = std::min(T, nrhs - r0);
        double2* zin = c->cheb[1].as<double2>();
        GBN_CK(c, cudaMemcpyAsync(zin, z_host + (size_t)2 * n * r0, sizeof(double2) * (size_t)n * cnt,
                                  cudaMemcpyHostToDevice, c->stream));
        void* bufA = c->vec[1].p;   // psi_n
        void* bufB = c->vec[2].p;   // psi_{n-1}, then psi_{n+1}
        if (prec == GBN_MIXED)
            k_cheb_start<float><<<sgrid, blk, 0, c->stream>>>(static_cast<float2*>(bufA), static_cast<float2*>(bufB), z,
                                                               zin, rp, n, npad, T, cnt, c_host[0], c_host[1]);
        else
            k_cheb_start<double><<<sgrid, blk, 0, c->stream>>>(static_cast<double2*>(bufA), static_cast<double2*>(bufB),
                                                                z, zin, rp, n, npad, T, cnt, c_host[0], c_host[1]);
        GBN_CK_LAUNCH(c);
        if (!c->ev0) {
            GBN_CK(c, cudaEventCreate(&c->ev0));
            GBN_CK(c, cudaEventCreate(&c->ev1));
        }
        GBN_CK(c, cudaEventRecord(c->ev0, c->stream));
        ChebParams p;
        p.slice_ptr = c->ell.slice_ptr.as<int64_t>();
        p.mat = c->ell.mat.as<unsigned char>();
        p.entry_bytes = c->ell.entry_bytes;
        p.h0 = c->ell.h0.p;
        p.z = z;
        p.ac = ac;
        p.nslices = c->ell.nslices;
        for (int k = 1; k < npol; ++k) {
            p.psi_n = bufA;
            p.psi_out = bufB;
            p.cr = c_host[2 * k];
            p.ci = c_host[2 * k + 1];
            p.alpha = (k == 1) ? 1.0 / (2.0 * bc) : 1.0 / bc;
            p.beta = (k == 1) ? 0.0 : 1.0;
            fn<<<grid, 256, 0, c->stream>>>(p);
            GBN_CK_LAUNCH(c);
            std::swap(bufA, bufB);
            ++launches;
        }
        GBN_CK(c, cudaEventRecord(c->ev1, c->stream));
        k_cheb_finish<<<fgrid, blk, 0, c->stream>>>(z, zin, rp, n, T, cnt);
        GBN_CK_LAUNCH(c);
        GBN_CK(c, cudaMemcpyAsync(z_host + (size_t)2 * n * r0, zin, sizeof(double2) * (size_t)n * cnt,
                                  cudaMemcpyDeviceToHost, c->stream));
        GBN_CK(c, cudaStreamSynchronize(c->stream));
        float ms = 0.f;
        GBN_CK(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
        ms_total += ms;
    }
    c->timing.step_ms = ms_total;
    c->timing.step_launches = launches;
    return GBN_OK;
}

int kubo_evol(gbn_ctx* c, int32_t, const double*, int32_t, double, double, int32_t, double*, double*)
{
    return fail(c, GBN_ERR_STATE, "Kubo time evolution is not built yet");
}

}  // namespace gbn
