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
    double cpr, cpi;     // c_n, when its term is added here (acc 2)
    int32_t acc;         // accumulator update: 0 none (deferred), 1 z += c_{n+1} psi_{n+1}, 2 z += c_n psi_n first
};

// z += c psi with psi as stored; both the deferred and the direct terms go through this one expression
__device__ __forceinline__ void acc_add(double2& z, double cr, double ci, double sr, double si)
{
    z.x += cr * sr - ci * si;
    z.y += cr * si + ci * sr;
}

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
        group_columns<VT, CPLX, G, RPT, TPR, false>(xn, w, reinterpret_cast<const int32_t*>(rec) + sub * kColUnroll,
                                                    reinterpret_cast<const HT*>(rec + (size_t)w * GPW * 4) +
                                                        val_thread_off<HT, G, TPR, 1>(sub, q),
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
                // z += c_{n+1} psi_{n+1}, with psi_{n+1} as stored (what the next step gathers); every
                // second step also adds the deferred c_n psi_n (psi_n is this row's own, loaded above),
                // in the same order, so the accumulator is read and written on every other step only
                if (p.acc != 0) {
                    double2 zz = p.z[e0 + t];
                    if (p.acc == 2) acc_add(zz, p.cpr, p.cpi, (double)own[t].x, (double)own[t].y);
                    acc_add(zz, p.cr, p.ci, (double)nxt[t].x, (double)nxt[t].y);
                    p.z[e0 + t] = zz;
                }
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

// Accumulator schedule of polynomial step k (1 .. npol-1, the step that forms psi_k): the term of an odd
// k is deferred to step k + 1, which adds c_k psi_k (its own row) before c_{k+1} psi_{k+1}; the last step
// adds its own term.
template <typename P>
static void set_acc(P& p, const double* c_host, int k, int npol)
{
    const bool last = k == npol - 1;
    if (k % 2 == 1 && !last) {
        p.acc = 0;
    } else if (k % 2 == 0) {
        p.acc = 2;
        p.cpr = c_host[2 * (k - 1)];
        p.cpi = c_host[2 * (k - 1) + 1];
    } else {
        p.acc = 1;
    }
}

// One tile of the Chebyshev propagation z <- U z: zin (device, [cnt][n] complex128, reference order) in
// and out; c->cheb[0] holds the accumulator, c->vec[1], c->vec[2] the recurrence.  *ms: device time of
// the polynomial loop.
static int cheb_tile(gbn_ctx* c, int prec, ChebFn fn, int grid, int T, int cnt, const double* c_host, int npol,
                     double ac, double bc, double2* zin, int64_t* launches, float* ms)
{
    const int64_t n = c->n, npad = c->ell.npad;
    double2* z = c->cheb[0].as<double2>();
    const int32_t* rp = c->ell.rperm.as<int32_t>();
    const int blk = 256;
    const unsigned sgrid = (unsigned)((npad * T + blk - 1) / blk);
    const unsigned fgrid = (unsigned)((n * T + blk - 1) / blk);
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
        set_acc(p, c_host, k, npol);
        fn<<<grid, 256, 0, c->stream>>>(p);
        GBN_CK_LAUNCH(c);
        std::swap(bufA, bufB);
        ++*launches;
    }
    GBN_CK(c, cudaEventRecord(c->ev1, c->stream));
    k_cheb_finish<<<fgrid, blk, 0, c->stream>>>(z, zin, rp, n, T, cnt);
    GBN_CK_LAUNCH(c);
    GBN_CK(c, cudaEventSynchronize(c->ev1));
    GBN_CK(c, cudaEventElapsedTime(ms, c->ev0, c->ev1));
    return GBN_OK;
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
    int64_t launches = 0;
    float ms_total = 0.f;
    for (int r0 = 0; r0 < nrhs; r0 += T) {
        const int cnt = std::min(T, nrhs - r0);
        double2* zin = c->cheb[1].as<double2>();
        GBN_CK(c, cudaMemcpyAsync(zin, z_host + (size_t)2 * n * r0, sizeof(double2) * (size_t)n * cnt,
                                  cudaMemcpyHostToDevice, c->stream));
        float ms = 0.f;
        rc = cheb_tile(c, prec, fn, grid, T, cnt, c_host, npol, ac, bc, zin, &launches, &ms);
        if (rc) return rc;
        GBN_CK(c, cudaMemcpyAsync(z_host + (size_t)2 * n * r0, zin, sizeof(double2) * (size_t)n * cnt,
                                  cudaMemcpyDeviceToHost, c->stream));
        GBN_CK(c, cudaStreamSynchronize(c->stream));
        ms_total += ms;
    }
    c->timing.step_ms = ms_total;
    c->timing.step_launches = launches;
    return GBN_OK;
}

// ---------------------------------------------------------------------------- KuboEvol
// KuboEvol (kubosubs.F90:438-553): psi <- U psi and zupsi <- U zupsi + [U, X] psi, U the Chebyshev
// propagator above and X the position along dir.  The commutator term runs a second recurrence beside
// psi_n:
//     X_0 = 0,  X_{n+1} = ((H - ac) X_n + D psi_n) * alpha - beta X_{n-1},   D = d (*) H off-diagonal,
// d the NeighD component (the neighbour's displacement) of each entry; zupsi accumulates c_n X_n.
// D is stored as a second value array with the indexing of the layout's values (built once per
// direction), so a union column's d * val sits beside its val.

template <typename HV>
__device__ __forceinline__ HV scaled_neg_hop(double2 h, double d);
template <> __device__ __forceinline__ float scaled_neg_hop<float>(double2 h, double d) { return (float)(-d * h.x); }
template <> __device__ __forceinline__ double scaled_neg_hop<double>(double2 h, double d) { return -d * h.x; }
template <> __device__ __forceinline__ float2 scaled_neg_hop<float2>(double2 h, double d)
{
    return make_float2((float)(-d * h.x), (float)(-d * h.y));
}
template <> __device__ __forceinline__ double2 scaled_neg_hop<double2>(double2 h, double d)
{
    return make_double2(-d * h.x, -d * h.y);
}
__device__ __forceinline__ void acc_into(float& a, float b) { a += b; }
__device__ __forceinline__ void acc_into(double& a, double b) { a += b; }
__device__ __forceinline__ void acc_into(float2& a, float2 b) { a.x += b.x; a.y += b.y; }
__device__ __forceinline__ void acc_into(double2& a, double2 b) { a.x += b.x; a.y += b.y; }

// One thread per group: every entry of the group's rows finds its union column in the slice record
// (first match among the stored columns) and adds -d * hopp there.  dval must be zeroed.
template <typename HV>
__global__ void k_fill_dvals(const int32_t* nneigh, const int32_t* nlist, const double2* hopp, const double* neighd,
                             int comp, const int32_t* rperm, const int32_t* riperm, int64_t n, int32_t max_neigh,
                             int G, int gpw, int64_t nslices, const int64_t* slice_ptr, const unsigned char* mat,
                             int64_t entry_bytes, HV* dval)
{
    const int64_t ng = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (ng >= nslices * gpw) return;
    const int64_t s = ng / gpw;
    const int j = (int)(ng % gpw);
    const int64_t base = slice_ptr[s];
    const int w = (int)((slice_ptr[s + 1] - base) / gpw);
    const int32_t* col = reinterpret_cast<const int32_t*>(mat + base * entry_bytes);
    for (int rr = 0; rr < G; ++rr) {
        const int64_t row = ng * G + rr;
        if (row >= n) break;
        const int64_t p = rperm[row];
        for (int e = 0; e < nneigh[p]; ++e) {
            const int64_t ent = p * max_neigh + e;
            const int32_t target = riperm[nlist[ent] - 1];
            int k = 0;
            while (k < w && col[rec_slot(k, j, gpw)] != target) ++k;
            if (k == w) continue;   // cannot happen: every entry's column is in its group's union
            acc_into(dval[base * G + val_slot(k, j, gpw, G, (int)sizeof(HV)) + rr], scaled_neg_hop<HV>(hopp[ent], neighd[3 * ent + comp]));
        }
    }
}

struct DualParams {
    const int64_t* slice_ptr;
    const unsigned char* mat;
    const void* dval;
    int64_t entry_bytes;
    const void* h0;
    const void* psi_n;   // gathered
    const void* x_n;     // gathered
    void* psi_out;       // psi_{n-1} in, psi_{n+1} out
    void* x_out;         // X_{n-1} in, X_{n+1} out
    double2* pacc;       // psi accumulator (FP64)
    double2* zacc;       // zupsi accumulator (FP64)
    double cr, ci, ac, alpha, beta;
    int64_t nslices;
    double cpr, cpi;     // c_n, when its terms are added here (acc 2)
    int32_t acc;         // as in ChebParams
};

template <typename VT, bool CPLX, int G, int RPT, int TPR>
__global__ void __launch_bounds__(256) k_dual_step(DualParams p)
{
    using C2 = typename V2<VT>::t;
    using HT = typename Hop<VT, CPLX>::t;
    constexpr int GPW = 32 / TPR;
    constexpr int R = RPT * TPR;
    constexpr int U = kColUnroll;
    const int lane = threadIdx.x & 31;
    const int sub = lane / TPR;
    const int q = lane % TPR;
    const C2* __restrict__ pn = static_cast<const C2*>(p.psi_n);
    const C2* __restrict__ xn = static_cast<const C2*>(p.x_n);
    C2* __restrict__ po = static_cast<C2*>(p.psi_out);
    C2* __restrict__ xo = static_cast<C2*>(p.x_out);
    const VT* __restrict__ h0 = static_cast<const VT*>(p.h0);
    const HT* __restrict__ dv = static_cast<const HT*>(p.dval);
    const int nwb = (int)(blockDim.x >> 5);
    const int64_t per = (p.nslices + gridDim.x - 1) / gridDim.x;
    const int64_t s0 = (int64_t)blockIdx.x * per;
    const int64_t s1e = (s0 + per < p.nslices) ? s0 + per : p.nslices;
    for (int64_t s = s0 + (threadIdx.x >> 5); s < s1e; s += nwb) {
        const int64_t base = p.slice_ptr[s];
        const int w = (int)((p.slice_ptr[s + 1] - base) / GPW);
        const unsigned char* rec = p.mat + base * p.entry_bytes;
        const int32_t* __restrict__ cp = reinterpret_cast<const int32_t*>(rec) + sub * U;
        const HT* __restrict__ vp = reinterpret_cast<const HT*>(rec + (size_t)w * GPW * 4) + val_thread_off<HT, G, TPR, 1>(sub, q);
        const HT* __restrict__ dp = dv + base * G + val_thread_off<HT, G, TPR, 1>(sub, q);
        C2 ap[G][RPT], ax[G][RPT];
#pragma unroll
        for (int g = 0; g < G; ++g)
#pragma unroll
            for (int t = 0; t < RPT; ++t) {
                ap[g][t].x = 0; ap[g][t].y = 0;
                ax[g][t].x = 0; ax[g][t].y = 0;
            }
        static_assert(U == 4, "one 16-byte load of a block's indices");
        for (int k = 0; k < w; k += U) {
            const int4 cb = __ldcs(reinterpret_cast<const int4*>(cp));   // the group's U columns of this block
            const int32_t cc[U] = {cb.x, cb.y, cb.z, cb.w};
            HT hb[U][G], hdb[U][G];
            load_block_vals<HT, G, GPW, U, false, 1>(vp, hb);
            load_block_vals<HT, G, GPW, U, false, 1>(dp, hdb);
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int32_t c = cc[u];
                const HT* h = hb[u];
                const HT* hd = hdb[u];
                C2 gp[RPT], gx[RPT];
                VecIO<VT, RPT>::load(pn + (size_t)(uint32_t)c * R + q * RPT, gp);
                VecIO<VT, RPT>::load(xn + (size_t)(uint32_t)c * R + q * RPT, gx);
#pragma unroll
                for (int g = 0; g < G; ++g)
#pragma unroll
                    for (int t = 0; t < RPT; ++t) {
                        Hop<VT, CPLX>::madd(ap[g][t], h[g], gp[t]);
                        Hop<VT, CPLX>::madd(ax[g][t], h[g], gx[t]);
                        Hop<VT, CPLX>::madd(ax[g][t], hd[g], gp[t]);
                    }
            }
            cp += U * GPW;
            vp += U * GPW * G;
            dp += U * GPW * G;
        }
        const int64_t row0 = (s * GPW + sub) * G;
#pragma unroll
        for (int g = 0; g < G; ++g) {
            const int64_t e0 = (row0 + g) * R + q * RPT;
            C2 ownp[RPT], ownx[RPT], prevp[RPT], prevx[RPT], np[RPT], nx[RPT];
            VecIO<VT, RPT>::load(pn + e0, ownp);
            VecIO<VT, RPT>::load(xn + e0, ownx);
#pragma unroll
            for (int t = 0; t < RPT; ++t) {   // read before the in-place writes below
                prevp[t] = po[e0 + t];
                prevx[t] = xo[e0 + t];
            }
            const VT d = h0[row0 + g];
#pragma unroll
            for (int t = 0; t < RPT; ++t) {
                C2 yp = ap[g][t], yx = ax[g][t];
                yp.x = fma(d, ownp[t].x, yp.x);
                yp.y = fma(d, ownp[t].y, yp.y);
                yx.x = fma(d, ownx[t].x, yx.x);
                yx.y = fma(d, ownx[t].y, yx.y);
                np[t].x = (VT)(((double)yp.x - p.ac * (double)ownp[t].x) * p.alpha - p.beta * (double)prevp[t].x);
                np[t].y = (VT)(((double)yp.y - p.ac * (double)ownp[t].y) * p.alpha - p.beta * (double)prevp[t].y);
                nx[t].x = (VT)(((double)yx.x - p.ac * (double)ownx[t].x) * p.alpha - p.beta * (double)prevx[t].x);
                nx[t].y = (VT)(((double)yx.y - p.ac * (double)ownx[t].y) * p.alpha - p.beta * (double)prevx[t].y);
                if (p.acc != 0) {   // the accumulators on every other step (see k_cheb_step)
                    double2 a1 = p.pacc[e0 + t], a2 = p.zacc[e0 + t];
                    if (p.acc == 2) {
                        acc_add(a1, p.cpr, p.cpi, (double)ownp[t].x, (double)ownp[t].y);
                        acc_add(a2, p.cpr, p.cpi, (double)ownx[t].x, (double)ownx[t].y);
                    }
                    acc_add(a1, p.cr, p.ci, (double)np[t].x, (double)np[t].y);
                    acc_add(a2, p.cr, p.ci, (double)nx[t].x, (double)nx[t].y);
                    p.pacc[e0 + t] = a1;
                    p.zacc[e0 + t] = a2;
                }
            }
            VecIO<VT, RPT>::store(po + e0, np);
            VecIO<VT, RPT>::store(xo + e0, nx);
        }
    }
}

// psi_0 = sqrt(2) psi, psi_{-1} = X_0 = X_{-1} = 0, pacc = c_0 psi, zacc = zupsi (already U zupsi)
template <typename VT>
__global__ void k_dual_start(typename V2<VT>::t* p0, typename V2<VT>::t* pm1, typename V2<VT>::t* x0,
                             typename V2<VT>::t* xm1, double2* pacc, double2* zacc, const double2* psi_in,
                             const double2* zu_in, const int32_t* rperm, int64_t n, int64_t npad, int R, int nrhs_real,
                             double c0r, double c0i)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npad * R) return;
    const int64_t row = i / R;
    const int r = (int)(i % R);
    double2 v = make_double2(0.0, 0.0), zu = make_double2(0.0, 0.0);
    if (row < n && r < nrhs_real) {
        v = psi_in[(int64_t)r * n + rperm[row]];
        zu = zu_in[(int64_t)r * n + rperm[row]];
    }
    typename V2<VT>::t a, zero;
    a.x = (VT)(1.4142135623730951 * v.x);
    a.y = (VT)(1.4142135623730951 * v.y);
    zero.x = 0;
    zero.y = 0;
    p0[i] = a;
    pm1[i] = zero;
    x0[i] = zero;
    xm1[i] = zero;
    pacc[i] = make_double2(c0r * v.x - c0i * v.y, c0r * v.y + c0i * v.x);
    zacc[i] = zu;
}

using DualFn = void (*)(DualParams);

template <typename VT, bool CPLX, int G>
static DualFn pick_dual_g(int rpt, int tpr)
{
#define GBN_CASE(RP, TP) \
    if (rpt == RP && tpr == TP) return k_dual_step<VT, CPLX, G, RP, TP>;
    GBN_CASE(1, 1) GBN_CASE(1, 2) GBN_CASE(1, 4) GBN_CASE(1, 8) GBN_CASE(1, 16) GBN_CASE(1, 32)
    GBN_CASE(2, 1) GBN_CASE(2, 2) GBN_CASE(2, 4) GBN_CASE(2, 8) GBN_CASE(2, 16)
    if constexpr (sizeof(VT) == 4) {
        GBN_CASE(4, 1) GBN_CASE(4, 2) GBN_CASE(4, 4) GBN_CASE(4, 8)
    }
#undef GBN_CASE
    return nullptr;
}

template <typename VT, bool CPLX>
static DualFn pick_dual(int G, int rpt, int tpr)
{
    if (G == 1) return pick_dual_g<VT, CPLX, 1>(rpt, tpr);
    if (G == 2) return pick_dual_g<VT, CPLX, 2>(rpt, tpr);
    if (G == 4) return pick_dual_g<VT, CPLX, 4>(rpt, tpr);
    return nullptr;
}

static int build_dvals(gbn_ctx* c, int dir)
{
    Ell& E = c->ell;
    if (E.dval_dir == dir) return GBN_OK;
    const size_t bytes = (size_t)E.val_size * E.G * (size_t)(E.nnz_stored > 0 ? E.nnz_stored : 1);
    GBN_CK(c, E.dval.ensure(bytes));
    GBN_CK(c, cudaMemsetAsync(E.dval.p, 0, bytes, c->stream));
    const unsigned grd = (unsigned)((E.nslices * E.gpw + 127) / 128);
#define GBN_DV(HV)                                                                                                  \
    k_fill_dvals<HV><<<grd, 128, 0, c->stream>>>(c->nneigh.as<int32_t>(), c->nlist.as<int32_t>(), c->hopp.as<double2>(), \
                                                 c->neighd.as<double>(), dir - 1, E.rperm.as<int32_t>(),                 \
                                                 E.riperm.as<int32_t>(), c->n, c->max_neigh, E.G, E.gpw, E.nslices,        \
                                                 E.slice_ptr.as<int64_t>(), E.mat.as<unsigned char>(), E.entry_bytes,     \
                                                 E.dval.as<HV>())
    if (E.prec == GBN_MIXED) {
        if (E.cplx) GBN_DV(float2);
        else GBN_DV(float);
    } else {
        if (E.cplx) GBN_DV(double2);
        else GBN_DV(double);
    }
#undef GBN_DV
    GBN_CK_LAUNCH(c);
    E.dval_dir = dir;
    return GBN_OK;
}

// One tile of KuboEvol's dual recurrence: pin, zin (device, [cnt][n] complex128, reference order) hold psi
// and zupsi (already propagated by U) in and psi <- U psi, zupsi <- zupsi + [U, X] psi out.
static int dual_tile(gbn_ctx* c, int prec, DualFn fn, int grid, int T, int cnt, const double* c_host, int npol,
                     double ac, double bc, double2* pin, double2* zin, int64_t* launches)
{
    const int64_t n = c->n, npad = c->ell.npad;
    double2* pacc = c->cheb[0].as<double2>();
    double2* zacc = c->cheb[2].as<double2>();
    const int32_t* rp = c->ell.rperm.as<int32_t>();
    const int blk = 256;
    const unsigned sgrid = (unsigned)((npad * T + blk - 1) / blk);
    const unsigned fgrid = (unsigned)((n * T + blk - 1) / blk);
    void* pA = c->vec[1].p;
    void* pB = c->vec[2].p;
    void* xA = c->cheb[3].p;
    void* xB = c->cheb[4].p;
    if (prec == GBN_MIXED)
        k_dual_start<float><<<sgrid, blk, 0, c->stream>>>(static_cast<float2*>(pA), static_cast<float2*>(pB),
                                                           static_cast<float2*>(xA), static_cast<float2*>(xB), pacc,
                                                           zacc, pin, zin, rp, n, npad, T, cnt, c_host[0], c_host[1]);
    else
        k_dual_start<double><<<sgrid, blk, 0, c->stream>>>(static_cast<double2*>(pA), static_cast<double2*>(pB),
                                                            static_cast<double2*>(xA), static_cast<double2*>(xB), pacc,
                                                            zacc, pin, zin, rp, n, npad, T, cnt, c_host[0], c_host[1]);
    GBN_CK_LAUNCH(c);
    DualParams p;
    p.slice_ptr = c->ell.slice_ptr.as<int64_t>();
    p.mat = c->ell.mat.as<unsigned char>();
    p.dval = c->ell.dval.p;
    p.entry_bytes = c->ell.entry_bytes;
    p.h0 = c->ell.h0.p;
    p.pacc = pacc;
    p.zacc = zacc;
    p.ac = ac;
    p.nslices = c->ell.nslices;
    for (int k = 1; k < npol; ++k) {
        p.psi_n = pA;
        p.x_n = xA;
        p.psi_out = pB;
        p.x_out = xB;
        p.cr = c_host[2 * k];
        p.ci = c_host[2 * k + 1];
        p.alpha = (k == 1) ? 1.0 / (2.0 * bc) : 1.0 / bc;
        p.beta = (k == 1) ? 0.0 : 1.0;
        set_acc(p, c_host, k, npol);
        fn<<<grid, 256, 0, c->stream>>>(p);
        GBN_CK_LAUNCH(c);
        std::swap(pA, pB);
        std::swap(xA, xB);
        ++*launches;
    }
    k_cheb_finish<<<fgrid, blk, 0, c->stream>>>(pacc, pin, rp, n, T, cnt);
    GBN_CK_LAUNCH(c);
    k_cheb_finish<<<fgrid, blk, 0, c->stream>>>(zacc, zin, rp, n, T, cnt);
    GBN_CK_LAUNCH(c);
    return GBN_OK;
}

// Kernels and buffers of KuboEvol for a tile of T right-hand sides (after cheb_evolve's preparation).
static int dual_prepare(gbn_ctx* c, int prec, int T, int dir, DualFn* fn, int* grid)
{
    int rpt, tpr;
    split_rhs(prec, T, c->tune_rpt, &rpt, &tpr);
    int rc = build_dvals(c, dir);
    if (rc) return rc;
    if (prec == GBN_MIXED) *fn = c->ell.cplx ? pick_dual<float, true>(c->ell.G, rpt, tpr)
                                             : pick_dual<float, false>(c->ell.G, rpt, tpr);
    else *fn = c->ell.cplx ? pick_dual<double, true>(c->ell.G, rpt, tpr) : pick_dual<double, false>(c->ell.G, rpt, tpr);
    if (!*fn) return fail(c, GBN_ERR_ARG, "no KuboEvol kernel for this tile width");
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, *fn, 256, 0) != cudaSuccess || per_sm < 1) per_sm = 1;
    *grid = c->num_sms * per_sm;
    const int64_t npad = c->ell.npad;
    const size_t esz = (prec == GBN_MIXED) ? sizeof(float2) : sizeof(double2);
    GBN_CK(c, c->cheb[0].ensure(sizeof(double2) * (size_t)npad * T));   // psi accumulator (Z of U as well)
    GBN_CK(c, c->cheb[2].ensure(sizeof(double2) * (size_t)npad * T));   // zupsi accumulator
    GBN_CK(c, c->cheb[3].ensure(esz * (size_t)npad * T));              // X_n
    GBN_CK(c, c->cheb[4].ensure(esz * (size_t)npad * T));              // X_{n-1}
    return GBN_OK;
}

int kubo_evol(gbn_ctx* c, int32_t prec, int32_t nrhs, const double* c_host, int32_t npol, double ac, double bc,
              int32_t dir, double* psi_host, double* zupsi_host)
{
    if (!c->have_neighd) return fail(c, GBN_ERR_STATE, "KuboEvol needs NeighD (gbn_neighbours or gbn_set_neighd)");
    if (dir != 1 && dir != 2) return fail(c, GBN_ERR_ARG, "dir must be 1 (x) or 2 (y)");
    // zupsi <- U zupsi (the reference's first call of KuboChebyshevEvolve)
    int rc = cheb_evolve(c, prec, nrhs, c_host, npol, ac, bc, zupsi_host);
    if (rc) return rc;
    const int T = tile_width(nrhs);   // the layout cheb_evolve prepared
    DualFn fn;
    int grid;
    rc = dual_prepare(c, prec, T, dir, &fn, &grid);
    if (rc) return rc;
    const int64_t n = c->n;
    GBN_CK(c, c->cheb[1].ensure(sizeof(double2) * (size_t)n * T));     // psi in / out
    GBN_CK(c, c->cheb[5].ensure(sizeof(double2) * (size_t)n * T));     // zupsi in / out
    double2* pin = c->cheb[1].as<double2>();
    double2* zin = c->cheb[5].as<double2>();
    int64_t launches = 0;
    for (int r0 = 0; r0 < nrhs; r0 += T) {
        const int cnt = std::min(T, nrhs - r0);
        GBN_CK(c, cudaMemcpyAsync(pin, psi_host + (size_t)2 * n * r0, sizeof(double2) * (size_t)n * cnt,
                                  cudaMemcpyHostToDevice, c->stream));
        GBN_CK(c, cudaMemcpyAsync(zin, zupsi_host + (size_t)2 * n * r0, sizeof(double2) * (size_t)n * cnt,
                                  cudaMemcpyHostToDevice, c->stream));
        rc = dual_tile(c, prec, fn, grid, T, cnt, c_host, npol, ac, bc, pin, zin, &launches);
        if (rc) return rc;
        GBN_CK(c, cudaMemcpyAsync(psi_host + (size_t)2 * n * r0, pin, sizeof(double2) * (size_t)n * cnt,
                                  cudaMemcpyDeviceToHost, c->stream));
        GBN_CK(c, cudaMemcpyAsync(zupsi_host + (size_t)2 * n * r0, zin, sizeof(double2) * (size_t)n * cnt,
                                  cudaMemcpyDeviceToHost, c->stream));
        GBN_CK(c, cudaStreamSynchronize(c->stream));
    }
    return GBN_OK;
}

// |z_r|^2 of a [cnt][n] complex128 block: per-block partial sums (fixed order), then their sum per r
__global__ void k_norm_parts(const double2* z, int64_t n, int cnt, int parts, double* out)
{
    const int r = blockIdx.x / parts, part = blockIdx.x % parts;
    if (r >= cnt) return;
    const int64_t per = (n + parts - 1) / parts, lo = part * per, hi = (lo + per < n) ? lo + per : n;
    double s = 0.0;
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const double2 v = z[(int64_t)r * n + i];
        s += v.x * v.x + v.y * v.y;
    }
    __shared__ double sh[256];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[(int64_t)r * parts + part] = sh[0];
}

__global__ void k_norm_sum(const double* parts_in, int parts, int cnt, double* norm)
{
    const int r = threadIdx.x;
    if (r >= cnt) return;
    double s = 0.0;
    for (int k = 0; k < parts; ++k) s += parts_in[(int64_t)r * parts + k];
    norm[r] = s;
}

// out_r = z_r / sqrt(norm_r) (the normalised ZUPsi of KuboTEvol), in [cnt][n] layout
__global__ void k_normalise(const double2* z, const double* norm, int64_t n, int cnt, double2* out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * cnt) return;
    const int r = (int)(i / n);
    const double s = sqrt(fabs(norm[r]));
    out[i] = make_double2(z[i].x / s, z[i].y / s);
}

// KuboTEvol (kubo.F90:321-397) with psi and zupsi resident on the device: nt steps of KuboEvol; after every
// nwr-th step the norm |zupsi|^2 and the recursion of zupsi / |zupsi| (nrecurs steps).  psi and zupsi
// are read at the start and written back at the end; norms [nrhs][nt/nwr], a, b [nrhs][nt/nwr][nrecurs].
int kubo_tevol(gbn_ctx* c, int32_t prec, int32_t nrhs, const double* c_host, int32_t npol, double ac, double bc,
               int32_t dir, int32_t nt, int32_t nwr, int32_t nrecurs, double* psi_host, double* zupsi_host,
               double* norms, double* a_out, double* b_out)
{
    if (!c->have_neighd) return fail(c, GBN_ERR_STATE, "KuboEvol needs NeighD (gbn_neighbours or gbn_set_neighd)");
    if (dir != 1 && dir != 2) return fail(c, GBN_ERR_ARG, "dir must be 1 (x) or 2 (y)");
    const int T = tile_width(nrhs);
    int rc = lanczos_prepare(c, prec, T);
    if (rc) return rc;
    c->staged = false;
    int rpt, tpr;
    split_rhs(prec, T, c->tune_rpt, &rpt, &tpr);
    ChebFn cfn;
    if (prec == GBN_MIXED) cfn = c->ell.cplx ? pick_cheb<float, true>(c->ell.G, rpt, tpr)
                                             : pick_cheb<float, false>(c->ell.G, rpt, tpr);
    else cfn = c->ell.cplx ? pick_cheb<double, true>(c->ell.G, rpt, tpr) : pick_cheb<double, false>(c->ell.G, rpt, tpr);
    if (!cfn) return fail(c, GBN_ERR_ARG, "no Chebyshev kernel for this tile width");
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cfn, 256, 0) != cudaSuccess || per_sm < 1) per_sm = 1;
    const int cgrid = c->num_sms * per_sm;
    DualFn dfn;
    int dgrid;
    rc = dual_prepare(c, prec, T, dir, &dfn, &dgrid);
    if (rc) return rc;
    const int64_t n = c->n;
    const int nw = nt / nwr;
    const int parts = 256;
    GBN_CK(c, c->cheb[6].ensure(sizeof(double2) * (size_t)n * T));   // psi state
    GBN_CK(c, c->cheb[7].ensure(sizeof(double2) * (size_t)n * T));   // zupsi state
    GBN_CK(c, c->upload.ensure(sizeof(double2) * (size_t)n * T));    // normalised zupsi
    DevBuf part_buf, norm_buf;
    GBN_CK(c, part_buf.ensure(sizeof(double) * (size_t)T * parts));
    GBN_CK(c, norm_buf.ensure(sizeof(double) * (size_t)T));
    double2* pin = c->cheb[6].as<double2>();
    double2* zin = c->cheb[7].as<double2>();
    std::vector<double> hn((size_t)T), hab;
    int64_t launches = 0;
    double loop_ms = 0.0;
    for (int r0 = 0; r0 < nrhs; r0 += T) {
        const int cnt = std::min(T, nrhs - r0);
        GBN_CK(c, cudaMemcpyAsync(pin, psi_host + (size_t)2 * n * r0, sizeof(double2) * (size_t)n * cnt,
                                  cudaMemcpyHostToDevice, c->stream));
        GBN_CK(c, cudaMemcpyAsync(zin, zupsi_host + (size_t)2 * n * r0, sizeof(double2) * (size_t)n * cnt,
                                  cudaMemcpyHostToDevice, c->stream));
        int w = 0;
        for (int it = 1; it <= nt; ++it) {
            float ms = 0.f;
            rc = cheb_tile(c, prec, cfn, cgrid, T, cnt, c_host, npol, ac, bc, zin, &launches, &ms);   // zupsi <- U zupsi
            if (rc) return rc;
            rc = dual_tile(c, prec, dfn, dgrid, T, cnt, c_host, npol, ac, bc, pin, zin, &launches);
            if (rc) return rc;
            if (it % nwr != 0 || w >= nw) continue;
            k_norm_parts<<<(unsigned)(cnt * parts), 256, 0, c->stream>>>(zin, n, cnt, parts, part_buf.as<double>());
            GBN_CK_LAUNCH(c);
            k_norm_sum<<<1, 32, 0, c->stream>>>(part_buf.as<double>(), parts, cnt, norm_buf.as<double>());
            GBN_CK_LAUNCH(c);
            GBN_CK(c, cudaMemcpyAsync(hn.data(), norm_buf.p, sizeof(double) * cnt, cudaMemcpyDeviceToHost, c->stream));
            GBN_CK(c, cudaStreamSynchronize(c->stream));
            bool all_pos = true;
            for (int r = 0; r < cnt; ++r) all_pos = all_pos && hn[(size_t)r] > 0.0;
            for (int r = 0; r < cnt; ++r) norms[(size_t)(r0 + r) * nw + w] = hn[(size_t)r];
            if (all_pos) {
                const unsigned g = (unsigned)((n * cnt + 255) / 256);
                k_normalise<<<g, 256, 0, c->stream>>>(zin, norm_buf.as<double>(), n, cnt, c->upload.as<double2>());
                GBN_CK_LAUNCH(c);
                rc = lanczos_start_from_psi(c, c->upload.as<double>(), cnt);
                if (rc) return rc;
                rc = lanczos_run(c, nrecurs);
                if (rc) return rc;
                loop_ms += c->timing.step_ms;
                hab.resize((size_t)2 * T * nrecurs);
                GBN_CK(c, cudaMemcpyAsync(hab.data(), c->ab.p, sizeof(double) * hab.size(), cudaMemcpyDeviceToHost,
                                          c->stream));
                GBN_CK(c, cudaStreamSynchronize(c->stream));
            }
            for (int r = 0; r < cnt; ++r) {
                double* ao = a_out + ((size_t)(r0 + r) * nw + w) * nrecurs;
                double* bo = b_out + ((size_t)(r0 + r) * nw + w) * nrecurs;
                for (int k = 0; k < nrecurs; ++k) {
                    ao[k] = all_pos ? hab[(size_t)r * nrecurs + k] : NAN;
                    bo[k] = all_pos ? hab[(size_t)T * nrecurs + (size_t)r * nrecurs + k] : NAN;
                }
            }
            ++w;
        }
        GBN_CK(c, cudaMemcpyAsync(psi_host + (size_t)2 * n * r0, pin, sizeof(double2) * (size_t)n * cnt,
                                  cudaMemcpyDeviceToHost, c->stream));
        GBN_CK(c, cudaMemcpyAsync(zupsi_host + (size_t)2 * n * r0, zin, sizeof(double2) * (size_t)n * cnt,
                                  cudaMemcpyDeviceToHost, c->stream));
        GBN_CK(c, cudaStreamSynchronize(c->stream));
    }
    c->timing.step_launches = launches;
    return GBN_OK;
}

}  // namespace gbn
