// Gradient of a DOS loss through the Lanczos recursion and the continued fraction (no counterpart in
// the reference): L = sum_E (DOS(E) - target(E))^2 with DOS from KuboRecursion + KuboFrac of one start
// vector, and dL/d(theta) for theta = (t, Vpp_sigma0, delta, w): the intralayer nearest-neighbour
// hopping [eV], the sigma two-centre amplitude [eV], the decay length of both two-centre terms [Ang] and
// the width of the smooth interlayer cutoff [Ang] (gbn_model.inter_smooth_w).
//
// Forward (FP64, one vector, the reference's three passes, kubosubs.F90:26-138):
//     u_k = H q_k,  a_k = Re q_k^+ u_k,  r_k = u_k - a_k q_k - b_{k-1} q_{k-1},  b_k = |r_k|,  q_{k+1} = r_k / b_k
// with (q_{k-1}, q_k) checkpointed every C steps.  The loss and its adjoints abar_k, bbar_k come from the
// continued fraction on the host.  The reverse sweep runs k = K-1 .. 0 through the same sparse product
// (H is Hermitian, so H^+ ubar = H ubar), recomputing each segment of C vectors from its checkpoint
// with the stored a, b (bit-identical to the forward pass):
//     rbar = qbar_{k+1} / b_k + (bbar_k - Re qbar_{k+1}^+ q_{k+1} / b_k) q_{k+1}
//     abar_k += -Re q_k^+ rbar;   bbar_{k-1} += -Re q_{k-1}^+ rbar;   ubar = rbar + abar_k q_k
//     qbar_k += -a_k rbar + abar_k u_k + H ubar   (u_k = b_k q_{k+1} + a_k q_k + b_{k-1} q_{k-1})
//     qbar_{k-1} += -b_{k-1} rbar;   Hbar_ij += Re conj(ubar_i) q_{k,j}
// and dL/dtheta = sum over entries of Hbar_ij dH_ij/dtheta, dH = -d(hopp), from the entries' geometry.
// Vectors are in the reference atom order; the sums are block partials reduced in a fixed order.
// Two variants: FP64 vectors and hoppings, or complex64 vectors and FP32 hoppings with the same FP64
// arithmetic, sums, scalars, continued fraction and Hbar accumulation (each stored vector rounded once).
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <complex>
#include <vector>

#include "gbn_internal.cuh"

namespace gbn {

namespace {

constexpr int kAdThreads = 256;

// Vector storage: complex128 (FP64 variant) or complex64 (FP32 variant).  Every kernel loads into FP64,
// computes in FP64 and rounds once when it stores; sums, scalars and Hbar stay FP64 in both variants.
__device__ __forceinline__ double2 ldv(const double2& v) { return v; }
__device__ __forceinline__ double2 ldv(const float2& v) { return make_double2(v.x, v.y); }
template <typename V> __device__ __forceinline__ V stv(double x, double y);
template <> __device__ __forceinline__ double2 stv<double2>(double x, double y) { return make_double2(x, y); }
template <> __device__ __forceinline__ float2 stv<float2>(double x, double y) { return make_float2((float)x, (float)y); }

// The adjoint's copy of the Hamiltonian: the reference tables (row i, slot j at i * mn + j, complex
// hoppings) transposed to slot-major order, entry (i, j) at j * n + i with the real hopping (HT: double or
// float) and the 0-based column, so that the threads of a warp (consecutive rows) read consecutive words.
template <typename HT>
struct AdTables {
    int64_t n;
    int32_t mn;
    const int32_t* nneigh;
    const int32_t* col;
    const HT* hop;
    const double* h0;
};

template <typename HT>
__global__ void k_ad_tables(int64_t n, int32_t mn, const int32_t* __restrict__ nneigh,
                            const int32_t* __restrict__ nlist, const double2* __restrict__ hopp,
                            int32_t* __restrict__ col, HT* __restrict__ hop)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int nn = nneigh[i];
    for (int j = 0; j < mn; ++j) {
        const int64_t src = i * mn + j, dst = (int64_t)j * n + i;
        col[dst] = j < nn ? nlist[src] - 1 : (int32_t)i;
        hop[dst] = (HT)(j < nn ? hopp[src].x : 0.0);
    }
}

// y = H x, one row per thread
template <typename V, typename HT>
__global__ void k_ad_apply(AdTables<HT> t, const V* __restrict__ x, V* __restrict__ y)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t.n) return;
    const double2 xi = ldv(x[i]);
    double cr = t.h0[i] * xi.x, ci = t.h0[i] * xi.y;
    const int nn = t.nneigh[i];
    for (int j = 0; j < nn; ++j) {
        const int64_t e = (int64_t)j * t.n + i;
        const double h = (double)t.hop[e];
        const double2 xj = ldv(x[t.col[e]]);
        cr -= h * xj.x;
        ci -= h * xj.y;
    }
    y[i] = stv<V>(cr, ci);
}

// fixed-order reduction: partial sums of up to 3 quantities per block
template <int NQ>
__device__ __forceinline__ void block_partials(double (&v)[NQ], double* partials)
{
    __shared__ double sh[NQ][kAdThreads / 32];
#pragma unroll
    for (int q = 0; q < NQ; ++q)
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int q = 0; q < NQ; ++q) sh[q][threadIdx.x >> 5] = v[q];
    __syncthreads();
    if (threadIdx.x < NQ) {
        double s = 0.0;
        for (int w = 0; w < kAdThreads / 32; ++w) s += sh[threadIdx.x][w];
        partials[(int64_t)blockIdx.x * NQ + threadIdx.x] = s;
    }
}

// sum of the block partials in a fixed order; op decides what becomes of the totals
enum : int { kSetA = 0, kSetB = 1, kSetS1 = 2, kRevDots = 3 };

constexpr int kFinThreads = 256;

__global__ void __launch_bounds__(kFinThreads) k_ad_finish(const double* partials, int nblocks, int nq, int op,
                                                           int k, double* a, double* b, double* abar, double* bbar,
                                                           double* scal)
{
    // thread t sums the partials of blocks t, t + 256, ... in block order, then a fixed tree
    __shared__ double sh[3][kFinThreads];
    double s[3] = {0.0, 0.0, 0.0};
    for (int blk = threadIdx.x; blk < nblocks; blk += kFinThreads) {
        const double* p = partials + (int64_t)blk * nq;
        s[0] += p[0];
        if (nq > 1) s[1] += p[1];
        if (nq > 2) s[2] += p[2];
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) sh[q][threadIdx.x] = s[q];
    __syncthreads();
    for (int w = kFinThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
#pragma unroll
            for (int q = 0; q < 3; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    const double s0 = sh[0][0], s1 = sh[1][0];
    if (op == kSetA) {
        a[k] = s0;
    } else if (op == kSetB) {
        b[k] = sqrt(fabs(s0));
    } else if (op == kSetS1) {
        scal[0] = s0;   // Re qbar_{k+1}^+ q_{k+1}
    } else {            // kRevDots: s0 = Re q_k^+ rbar, s1 = Re q_{k-1}^+ rbar
        scal[1] = abar[k] - s0;   // total abar_k
        if (k > 0) bbar[k - 1] -= s1;
    }
}

// forward: a_k = Re q^+ u (partials)
template <typename V>
__global__ void k_ad_dot_au(int64_t n, const V* q, const V* u, double* partials)
{
    double v[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 qi = ldv(q[i]), ui = ldv(u[i]);
        v[0] += qi.x * ui.x + qi.y * ui.y;
    }
    block_partials<1>(v, partials);
}

// forward: r = u - a_k q - b_{k-1} qm (into u) and |r|^2 partials (of the stored r)
template <typename V>
__global__ void k_ad_residual(int64_t n, V* u, const V* q, const V* qm, const double* a, const double* b, int k,
                              double* partials)
{
    const double ak = a[k], bp = k > 0 ? b[k - 1] : 0.0;
    double v[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 ui = ldv(u[i]), qi = ldv(q[i]), qmi = ldv(qm[i]);
        const V r = stv<V>((ui.x - ak * qi.x) - bp * qmi.x, (ui.y - ak * qi.y) - bp * qmi.y);
        u[i] = r;
        const double2 rd = ldv(r);
        v[0] += rd.x * rd.x + rd.y * rd.y;
    }
    block_partials<1>(v, partials);
}

// forward: q_{k+1} = r / b_k
template <typename V>
__global__ void k_ad_scale(int64_t n, const V* r, V* qn, const double* b, int k)
{
    const double bk = b[k];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 ri = ldv(r[i]);
        qn[i] = stv<V>(ri.x / bk, ri.y / bk);
    }
}

// reverse: Re qbar_{k+1}^+ q_{k+1}
template <typename V>
__global__ void k_ad_dot(int64_t n, const V* x, const V* y, double* partials)
{
    double v[1] = {0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 xi = ldv(x[i]), yi = ldv(y[i]);
        v[0] += xi.x * yi.x + xi.y * yi.y;
    }
    block_partials<1>(v, partials);
}

// reverse: rbar = qa / b_k + beta q_{k+1}, beta = bbar_k - s1 / b_k; dots with q_k and q_{k-1}
template <typename V>
__global__ void k_ad_rbar(int64_t n, const V* qa, const V* qk1, const V* qk, const V* qkm, V* rbar,
                          const double* b, const double* bbar, const double* scal, int k, double* partials)
{
    const double bk = b[k];
    const double beta = bbar[k] - scal[0] / bk;
    double v[2] = {0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 qai = ldv(qa[i]), q1 = ldv(qk1[i]), q0 = ldv(qk[i]);
        const V rs = stv<V>(qai.x / bk + beta * q1.x, qai.y / bk + beta * q1.y);
        rbar[i] = rs;
        const double2 r = ldv(rs);
        v[0] += q0.x * r.x + q0.y * r.y;
        if (qkm) {
            const double2 qmi = ldv(qkm[i]);
            v[1] += qmi.x * r.x + qmi.y * r.y;
        }
    }
    block_partials<2>(v, partials);
}

// reverse: ubar = rbar + abar_k q_k
template <typename V>
__global__ void k_ad_ubar(int64_t n, const V* rbar, const V* qk, V* ubar, const double* scal)
{
    const double ab = scal[1];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 r = ldv(rbar[i]), q = ldv(qk[i]);
        ubar[i] = stv<V>(r.x + ab * q.x, r.y + ab * q.y);
    }
}

// reverse: qbar_k = qb - a_k rbar + abar_k u_k + H ubar (into out); qbar_{k-1} partial = -b_{k-1} rbar
// (into qnext); Hbar_ij += Re conj(ubar_i) q_{k,j} (FP64)
template <typename V, typename HT>
__global__ void k_ad_back(AdTables<HT> t, const V* __restrict__ ubar, const V* __restrict__ rbar,
                          const V* __restrict__ qb, const V* __restrict__ qk1, const V* __restrict__ qk,
                          const V* __restrict__ qkm, V* __restrict__ out, V* __restrict__ qnext,
                          const double* a, const double* b, const double* scal, int k, double* __restrict__ hbar)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= t.n) return;
    const double ak = a[k], bk = b[k], bp = k > 0 ? b[k - 1] : 0.0, ab = scal[1];
    const double2 ui = ldv(ubar[i]);
    double hr = t.h0[i] * ui.x, hi = t.h0[i] * ui.y;
    const int nn = t.nneigh[i];
    for (int j = 0; j < nn; ++j) {
        const int64_t e = (int64_t)j * t.n + i;
        const int32_t jj = t.col[e];
        const double h = (double)t.hop[e];
        const double2 uj = ldv(ubar[jj]);
        hr -= h * uj.x;
        hi -= h * uj.y;
        const double2 qj = ldv(qk[jj]);
        hbar[e] += ui.x * qj.x + ui.y * qj.y;
    }
    const double2 r = ldv(rbar[i]), q1 = ldv(qk1[i]), q0 = ldv(qk[i]);
    const double2 qm = qkm ? ldv(qkm[i]) : make_double2(0.0, 0.0);
    const double2 qbi = ldv(qb[i]);
    const double2 uk = make_double2(bk * q1.x + ak * q0.x + bp * qm.x, bk * q1.y + ak * q0.y + bp * qm.y);
    out[i] = stv<V>(qbi.x - ak * r.x + ab * uk.x + hr, qbi.y - ak * r.y + ab * uk.y + hi);
    qnext[i] = stv<V>(-bp * r.x, -bp * r.y);
}

__device__ __forceinline__ double smooth_cut_w(double rho, double rc, double w, double* ds_dw)
{
    *ds_dw = 0.0;
    if (!(w > 0.0)) return 1.0;
    const double r0 = rc - w;
    if (rho <= r0) return 1.0;
    if (rho >= rc) return 0.0;
    const double x = (rho - r0) / w;
    *ds_dw = -0.5 * M_PI * sin(M_PI * x) * (rc - rho) / (w * w);
    return 0.5 * (1.0 + cos(M_PI * x));
}

// dL/dtheta = sum_e Hbar_e * (-d hopp_e / d theta), per-block partials of the four derivatives
template <typename HT>
__global__ void k_ad_params(AdTables<HT> t, gbn_model m, double g0, const double* neighd, const int32_t* layer,
                            const double* hbar, double* partials)
{
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < t.n; i += (int64_t)gridDim.x * blockDim.x) {
        const int nn = t.nneigh[i];
        for (int j = 0; j < nn; ++j) {
            const int64_t e = (int64_t)j * t.n + i, r = i * t.mn + j;   // slot-major; reference order
            const double hb = hbar[e];
            if (hb == 0.0) continue;
            const int32_t jj = t.col[e];
            const double Dx = neighd[3 * r], Dy = neighd[3 * r + 1], Dz = neighd[3 * r + 2];
            if (layer[i] == layer[jj]) {
                const double d = sqrt(Dx * Dx + Dy * Dy);
                if (d < 1.7) v[0] -= hb / g0;   // nearest neighbours: hopp = t / g0
            } else if (m.interlayer == 1) {
                const double dist = sqrt(Dx * Dx + Dy * Dy + Dz * Dz);
                const double rho = sqrt(Dx * Dx + Dy * Dy);
                // KoshinoSR and the coupling factor scale the whole term (constants of theta)
                const double f = (m.koshino_sr ? exp((fabs(Dz) - 3.25) / 1.34) : 1.0) *
                                 (m.renormalize_coupling ? m.coupling_factor : 1.0);
                const double es = exp(-(dist - m.d_interlayer) / m.bl_delta) * f;
                const double ep = exp(-(dist - m.aCC) / m.bl_delta) * f;
                const double vsig = m.vppsigma0 * es, vpi = m.vpppi0 * ep;
                const double q2 = (Dz / dist) * (Dz / dist);
                double dsw;
                const double sc = smooth_cut_w(rho, m.inter_cut_rho, m.inter_smooth_w, &dsw);
                const double core = vpi * (1.0 - q2) + vsig * q2;
                v[1] -= hb * sc * (-1.0 / g0) * es * q2;
                v[2] -= hb * sc * (vpi * (1.0 - q2) * (dist - m.aCC) + vsig * q2 * (dist - m.d_interlayer)) /
                        (m.bl_delta * m.bl_delta);
                v[3] -= hb * dsw * core;
            }
        }
    }
    __shared__ double sh[4][kAdThreads / 32];
#pragma unroll
    for (int q = 0; q < 4; ++q)
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    if ((threadIdx.x & 31) == 0)
        for (int q = 0; q < 4; ++q) sh[q][threadIdx.x >> 5] = v[q];
    __syncthreads();
    if (threadIdx.x < 4) {
        double s = 0.0;
        for (int w = 0; w < kAdThreads / 32; ++w) s += sh[threadIdx.x][w];
        partials[(int64_t)blockIdx.x * 4 + threadIdx.x] = s;
    }
}

template <typename V>
__global__ void k_ad_start(int64_t n, const double* u, V* q0, V* qm)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s, c;
    sincos(6.283185307179586 * u[i], &s, &c);
    const double isn = 1.0 / sqrt((double)n);
    q0[i] = stv<V>(c * isn, s * isn);
    qm[i] = stv<V>(0.0, 0.0);
}

// DOS of the continued fraction (KuboFrac), the loss and its adjoints abar, bbar (host, FP64)
double cf_loss_adjoint(const std::vector<double>& a, const std::vector<double>& b, double eta, int n_en, double emin,
                       double emax, const double* target, std::vector<double>& abar, std::vector<double>& bbar,
                       double* dos)
{
    typedef std::complex<double> cd;
    const int K = (int)a.size();
    abar.assign(K, 0.0);
    bbar.assign(K, 0.0);
    std::vector<cd> g(K);
    const double de = (emax - emin) / n_en;
    double loss = 0.0;
    for (int ie = 0; ie <= n_en; ++ie) {
        const cd z(emin + ie * de, eta);
        const double ainf = a[K - 1], binf = b[K - 1];
        const cd w = z - ainf;
        const cd s = std::sqrt(w * w - 4.0 * binf * binf);
        double sigma = 1.0;
        cd gt = (w - s) / (2.0 * binf * binf);
        if (gt.imag() >= 0.0) {
            sigma = -1.0;
            gt = (w + s) / (2.0 * binf * binf);
        }
        g[K - 1] = gt;
        for (int i = K - 2; i >= 0; --i) g[i] = 1.0 / (z - a[i] - b[i] * b[i] * g[i + 1]);
        const double D = -g[0].imag() / M_PI;
        if (dos) dos[ie] = D;
        const double diff = D - target[ie];
        loss += diff * diff;
        // adjoint: dL = c Im(dg_0) = Re(conj(gbar) dg_0) with gbar = i c
        cd gbar(0.0, 2.0 * diff * (-1.0 / M_PI));
        for (int i = 0; i <= K - 2; ++i) {
            const cd wbar = gbar * std::conj(-g[i] * g[i]);
            abar[i] += -wbar.real();
            bbar[i] += (std::conj(wbar) * (-2.0 * b[i] * g[i + 1])).real();
            gbar = -b[i] * b[i] * wbar;
        }
        const cd dg_dw = (1.0 - sigma * w / s) / (2.0 * binf * binf);
        const cd dg_db = 2.0 * sigma / (binf * s) - 2.0 * gt / binf;
        abar[K - 1] += (std::conj(gbar) * (-dg_dw)).real();
        bbar[K - 1] += (std::conj(gbar) * dg_db).real();
    }
    return loss;
}

}  // namespace

template <typename V, typename HT>
static int dos_gradient_t(gbn_ctx* c, const gbn_model* m, double g0, const double* u_host, int32_t K, int32_t C, double eta,
                 int32_t n_en, double emin, double emax, const double* target, double* loss_out, double* grad,
                 double* dos, double* a_out, double* b_out)
{
    if (!c->have_ham || !c->have_neighd || !c->have_geometry)
        return fail(c, GBN_ERR_STATE, "the gradient needs the geometry, neighbour tables and an assembled Hamiltonian");
    if (c->ham_complex) return fail(c, GBN_ERR_ARG, "the gradient is built for real hoppings (no field)");
    if (!m || !u_host || !target || !loss_out || !grad || K < 2 || n_en < 1 || !(eta > 0.0) || !(g0 > 0.0))
        return fail(c, GBN_ERR_ARG, "bad gradient arguments");
    if (C < 1 || C > K) C = K;
    const int64_t n = c->n;
    const int nseg = (K + C - 1) / C;
    const size_t vb = sizeof(V) * (size_t)n;
    // device memory: checkpoints (q_{c-1}, q_c) per segment, a segment of C + 2 vectors, 5 work vectors,
    // Hbar per entry, scalars and partial sums
    DevBuf ck, seg, work, hbar, scal, parts, ab, bb, abr, bbr, ud;
    GBN_CK(c, ck.ensure(vb * 2 * nseg));
    GBN_CK(c, seg.ensure(vb * (size_t)(C + 2)));
    GBN_CK(c, work.ensure(vb * 5));
    GBN_CK(c, hbar.ensure(sizeof(double) * (size_t)n * c->max_neigh));
    GBN_CK(c, scal.ensure(sizeof(double) * 4));
    const int blocks = (int)std::min<int64_t>((n + kAdThreads - 1) / kAdThreads, (int64_t)c->num_sms * 8);
    GBN_CK(c, parts.ensure(sizeof(double) * 4 * (size_t)std::max(blocks, (int)((n + kAdThreads - 1) / kAdThreads))));
    GBN_CK(c, ab.ensure(sizeof(double) * K));
    GBN_CK(c, bb.ensure(sizeof(double) * K));
    GBN_CK(c, abr.ensure(sizeof(double) * K));
    GBN_CK(c, bbr.ensure(sizeof(double) * K));
    GBN_CK(c, ud.ensure(sizeof(double) * (size_t)n));
    DevBuf tcol, thop;
    GBN_CK(c, tcol.ensure(sizeof(int32_t) * (size_t)n * c->max_neigh));
    GBN_CK(c, thop.ensure(sizeof(HT) * (size_t)n * c->max_neigh));
    AdTables<HT> t{n, c->max_neigh, c->nneigh.as<int32_t>(), tcol.as<int32_t>(), thop.as<HT>(), c->h0.as<double>()};
    V* CK = ck.as<V>();
    V* W = work.as<V>();
    double* A = ab.as<double>();
    double* B = bb.as<double>();
    double* P = parts.as<double>();
    const unsigned rows_grid = (unsigned)((n + kAdThreads - 1) / kAdThreads);
    cudaStream_t st = c->stream;
    GBN_CK(c, cudaMemcpyAsync(ud.p, u_host, sizeof(double) * n, cudaMemcpyHostToDevice, st));

    // forward pass with checkpoints: q_k in W[0], q_{k-1} in W[1], u/r in W[2], q_{k+1} in W[3]
    V *qk = W, *qm = W + n, *ur = W + 2 * n, *qn = W + 3 * n;
    k_ad_tables<<<rows_grid, kAdThreads, 0, st>>>(n, c->max_neigh, c->nneigh.as<int32_t>(), c->nlist.as<int32_t>(),
                                                  c->hopp.as<double2>(), tcol.as<int32_t>(), thop.as<HT>());
    k_ad_start<<<rows_grid, kAdThreads, 0, st>>>(n, ud.as<double>(), qk, qm);
    GBN_CK_LAUNCH(c);
    c->launches += 2;
    auto fwd_step = [&](V* q, V* qmm, V* u, V* qnext, int k) -> int {
        k_ad_apply<<<rows_grid, kAdThreads, 0, st>>>(t, q, u);
        k_ad_dot_au<<<blocks, kAdThreads, 0, st>>>(n, q, u, P);
        k_ad_finish<<<1, kFinThreads, 0, st>>>(P, blocks, 1, kSetA, k, A, B, nullptr, nullptr, nullptr);
        k_ad_residual<<<blocks, kAdThreads, 0, st>>>(n, u, q, qmm, A, B, k, P);
        k_ad_finish<<<1, kFinThreads, 0, st>>>(P, blocks, 1, kSetB, k, A, B, nullptr, nullptr, nullptr);
        k_ad_scale<<<blocks, kAdThreads, 0, st>>>(n, u, qnext, B, k);
        GBN_CK_LAUNCH(c);
        c->launches += 6;
        return GBN_OK;
    };
    for (int k = 0; k < K; ++k) {
        if (k % C == 0) {
            const int sI = k / C;
            GBN_CK(c, cudaMemcpyAsync(CK + (size_t)(2 * sI) * n, qm, vb, cudaMemcpyDeviceToDevice, st));
            GBN_CK(c, cudaMemcpyAsync(CK + (size_t)(2 * sI + 1) * n, qk, vb, cudaMemcpyDeviceToDevice, st));
        }
        int rc = fwd_step(qk, qm, ur, qn, k);
        if (rc) return rc;
        V* tmp = qm;
        qm = qk;
        qk = qn;
        qn = tmp;
    }
    std::vector<double> a(K), b(K);
    GBN_CK(c, cudaMemcpyAsync(a.data(), A, sizeof(double) * K, cudaMemcpyDeviceToHost, st));
    GBN_CK(c, cudaMemcpyAsync(b.data(), B, sizeof(double) * K, cudaMemcpyDeviceToHost, st));
    GBN_CK(c, cudaStreamSynchronize(st));
    for (int k = 0; k < K; ++k)
        if (!(b[k] > 0.0) || !isfinite(b[k]) || !isfinite(a[k]))
            return fail(c, GBN_ERR_NUMERIC, "recursion produced a non-positive or non-finite b_n");
    if (a_out) std::copy(a.begin(), a.end(), a_out);
    if (b_out) std::copy(b.begin(), b.end(), b_out);

    // loss and its adjoints
    std::vector<double> abar, bbar;
    const double loss = cf_loss_adjoint(a, b, eta, n_en, emin, emax, target, abar, bbar, dos);
    *loss_out = loss;
    GBN_CK(c, cudaMemcpyAsync(abr.p, abar.data(), sizeof(double) * K, cudaMemcpyHostToDevice, st));
    GBN_CK(c, cudaMemcpyAsync(bbr.p, bbar.data(), sizeof(double) * K, cudaMemcpyHostToDevice, st));

    // reverse sweep by segments: seg[j] = q_{c-1+j}, j = 0 .. len+1 (q_{c-1} .. q_{c+len})
    V* S = seg.as<V>();
    V *qa = W, *qb = W + n, *rb = W + 2 * n, *ub = W + 3 * n, *tmpv = W + 4 * n;
    GBN_CK(c, cudaMemsetAsync(qa, 0, vb, st));   // qbar_K = 0
    GBN_CK(c, cudaMemsetAsync(qb, 0, vb, st));   // qbar_{K-1} (partial) = 0
    GBN_CK(c, cudaMemsetAsync(hbar.p, 0, sizeof(double) * (size_t)n * c->max_neigh, st));
    double* SC = scal.as<double>();
    double* AB = abr.as<double>();
    double* BB = bbr.as<double>();
    for (int sI = nseg - 1; sI >= 0; --sI) {
        const int c0 = sI * C;
        const int len = std::min(C, K - c0);
        GBN_CK(c, cudaMemcpyAsync(S, CK + (size_t)(2 * sI) * n, vb, cudaMemcpyDeviceToDevice, st));
        GBN_CK(c, cudaMemcpyAsync(S + n, CK + (size_t)(2 * sI + 1) * n, vb, cudaMemcpyDeviceToDevice, st));
        for (int j = 0; j < len; ++j) {   // recompute q_{c0+1} .. q_{c0+len} with the stored a, b
            const int k = c0 + j;
            V *q = S + (size_t)(j + 1) * n, *qmm = S + (size_t)j * n, *qnext = S + (size_t)(j + 2) * n;
            k_ad_apply<<<rows_grid, kAdThreads, 0, st>>>(t, q, tmpv);
            k_ad_residual<<<blocks, kAdThreads, 0, st>>>(n, tmpv, q, qmm, A, B, k, P);
            k_ad_scale<<<blocks, kAdThreads, 0, st>>>(n, tmpv, qnext, B, k);
            GBN_CK_LAUNCH(c);
            c->launches += 3;
        }
        for (int j = len - 1; j >= 0; --j) {
            const int k = c0 + j;
            const V* qk1 = S + (size_t)(j + 2) * n;
            const V* q0 = S + (size_t)(j + 1) * n;
            const V* qkm = (k > 0) ? S + (size_t)j * n : nullptr;
            k_ad_dot<<<blocks, kAdThreads, 0, st>>>(n, qa, qk1, P);
            k_ad_finish<<<1, kFinThreads, 0, st>>>(P, blocks, 1, kSetS1, k, nullptr, nullptr, AB, BB, SC);
            k_ad_rbar<<<blocks, kAdThreads, 0, st>>>(n, qa, qk1, q0, qkm, rb, B, BB, SC, k, P);
            k_ad_finish<<<1, kFinThreads, 0, st>>>(P, blocks, 2, kRevDots, k, nullptr, nullptr, AB, BB, SC);
            k_ad_ubar<<<blocks, kAdThreads, 0, st>>>(n, rb, q0, ub, SC);
            // qbar_k into tmpv, the partial qbar_{k-1} into qa (no longer needed)
            k_ad_back<<<rows_grid, kAdThreads, 0, st>>>(t, ub, rb, qb, qk1, q0, qkm, tmpv, qa, A, B, SC, k,
                                                       hbar.as<double>());
            GBN_CK_LAUNCH(c);
            c->launches += 6;
            V* old_qa = qa;
            qa = tmpv;   // qbar_k (complete)
            tmpv = qb;   // free
            qb = old_qa; // qbar_{k-1} (partial)
        }
    }
    // contraction with the parameter derivatives
    const int pblocks = (int)rows_grid;
    k_ad_params<<<pblocks, kAdThreads, 0, st>>>(t, *m, g0, c->neighd.as<double>(), c->layer.as<int32_t>(),
                                                hbar.as<double>(), P);
    GBN_CK_LAUNCH(c);
    c->launches += 1;
    std::vector<double> hp((size_t)pblocks * 4);
    GBN_CK(c, cudaMemcpyAsync(hp.data(), P, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, st));
    GBN_CK(c, cudaStreamSynchronize(st));
    for (int q = 0; q < 4; ++q) {
        double s = 0.0;
        for (int blk = 0; blk < pblocks; ++blk) s += hp[(size_t)blk * 4 + q];
        grad[q] = s;
    }
    return GBN_OK;
}

int dos_gradient(gbn_ctx* c, int32_t prec, const gbn_model* m, double g0, const double* u_host, int32_t K, int32_t C,
                 double eta, int32_t n_en, double emin, double emax, const double* target, double* loss_out,
                 double* grad, double* dos, double* a_out, double* b_out)
{
    if (prec == GBN_FP64)
        return dos_gradient_t<double2, double>(c, m, g0, u_host, K, C, eta, n_en, emin, emax, target, loss_out, grad,
                                               dos, a_out, b_out);
    if (prec == GBN_MIXED)
        return dos_gradient_t<float2, float>(c, m, g0, u_host, K, C, eta, n_en, emin, emax, target, loss_out, grad,
                                             dos, a_out, b_out);
    return fail(c, GBN_ERR_ARG, "bad precision");
}

}  // namespace gbn
