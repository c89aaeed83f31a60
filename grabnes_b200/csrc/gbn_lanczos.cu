// Batched Lanczos recursion on the B200: two launches per recursion step.
//
// The reference (lanczosKuboCode/Src/kubosubs.F90:26-138) makes three passes over the vectors per
// step: H psi with <psi, H psi>; w = H psi - a psi - b psi_prev with |w|; the scaling psi = w / b.
// Here the carried state is the pair
//     v_k = H x_{k-1} - b_{k-2} x_{k-2}      and     x_{k-1},
// and a step is
//   k_update    x_k = (v_k - a_{k-1} x_{k-1}) / b_{k-1}             stream: read v, x_{k-1}; write x_k
//   k_spmm_*    y = H x_k (one gather of x_k per union column of a row group), v_{k+1} = y - b_{k-1} x_{k-1},
//               and four FP64 dot products per vector
//                  S1 = Re<x_k, y>, S2 = |v_{k+1}|^2, S3 = Re<x_k, v_{k+1}>, S4 = |x_k|^2,
//               from which a_k = S1 and b_k^2 = |v_{k+1} - a_k x_k|^2 = S2 - 2 a_k S3 + a_k^2 S4.
// The partial sums of the blocks are reduced in a fixed order by the last block to finish (so the
// result does not depend on scheduling), which also writes a_k, b_k and the scalars of the next step.
//
// Vectors of R right-hand sides are interleaved per row ([row][R] complex): TPR threads share a row
// group, each holding RPT right-hand sides (8-32 bytes per gather).  With 16 vectors a gathered row is
// one 128-byte line.  The product is bound by the latency of the chain column index -> gather: the
// grouped layout (struct Ell) gathers a column once for the G rows of a group, and the staged kernel
// brings each warp's next slice record (column indices and values) into shared memory with one bulk
// asynchronous copy, so that only the gathers themselves wait on memory.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include "gbn_step.cuh"

namespace gbn {

// ---------------------------------------------------------------------------- update kernel
// x_k = (v_k - a x_{k-1}) * (1/b) for all rows and right-hand sides (streaming).  The grid stride and
// the block size are multiples of R, so every thread keeps one right-hand side and its 1/b.
template <typename VT>
__global__ void __launch_bounds__(256) k_update(const typename V2<VT>::t* __restrict__ v,
                                                const typename V2<VT>::t* __restrict__ xp,
                                                typename V2<VT>::t* __restrict__ xc, const double* __restrict__ scal,
                                                int64_t total, int R)
{
    const int r = (int)(threadIdx.x & (unsigned)(R - 1));
    const double a = scal[2 * r], ib = 1.0 / scal[2 * r + 1];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += stride) {
        const typename V2<VT>::t vv = __ldcs(v + e), xx = __ldcs(xp + e);
        typename V2<VT>::t o;   // FP64 arithmetic, one rounding to the storage type
        o.x = (VT)(((double)vv.x - a * (double)xx.x) * ib);
        o.y = (VT)(((double)vv.y - a * (double)xx.y) * ib);
        xc[e] = o;
    }
}

// ---------------------------------------------------------------------------- sparse product
// ---------------------------------------------------------------------------- start vectors
// v <- psi (rows in the solver order), x_prev <- 0; then the first update gives x_1 = psi (a_0 = 0, b_0 = 1).
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
void split_rhs(int prec, int R, int want, int* rpt, int* tpr)
{
    const int maxr = (prec == GBN_MIXED) ? 4 : 2;
    int r = R < maxr ? R : maxr;
    if (want > 0 && want < r && R % want == 0) r = want;
    if (R / r > 32) r = R / 32;
    *rpt = r;
    *tpr = R / r;
}


template <typename VT, bool CPLX, int G>
static StepFn pick_g(int rpt, int tpr, bool staged)
{
#define GBN_CASE(RP, TP) \
    if (rpt == RP && tpr == TP) return staged ? k_spmm_staged<VT, CPLX, G, RP, TP> : k_spmm_step<VT, CPLX, G, RP, TP>;
    GBN_CASE(1, 1) GBN_CASE(1, 2) GBN_CASE(1, 4) GBN_CASE(1, 8) GBN_CASE(1, 16) GBN_CASE(1, 32)
    GBN_CASE(2, 1) GBN_CASE(2, 2) GBN_CASE(2, 4) GBN_CASE(2, 8) GBN_CASE(2, 16)
    if constexpr (sizeof(VT) == 4) {
        GBN_CASE(4, 1) GBN_CASE(4, 2) GBN_CASE(4, 4) GBN_CASE(4, 8)
    }
#undef GBN_CASE
    return nullptr;
}

template <typename VT, bool CPLX>
static StepFn pick(int G, int rpt, int tpr, bool staged)
{
    if (G == 1) return pick_g<VT, CPLX, 1>(rpt, tpr, staged);
    if (G == 2) return pick_g<VT, CPLX, 2>(rpt, tpr, staged);
    if (G == 4) return pick_g<VT, CPLX, 4>(rpt, tpr, staged);
    return nullptr;
}

static StepFn step_kernel(int prec, bool cplx, int G, int R, int want_rpt, bool staged)
{
    int rpt, tpr;
    split_rhs(prec, R, want_rpt, &rpt, &tpr);
    if (prec == GBN_MIXED) return cplx ? pick<float, true>(G, rpt, tpr, staged) : pick<float, false>(G, rpt, tpr, staged);
    return cplx ? pick<double, true>(G, rpt, tpr, staged) : pick<double, false>(G, rpt, tpr, staged);
}

// Launch shape of the sparse product.  Staged: warps per block such that two record buffers per warp
// fit the shared-memory budget (the plain kernel when the block reduction's 4 R threads do not fit).
struct StepLaunch {
    StepFn fn = nullptr;
    int grid = 0, block = 256;
    size_t smem = 0;
    bool staged = false;
};

constexpr size_t kStagedSmemBudget = 200 * 1024;

static int step_launch(gbn_ctx* c, int R, StepLaunch* L)
{
    const Ell& E = c->ell;
    const size_t per_warp = 2 * (size_t)E.cap_record;
    const size_t min_warps = (size_t)((4 * R + 31) / 32);
    const bool staged = c->tune_staged != 0 && per_warp > 0 && 128 + min_warps * per_warp <= kStagedSmemBudget;
    L->staged = staged;
    if (E.field) {
        int rpt, tpr;
        split_rhs(c->prec, R, c->tune_rpt, &rpt, &tpr);
        L->fn = field_step_kernel(c->prec, E.G, rpt, tpr, staged);
    } else {
        L->fn = step_kernel(c->prec, E.cplx, E.G, R, c->tune_rpt, staged);
    }
    if (!L->fn) return fail(c, GBN_ERR_ARG, "no recursion kernel for this tile width");
    L->block = 256;
    L->smem = 0;
    if (staged) {
        size_t nw = (kStagedSmemBudget - 128) / per_warp;
        nw = nw > 8 ? 8 : nw;   // >= min_warps by the test above
        L->block = (int)(32 * nw);
        L->smem = 128 + nw * per_warp;
        GBN_CK(c, cudaFuncSetAttribute(L->fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L->smem));
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
    const int G = c->tune_group > 0 ? c->tune_group : auto_group(c, nrhs);
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
    GBN_CK(c, c->partials.ensure(sizeof(double) * (size_t)L.grid * nrhs * 4));
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
    const int64_t extra[4] = {total, ublk, ugrid, ((int64_t)c->prec << 32) | (int64_t)c->nrhs};
    memcpy(key.data(), &q, sizeof q);
    memcpy(key.data() + sizeof q, &L, sizeof L);
    memcpy(key.data() + sizeof q + sizeof L, extra, sizeof extra);
    const void* vp[3] = {c->vec[0].p, c->vec[1].p, c->vec[2].p};
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
    GBN_CK(c, c->ab.ensure(sizeof(double) * 2 * (size_t)R * nmax));
    k_init_scalars<<<1, 64, 0, c->stream>>>(c->scal.as<double>(), c->counter.as<unsigned int>(), R);
    GBN_CK_LAUNCH(c);
    StepLaunch L;
    memset(&L, 0, sizeof L);   // the graph key compares these structures bytewise, padding included
    const int rc = step_launch(c, R, &L);
    if (rc) return rc;
    c->last_staged = L.staged;
    StepParams p;
    memset(&p, 0, sizeof p);
    p.slice_ptr = c->ell.slice_ptr.as<int64_t>();
    p.mat = c->ell.mat.as<unsigned char>();
    p.entry_bytes = c->ell.entry_bytes;
    p.cap_record = c->ell.cap_record;
    p.prefetch = c->tune_prefetch < 0 ? 4 : c->tune_prefetch;   // default: the epilogue rows into L2
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
    const int64_t total = c->ell.npad * R;
    const int ublk = 256;   // a multiple of R (k_update keeps one right-hand side per thread)
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
    // step k (0-based): x_prev in vec[1 + k%2], x_cur written to vec[1 + (k+1)%2]; the step index of the
    // a_n, b_n outputs lives on the device (counter[1]), so a run of an even number of steps replays as is
    auto launch_step = [&](int32_t k) -> int {
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
    // small cells), unless the caller is capturing this stream into a graph of its own.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    GBN_CK(c, cudaStreamIsCapturing(c->stream, &cap));
    if (cap == cudaStreamCaptureStatusNone && nmax - k >= 2 * kGraphSteps) {
        const int rc2 = ensure_step_graph(c, L, p, total, ublk, ugrid, launch_step, k);
        if (rc2) return rc2;
        for (; nmax - k >= kGraphSteps; k += kGraphSteps) {
            GBN_CK(c, cudaGraphLaunch(c->step_graph, c->stream));
            c->launches += 2 * kGraphSteps;
            ++c->graph_replays;
        }
    }
    for (; k < nmax; ++k) {
        const int rc2 = launch_step(k);
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
