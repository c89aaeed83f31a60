// Neighbour search on the device with the entries, their order and their displacement vectors of the
// reference's NeighSearchLayered (lanczosKuboCode/Src/neigh.F90:117-316, periodicZ = .false.).
//
// The reference enumerates periodic-image candidates in the order (u1, u2, atom), drops them into
// bins at least rmax wide by head insertion, and for each atom walks the 3 x 3 neighbouring bins
// (x outer, y inner), each bin's list from the last candidate inserted to the first.  Here the same
// order comes from data-parallel steps: the candidates are compacted in (u1, u2, atom) order, sorted
// by (bin ascending, candidate number descending), and one thread per atom walks the same nine bins.
// Every floating-point expression that decides an entry or enters NeighD is written with explicitly
// rounded operations (no FMA contraction), in the reference's association order, so the tables are
// bit-identical to the reference's.
#include <cuda_runtime.h>
#include <math.h>
#include <thrust/copy.h>
#include <thrust/count.h>
#include <thrust/for_each.h>
#include <thrust/reduce.h>
#include <thrust/sequence.h>
#include <thrust/device_ptr.h>
#include <thrust/execution_policy.h>
#include <thrust/extrema.h>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/sort.h>

#include <vector>

#include "gbn_internal.cuh"

namespace gbn {

struct SearchGeom {
    double a1x, a1y, a2x, a2y;
    double xlo, xhi, ylo, yhi, zlo, zhi;
    double wx, wy;
    double cut2intra, cut2inter;
    int32_t n1, n2, nbx, nby, second;
    int64_t natoms;
};

__device__ __forceinline__ double mulr(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double addr(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double subr(double a, double b) { return __dsub_rn(a, b); }

// per-block min/max of s1, s2, x, y, z (10 values)
__global__ void k_extent(const double* rat, int64_t n, double a1x, double a1y, double a2x, double a2y, double det,
                         double* out)
{
    __shared__ double sh[10][256];
    double v[10];
    for (int k = 0; k < 5; ++k) { v[2 * k] = INFINITY; v[2 * k + 1] = -INFINITY; }
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double x = rat[3 * i], y = rat[3 * i + 1], z = rat[3 * i + 2];
        const double s1 = __ddiv_rn(subr(mulr(x, a2y), mulr(y, a2x)), det);
        const double s2 = __ddiv_rn(addr(-mulr(x, a1y), mulr(y, a1x)), det);
        const double q[5] = {s1, s2, x, y, z};
        for (int k = 0; k < 5; ++k) {
            v[2 * k] = fmin(v[2 * k], q[k]);
            v[2 * k + 1] = fmax(v[2 * k + 1], q[k]);
        }
    }
    for (int k = 0; k < 10; ++k) sh[k][threadIdx.x] = v[k];
    __syncthreads();
    for (int off = 128; off > 0; off >>= 1) {
        if ((int)threadIdx.x < off)
            for (int k = 0; k < 10; ++k)
                sh[k][threadIdx.x] = (k & 1) ? fmax(sh[k][threadIdx.x], sh[k][threadIdx.x + off])
                                             : fmin(sh[k][threadIdx.x], sh[k][threadIdx.x + off]);
        __syncthreads();
    }
    if (threadIdx.x < 10) out[blockIdx.x * 10 + threadIdx.x] = sh[threadIdx.x][0];
}

// is the image (u1, u2) of atom m inside the box around the home cell?
struct InBox {
    const double* rat;
    SearchGeom g;
    __device__ bool operator()(int64_t L) const {
        const int64_t img = L / g.natoms, m = L % g.natoms;
        const int u1 = (int)(img / (2 * g.n2 + 1)) - g.n1;
        const int u2 = (int)(img % (2 * g.n2 + 1)) - g.n2;
        const double tx = addr(mulr((double)u1, g.a1x), mulr((double)u2, g.a2x));
        const double ty = addr(mulr((double)u1, g.a1y), mulr((double)u2, g.a2y));
        const double px = addr(rat[3 * m], tx);
        if (px < g.xlo || px > g.xhi) return false;
        const double py = addr(rat[3 * m + 1], ty);
        if (py < g.ylo || py > g.yhi) return false;
        const double pz = addr(rat[3 * m + 2], 0.0);
        if (pz < g.zlo || pz > g.zhi) return false;
        return true;
    }
};

__device__ __forceinline__ int bin_of(double p, double lo, double w, int nb)
{
    int i = 1 + (int)__ddiv_rn(subr(p, lo), w);
    i = i < 1 ? 1 : i;
    return i > nb ? nb : i;
}

__global__ void k_cand_keys(const int64_t* cand, int64_t ncand, const double* rat, SearchGeom g, uint64_t* keys,
                            int32_t* cidx, int32_t* cu)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncand) return;
    const int64_t L = cand[c];
    const int64_t img = L / g.natoms, m = L % g.natoms;
    const int u1 = (int)(img / (2 * g.n2 + 1)) - g.n1;
    const int u2 = (int)(img % (2 * g.n2 + 1)) - g.n2;
    const double px = addr(addr(rat[3 * m], mulr((double)u1, g.a1x)), mulr((double)u2, g.a2x));
    const double py = addr(addr(rat[3 * m + 1], mulr((double)u1, g.a1y)), mulr((double)u2, g.a2y));
    const int ibx = bin_of(px, g.xlo, g.wx, g.nbx);
    const int iby = bin_of(py, g.ylo, g.wy, g.nby);
    const uint32_t bin = (uint32_t)((iby - 1) * g.nbx + (ibx - 1));
    keys[c] = ((uint64_t)bin << 32) | (uint64_t)(0xffffffffu - (uint32_t)c);
    cidx[c] = (int32_t)m;
    cu[2 * c] = u1;
    cu[2 * c + 1] = u2;
}

__global__ void k_bin_ranges(const uint64_t* keys, int64_t ncand, int64_t* bstart, int64_t* bend)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ncand) return;
    const uint32_t b = (uint32_t)(keys[p] >> 32);
    if (p == 0 || (uint32_t)(keys[p - 1] >> 32) != b) bstart[b] = p;
    if (p == ncand - 1 || (uint32_t)(keys[p + 1] >> 32) != b) bend[b] = p + 1;
}

// pass 0: count; pass 1: fill (reference layout [n][maxNeigh])
__global__ void k_search(const double* rat, SearchGeom g, const uint64_t* keys, const int64_t* bstart,
                         const int64_t* bend, const int32_t* cidx_sorted, const int32_t* cu_sorted, int pass,
                         int32_t* nneigh, int32_t max_neigh, int32_t* nlist, double* neighd, int32_t* ncell)
{
    const int64_t nn = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (nn >= g.natoms) return;
    const double xn = rat[3 * nn], yn = rat[3 * nn + 1], zn = rat[3 * nn + 2];
    const int ibx = bin_of(xn, g.xlo, g.wx, g.nbx);
    const int iby = bin_of(yn, g.ylo, g.wy, g.nby);
    int cnt = 0;
    const int ax0 = ibx - 1 > 1 ? ibx - 1 : 1, ax1 = ibx + 1 < g.nbx ? ibx + 1 : g.nbx;
    const int ay0 = iby - 1 > 1 ? iby - 1 : 1, ay1 = iby + 1 < g.nby ? iby + 1 : g.nby;
    for (int ax = ax0; ax <= ax1; ++ax)
        for (int ay = ay0; ay <= ay1; ++ay) {
            const int64_t b = (int64_t)(ay - 1) * g.nbx + (ax - 1);
            const int64_t e0 = bstart[b], e1 = bend[b];
            for (int64_t p = e0; p < e1; ++p) {
                const int64_t m = cidx_sorted[p];
                const int c1 = cu_sorted[2 * p], c2 = cu_sorted[2 * p + 1];
                if (m == nn && c1 == 0 && c2 == 0) continue;
                const double tx = addr(mulr((double)c1, g.a1x), mulr((double)c2, g.a2x));
                const double ty = addr(mulr((double)c1, g.a1y), mulr((double)c2, g.a2y));
                const double ddx = addr(subr(rat[3 * m], xn), tx);
                const double ddy = addr(subr(rat[3 * m + 1], yn), ty);
                const double ddz = addr(subr(rat[3 * m + 2], zn), 0.0);
                const double adz = fabs(ddz);
                const double d2 = addr(mulr(ddx, ddx), mulr(ddy, ddy));
                bool keep;
                if (adz < 1.5) keep = d2 < g.cut2intra;
                else if (adz > 1.5 && adz < 4.5) keep = d2 < g.cut2inter;
                else if (g.second && adz > 4.5 && adz < 7.5) keep = d2 < g.cut2inter;
                else keep = false;
                if (keep) {
                    if (pass == 1 && cnt < max_neigh) {
                        const int64_t e = nn * max_neigh + cnt;
                        nlist[e] = (int32_t)(m + 1);
                        neighd[3 * e] = ddx;
                        neighd[3 * e + 1] = ddy;
                        neighd[3 * e + 2] = ddz;
                        ncell[3 * e] = c1;
                        ncell[3 * e + 1] = c2;
                        ncell[3 * e + 2] = 0;
                    }
                    ++cnt;
                }
            }
        }
    if (pass == 0) nneigh[nn] = cnt;
}

int neigh_search(gbn_ctx* c, double cut2intra, double cut2inter, int32_t second_layer)
{
    const int64_t n = c->n;
    SearchGeom g;
    g.a1x = c->ucell[0]; g.a1y = c->ucell[1]; g.a2x = c->ucell[3]; g.a2y = c->ucell[4];
    g.natoms = n;
    g.cut2intra = cut2intra;
    g.cut2inter = cut2inter;
    g.second = second_layer ? 1 : 0;
    // host scalars in the reference's operation order (this file is compiled without FMA contraction)
    volatile double det = g.a1x * g.a2y - g.a1y * g.a2x;
    if (fabs(det) < 2.2250738585072014e-308) return fail(c, GBN_ERR_ARG, "the in-plane lattice vectors are parallel");
    const double rmax = sqrt(fmax(cut2intra, cut2inter));
    const double dzmax = second_layer ? 7.5 : 4.5;
    const int eblocks = 256;
    DevBuf ext;
    GBN_CK(c, ext.ensure(sizeof(double) * 10 * eblocks));
    k_extent<<<eblocks, 256, 0, c->stream>>>(c->rat.as<double>(), n, g.a1x, g.a1y, g.a2x, g.a2y, det, ext.as<double>());
    GBN_CK_LAUNCH(c);
    std::vector<double> hext(10 * eblocks);
    GBN_CK(c, cudaMemcpyAsync(hext.data(), ext.p, sizeof(double) * hext.size(), cudaMemcpyDeviceToHost, c->stream));
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    double v[10];
    for (int k = 0; k < 10; ++k) v[k] = (k & 1) ? -INFINITY : INFINITY;
    for (int bI = 0; bI < eblocks; ++bI)
        for (int k = 0; k < 10; ++k) v[k] = (k & 1) ? fmax(v[k], hext[bI * 10 + k]) : fmin(v[k], hext[bI * 10 + k]);
    const double h1 = fabs(det) / sqrt(g.a2x * g.a2x + g.a2y * g.a2y);
    const double h2 = fabs(det) / sqrt(g.a1x * g.a1x + g.a1y * g.a1y);
    g.n1 = (int32_t)ceil(rmax / h1 + (v[1] - v[0]));
    g.n2 = (int32_t)ceil(rmax / h2 + (v[3] - v[2]));
    g.xlo = v[4] - rmax; g.xhi = v[5] + rmax;
    g.ylo = v[6] - rmax; g.yhi = v[7] + rmax;
    g.zlo = v[8] - dzmax; g.zhi = v[9] + dzmax;
    g.nbx = (int32_t)((g.xhi - g.xlo) / rmax); if (g.nbx < 1) g.nbx = 1;
    g.nby = (int32_t)((g.yhi - g.ylo) / rmax); if (g.nby < 1) g.nby = 1;
    g.wx = (g.xhi - g.xlo) / g.nbx;
    g.wy = (g.yhi - g.ylo) / g.nby;
    const int64_t nimg = (int64_t)(2 * g.n1 + 1) * (2 * g.n2 + 1);
    if ((int64_t)g.nbx * g.nby >= ((int64_t)1 << 32)) return fail(c, GBN_ERR_ARG, "too many search bins");

    // candidates in (u1, u2, atom) order
    DevBuf cand;
    GBN_CK(c, cand.ensure(sizeof(int64_t) * (size_t)(n * 2 + 64)));
    int64_t cap = n * 2 + 64;
    InBox pred{c->rat.as<double>(), g};
    thrust::counting_iterator<int64_t> first(0), last(nimg * n);
    // count first so that the output buffer is large enough
    const int64_t ncand = thrust::count_if(thrust::cuda::par.on(c->stream), first, last, pred);
    c->launches += 2;
    if (ncand >= ((int64_t)1 << 32) - 1) return fail(c, GBN_ERR_ARG, "too many periodic-image candidates");
    if (ncand > cap) GBN_CK(c, cand.ensure(sizeof(int64_t) * (size_t)ncand));
    thrust::device_ptr<int64_t> cp(cand.as<int64_t>());
    thrust::copy_if(thrust::cuda::par.on(c->stream), first, last, cp, pred);
    c->launches += 2;

    DevBuf keys, cidx, cu, cidx_s, cu_s, bstart, bend, order;
    GBN_CK(c, keys.ensure(sizeof(uint64_t) * ncand));
    GBN_CK(c, cidx.ensure(sizeof(int32_t) * ncand));
    GBN_CK(c, cu.ensure(sizeof(int32_t) * 2 * ncand));
    k_cand_keys<<<(unsigned)((ncand + 255) / 256), 256, 0, c->stream>>>(cand.as<int64_t>(), ncand, c->rat.as<double>(), g,
                                                                        keys.as<uint64_t>(), cidx.as<int32_t>(),
                                                                        cu.as<int32_t>());
    GBN_CK_LAUNCH(c);
    // sort candidate numbers by (bin, descending candidate number); keys are unique
    GBN_CK(c, order.ensure(sizeof(int32_t) * ncand));
    {
        thrust::device_ptr<int32_t> op(order.as<int32_t>());
        thrust::sequence(thrust::cuda::par.on(c->stream), op, op + ncand);
        thrust::device_ptr<uint64_t> kp(keys.as<uint64_t>());
        thrust::sort_by_key(thrust::cuda::par.on(c->stream), kp, kp + ncand, op);
        c->launches += 6;
    }
    GBN_CK(c, cidx_s.ensure(sizeof(int32_t) * ncand));
    GBN_CK(c, cu_s.ensure(sizeof(int32_t) * 2 * ncand));
    {
        const int32_t* ord = order.as<int32_t>();
        const int32_t* ci = cidx.as<int32_t>();
        const int32_t* cuu = cu.as<int32_t>();
        int32_t* cis = cidx_s.as<int32_t>();
        int32_t* cus = cu_s.as<int32_t>();
        thrust::for_each(thrust::cuda::par.on(c->stream), thrust::counting_iterator<int64_t>(0),
                         thrust::counting_iterator<int64_t>(ncand), [=] __device__(int64_t p) {
                             const int32_t o = ord[p];
                             cis[p] = ci[o];
                             cus[2 * p] = cuu[2 * o];
                             cus[2 * p + 1] = cuu[2 * o + 1];
                         });
        c->launches += 1;
    }
    const int64_t nbins = (int64_t)g.nbx * g.nby;
    GBN_CK(c, bstart.ensure(sizeof(int64_t) * nbins));
    GBN_CK(c, bend.ensure(sizeof(int64_t) * nbins));
    GBN_CK(c, cudaMemsetAsync(bstart.p, 0, sizeof(int64_t) * nbins, c->stream));
    GBN_CK(c, cudaMemsetAsync(bend.p, 0, sizeof(int64_t) * nbins, c->stream));
    k_bin_ranges<<<(unsigned)((ncand + 255) / 256), 256, 0, c->stream>>>(keys.as<uint64_t>(), ncand,
                                                                         bstart.as<int64_t>(), bend.as<int64_t>());
    GBN_CK_LAUNCH(c);

    GBN_CK(c, c->nneigh.ensure(sizeof(int32_t) * n));
    const unsigned ag = (unsigned)((n + 127) / 128);
    k_search<<<ag, 128, 0, c->stream>>>(c->rat.as<double>(), g, keys.as<uint64_t>(), bstart.as<int64_t>(),
                                        bend.as<int64_t>(), cidx_s.as<int32_t>(), cu_s.as<int32_t>(), 0,
                                        c->nneigh.as<int32_t>(), 0, nullptr, nullptr, nullptr);
    GBN_CK_LAUNCH(c);
    thrust::device_ptr<int32_t> np(c->nneigh.as<int32_t>());
    const int32_t mx = *thrust::max_element(thrust::cuda::par.on(c->stream), np, np + n);
    const int64_t tot = thrust::reduce(thrust::cuda::par.on(c->stream), np, np + n, (int64_t)0);
    c->launches += 4;
    c->max_neigh = mx < 1 ? 1 : mx;
    c->total = tot;
    const size_t e = (size_t)n * c->max_neigh;
    GBN_CK(c, c->nlist.ensure(sizeof(int32_t) * e));
    GBN_CK(c, c->neighd.ensure(sizeof(double) * 3 * e));
    GBN_CK(c, c->ncell.ensure(sizeof(int32_t) * 3 * e));
    GBN_CK(c, cudaMemsetAsync(c->nlist.p, 0, sizeof(int32_t) * e, c->stream));
    GBN_CK(c, cudaMemsetAsync(c->neighd.p, 0, sizeof(double) * 3 * e, c->stream));
    GBN_CK(c, cudaMemsetAsync(c->ncell.p, 0, sizeof(int32_t) * 3 * e, c->stream));
    k_search<<<ag, 128, 0, c->stream>>>(c->rat.as<double>(), g, keys.as<uint64_t>(), bstart.as<int64_t>(),
                                        bend.as<int64_t>(), cidx_s.as<int32_t>(), cu_s.as<int32_t>(), 1,
                                        c->nneigh.as<int32_t>(), c->max_neigh, c->nlist.as<int32_t>(),
                                        c->neighd.as<double>(), c->ncell.as<int32_t>());
    GBN_CK_LAUNCH(c);
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    c->have_neigh = true;
    c->have_neighd = true;
    c->have_ham = false;
    c->ell.valid = false;
    return GBN_OK;
}

}  // namespace gbn
