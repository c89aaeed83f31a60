// Row order and sliced-ELL layout of the Hamiltonian for the recursion kernels.
//
// Rows are renumbered along a Morton (Z-order) curve over the fractional coordinates of the atoms
// (cells of about 4 Angstrom), both layers of a bilayer falling into the same cells.  Consecutive
// slices then touch a compact region of the vectors, so the gathers of neighbouring rows hit L2.
// The reference's own atom order (kept for all exchanged arrays) is restored at the boundary by the
// permutation perm[new] = reference index.
#include <cuda_runtime.h>
#include <thrust/device_ptr.h>
#include <thrust/execution_policy.h>
#include <thrust/scan.h>
#include <thrust/sequence.h>
#include <thrust/sort.h>

#include <algorithm>
#include <vector>

#include "gbn_internal.cuh"

namespace gbn {

__global__ void k_identity(int32_t* perm, int32_t* iperm, int64_t n)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        perm[i] = (int32_t)i;
        iperm[i] = (int32_t)i;
    }
}

__device__ __forceinline__ uint64_t spread_bits(uint32_t v)
{
    uint64_t x = v & 0x1fffffu;
    x = (x | (x << 32)) & 0x1f00000000ffffULL;
    x = (x | (x << 16)) & 0x1f0000ff0000ffULL;
    x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
    x = (x | (x << 2)) & 0x1249249249249249ULL;
    return x;
}

__global__ void k_morton_keys(const double* rat, int64_t n, double a1x, double a1y, double a2x, double a2y,
                              int32_t g1, int32_t g2, uint64_t* keys, int32_t* idx)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double det = a1x * a2y - a1y * a2x;
    const double x = rat[3 * i], y = rat[3 * i + 1];
    double s1 = (x * a2y - y * a2x) / det;
    double s2 = (-x * a1y + y * a1x) / det;
    s1 -= floor(s1);
    s2 -= floor(s2);
    int32_t ix = (int32_t)(s1 * g1), iy = (int32_t)(s2 * g2);
    ix = ix < 0 ? 0 : (ix >= g1 ? g1 - 1 : ix);
    iy = iy < 0 ? 0 : (iy >= g2 ? g2 - 1 : iy);
    keys[i] = spread_bits((uint32_t)ix) | (spread_bits((uint32_t)iy) << 1);
    idx[i] = (int32_t)i;
}

__global__ void k_invert(const int32_t* perm, int32_t* iperm, int64_t n)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) iperm[perm[i]] = (int32_t)i;
}

int build_identity_perm(gbn_ctx* c)
{
    GBN_CK(c, c->perm.ensure(sizeof(int32_t) * c->n));
    GBN_CK(c, c->iperm.ensure(sizeof(int32_t) * c->n));
    k_identity<<<(unsigned)((c->n + 255) / 256), 256, 0, c->stream>>>(c->perm.as<int32_t>(), c->iperm.as<int32_t>(), c->n);
    GBN_CK_LAUNCH(c);
    c->perm_spatial = false;
    c->ell.valid = false;
    return GBN_OK;
}

int build_spatial_perm(gbn_ctx* c)
{
    if (!c->have_geometry) return build_identity_perm(c);
    const double a1x = c->ucell[0], a1y = c->ucell[1], a2x = c->ucell[3], a2y = c->ucell[4];
    const double l1 = sqrt(a1x * a1x + a1y * a1y), l2 = sqrt(a2x * a2x + a2y * a2y);
    const double cell = 4.0;
    int32_t g1 = (int32_t)ceil(l1 / cell), g2 = (int32_t)ceil(l2 / cell);
    g1 = g1 < 1 ? 1 : (g1 > (1 << 21) ? (1 << 21) : g1);
    g2 = g2 < 1 ? 1 : (g2 > (1 << 21) ? (1 << 21) : g2);
    DevBuf keys;
    GBN_CK(c, keys.ensure(sizeof(uint64_t) * c->n));
    GBN_CK(c, c->perm.ensure(sizeof(int32_t) * c->n));
    GBN_CK(c, c->iperm.ensure(sizeof(int32_t) * c->n));
    const unsigned grd = (unsigned)((c->n + 255) / 256);
    k_morton_keys<<<grd, 256, 0, c->stream>>>(c->rat.as<double>(), c->n, a1x, a1y, a2x, a2y, g1, g2,
                                              keys.as<uint64_t>(), c->perm.as<int32_t>());
    GBN_CK_LAUNCH(c);
    thrust::device_ptr<uint64_t> kp(keys.as<uint64_t>());
    thrust::device_ptr<int32_t> vp(c->perm.as<int32_t>());
    thrust::stable_sort_by_key(thrust::cuda::par.on(c->stream), kp, kp + c->n, vp);
    c->launches += 4;  // radix-sort passes issued by thrust (setup only)
    k_invert<<<grd, 256, 0, c->stream>>>(c->perm.as<int32_t>(), c->iperm.as<int32_t>(), c->n);
    GBN_CK_LAUNCH(c);
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    keys.release();
    c->perm_spatial = true;
    c->ell.valid = false;
    return GBN_OK;
}

// entries of every slice: sh rows times the longest row, the width rounded up so that a slice holds a
// multiple of 4 entries (every slice then starts on a 16-byte boundary for the bulk copies)
__global__ void k_slice_width(const int32_t* nneigh, const int32_t* perm, int64_t n, int sh, int64_t nslices,
                              int64_t* width_x_sh)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslices) return;
    int w = 0;
    for (int r = 0; r < sh; ++r) {
        const int64_t row = s * sh + r;
        if (row < n) {
            const int k = nneigh[perm[row]];
            w = k > w ? k : w;
        }
    }
    const int unit = sh >= 4 ? 1 : 4 / sh;
    w = (w + unit - 1) / unit * unit;
    width_x_sh[s] = (int64_t)w * sh;
}

template <typename HV>
__device__ __forceinline__ HV conv_hop(double2 h);
template <> __device__ __forceinline__ float conv_hop<float>(double2 h) { return (float)h.x; }
template <> __device__ __forceinline__ double conv_hop<double>(double2 h) { return h.x; }
template <> __device__ __forceinline__ float2 conv_hop<float2>(double2 h) { return make_float2((float)h.x, (float)h.y); }
template <> __device__ __forceinline__ double2 conv_hop<double2>(double2 h) { return h; }
template <typename HV> __device__ __forceinline__ HV zero_hop();
template <> __device__ __forceinline__ float zero_hop<float>() { return 0.f; }
template <> __device__ __forceinline__ double zero_hop<double>() { return 0.0; }
template <> __device__ __forceinline__ float2 zero_hop<float2>() { return make_float2(0.f, 0.f); }
template <> __device__ __forceinline__ double2 zero_hop<double2>() { return make_double2(0.0, 0.0); }

template <typename HV, typename DV>
__global__ void k_fill_ell(const int32_t* nneigh, const int32_t* nlist, const double2* hopp, const double* h0,
                           const int32_t* perm, const int32_t* iperm, int64_t n, int32_t max_neigh, int sh,
                           int64_t npad, const int64_t* slice_ptr, int32_t* col, HV* val, DV* h0p)
{
    const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= npad) return;
    const int64_t s = row / sh;
    const int r = (int)(row % sh);
    const int64_t base = slice_ptr[s];
    const int w = (int)((slice_ptr[s + 1] - base) / sh);
    int k = 0;
    if (row < n) {
        const int64_t p = perm[row];
        k = nneigh[p];
        for (int j = 0; j < k; ++j) {
            const int64_t e = p * max_neigh + j;
            col[base + (int64_t)j * sh + r] = iperm[nlist[e] - 1];
            val[base + (int64_t)j * sh + r] = conv_hop<HV>(hopp[e]);
        }
        h0p[row] = (DV)h0[p];
    } else {
        h0p[row] = (DV)0;
    }
    for (int j = k; j < w; ++j) {
        col[base + (int64_t)j * sh + r] = (int32_t)row;
        val[base + (int64_t)j * sh + r] = zero_hop<HV>();
    }
}

int build_ell(gbn_ctx* c, int prec, int sh)
{
    if (!c->have_ham) return fail(c, GBN_ERR_STATE, "no Hamiltonian loaded");
    if (!c->perm.p) {
        const int rc = build_identity_perm(c);
        if (rc) return rc;
    }
    Ell& E = c->ell;
    E.valid = false;
    E.sh = sh;
    E.prec = prec;
    E.cplx = c->ham_complex;
    E.nslices = (c->n + sh - 1) / sh;
    E.npad = E.nslices * sh;
    GBN_CK(c, E.slice_ptr.ensure(sizeof(int64_t) * (E.nslices + 1)));
    int64_t* sp = E.slice_ptr.as<int64_t>();
    GBN_CK(c, cudaMemsetAsync(sp + E.nslices, 0, sizeof(int64_t), c->stream));
    k_slice_width<<<(unsigned)((E.nslices + 255) / 256), 256, 0, c->stream>>>(
        c->nneigh.as<int32_t>(), c->perm.as<int32_t>(), c->n, sh, E.nslices, sp);
    GBN_CK_LAUNCH(c);
    thrust::device_ptr<int64_t> tp(sp);
    thrust::exclusive_scan(thrust::cuda::par.on(c->stream), tp, tp + E.nslices + 1, tp);
    c->launches += 2;
    GBN_CK(c, cudaMemcpyAsync(&E.nnz_stored, sp + E.nslices, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    size_t vsz;
    if (prec == GBN_MIXED) vsz = E.cplx ? sizeof(float2) : sizeof(float);
    else vsz = E.cplx ? sizeof(double2) : sizeof(double);
    GBN_CK(c, E.col.ensure(sizeof(int32_t) * (size_t)(E.nnz_stored > 0 ? E.nnz_stored : 1)));
    GBN_CK(c, E.val.ensure(vsz * (size_t)(E.nnz_stored > 0 ? E.nnz_stored : 1)));
    GBN_CK(c, E.h0.ensure((prec == GBN_MIXED ? sizeof(float) : sizeof(double)) * (size_t)E.npad));
    const unsigned grd = (unsigned)((E.npad + 255) / 256);
    const int32_t* nn = c->nneigh.as<int32_t>();
    const int32_t* nl = c->nlist.as<int32_t>();
    const double2* hp = c->hopp.as<double2>();
    const double* h0 = c->h0.as<double>();
    const int32_t* pm = c->perm.as<int32_t>();
    const int32_t* ip = c->iperm.as<int32_t>();
    if (prec == GBN_MIXED) {
        if (E.cplx)
            k_fill_ell<float2, float><<<grd, 256, 0, c->stream>>>(nn, nl, hp, h0, pm, ip, c->n, c->max_neigh, sh, E.npad, sp,
                                                                  E.col.as<int32_t>(), E.val.as<float2>(), E.h0.as<float>());
        else
            k_fill_ell<float, float><<<grd, 256, 0, c->stream>>>(nn, nl, hp, h0, pm, ip, c->n, c->max_neigh, sh, E.npad, sp,
                                                                 E.col.as<int32_t>(), E.val.as<float>(), E.h0.as<float>());
    } else {
        if (E.cplx)
            k_fill_ell<double2, double><<<grd, 256, 0, c->stream>>>(nn, nl, hp, h0, pm, ip, c->n, c->max_neigh, sh, E.npad,
                                                                    sp, E.col.as<int32_t>(), E.val.as<double2>(),
                                                                    E.h0.as<double>());
        else
            k_fill_ell<double, double><<<grd, 256, 0, c->stream>>>(nn, nl, hp, h0, pm, ip, c->n, c->max_neigh, sh, E.npad,
                                                                   sp, E.col.as<int32_t>(), E.val.as<double>(),
                                                                   E.h0.as<double>());
    }
    GBN_CK_LAUNCH(c);
    // largest chunk of kChunkSlices consecutive slices (the unit the staged kernel copies to shared memory)
    std::vector<int64_t> hsp((size_t)E.nslices + 1);
    GBN_CK(c, cudaMemcpyAsync(hsp.data(), sp, sizeof(int64_t) * hsp.size(), cudaMemcpyDeviceToHost, c->stream));
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    E.max_chunk_entries = 0;
    for (int64_t a = 0; a < E.nslices; a += kChunkSlices) {
        const int64_t b = a + kChunkSlices < E.nslices ? a + kChunkSlices : E.nslices;
        E.max_chunk_entries = std::max(E.max_chunk_entries, hsp[b] - hsp[a]);
    }
    E.val_size = (int)vsz;
    E.valid = true;
    return GBN_OK;
}

}  // namespace gbn
