// Row order and grouped sliced-ELL layout of the Hamiltonian for the recursion kernels.
//
// Rows are renumbered along a Hilbert curve over the fractional coordinates of the atoms (cells of about
// 4 Angstrom), both layers of a bilayer falling into the same cells.  Consecutive
// slices then touch a compact region of the vectors, so the gathers of neighbouring rows hit L1/L2.
// The reference's own atom order (kept for all exchanged arrays) is restored at the boundary by the
// permutation perm[new] = reference index.  Groups of G consecutive rows then share one list of
// union columns (the layout is described with struct Ell).
#include <cuda_runtime.h>
#include <thrust/device_ptr.h>
#include <thrust/execution_policy.h>
#include <thrust/scan.h>
#include <thrust/sequence.h>
#include <thrust/sort.h>
#include <thrust/transform.h>
#include <thrust/unique.h>

#include <algorithm>
#include <vector>

#include "gbn_internal.cuh"
#include "gbn_spmm.cuh"

namespace gbn {

__global__ void k_identity(int32_t* perm, int32_t* iperm, int64_t n)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        perm[i] = (int32_t)i;
        iperm[i] = (int32_t)i;
    }
}

// Position of cell (x, y) along a Hilbert curve filling the 2^order x 2^order grid (the classic
// quadrant-rotation construction: at each level take the quadrant's two bits, then rotate / reflect the
// coordinates into that quadrant's frame).  Unlike the Z-order curve it never jumps between distant
// cells, so atoms close in the row order are close in space.
__device__ __forceinline__ uint64_t hilbert_index(uint32_t x, uint32_t y, int order)
{
    uint64_t d = 0;
    for (uint32_t s = 1u << (order - 1); s > 0; s >>= 1) {
        const uint32_t rx = (x & s) ? 1u : 0u;
        const uint32_t ry = (y & s) ? 1u : 0u;
        d += (uint64_t)s * s * ((3u * rx) ^ ry);
        if (ry == 0) {   // rotate the quadrant
            if (rx == 1) {
                x = s - 1 - (x & (s - 1)) + (x & ~(s - 1));
                y = s - 1 - (y & (s - 1)) + (y & ~(s - 1));
            }
            const uint32_t t = x;
            x = y;
            y = t;
        }
    }
    return d;
}

__global__ void k_curve_keys(const double* rat, int64_t n, double a1x, double a1y, double a2x, double a2y,
                              int32_t g1, int32_t g2, int order, uint64_t* keys, int32_t* idx)
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
    keys[i] = hilbert_index((uint32_t)ix, (uint32_t)iy, order);
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
    int order = 1;   // Hilbert curve over the smallest 2^order grid that holds the cells
    while ((1 << order) < g1 || (1 << order) < g2) ++order;
    k_curve_keys<<<grd, 256, 0, c->stream>>>(c->rat.as<double>(), c->n, a1x, a1y, a2x, a2y, g1, g2, order,
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

// ---- grouped sliced ELL -------------------------------------------------------------------------

// entry offsets of the rows in the base order (exclusive scan follows)
__global__ void k_row_counts(const int32_t* nneigh, const int32_t* perm, int64_t n, int64_t* cnt)
{
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) cnt[r] = nneigh[perm[r]];
}

// key of every entry: (group of its row in the base order, reference column)
__global__ void k_group_keys(const int32_t* nneigh, const int32_t* nlist, const int32_t* perm, int64_t n,
                             int32_t max_neigh, int G, const int64_t* off, uint64_t* keys)
{
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int64_t p = perm[r];
    const uint64_t g = (uint64_t)(r / G);
    const int k = nneigh[p];
    const int64_t o = off[r];
    for (int j = 0; j < k; ++j) keys[o + j] = (g << 32) | (uint32_t)(nlist[p * max_neigh + j] - 1);
}

// union columns per group: the sorted keys are unique after thrust::unique; count them per group
__global__ void k_union_counts(const uint64_t* ukeys, int64_t nu, int32_t* ucount)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nu) atomicAdd(&ucount[ukeys[i] >> 32], 1);
}

// Groups are reordered inside windows of kSortWindow full groups by decreasing union size, so that
// the groups of a slice have similar widths (less padding) while staying spatially close.
constexpr int kSortWindow = 16;

__global__ void k_group_order(const int32_t* ucount, int64_t ngroups, int64_t nfull, int32_t* gorder)
{
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t g0 = w * kSortWindow;
    if (g0 >= ngroups) return;
    const int64_t g1 = g0 + kSortWindow <= ngroups ? g0 + kSortWindow : ngroups;
    int32_t idx[kSortWindow];
    const int m = (int)(g1 - g0);
    for (int i = 0; i < m; ++i) idx[i] = (int32_t)(g0 + i);
    if (g1 <= nfull) {   // only windows of full groups are reordered (stable insertion sort, largest first)
        for (int i = 1; i < m; ++i) {
            const int32_t v = idx[i];
            int j = i - 1;
            while (j >= 0 && ucount[idx[j]] < ucount[v]) {
                idx[j + 1] = idx[j];
                --j;
            }
            idx[j + 1] = v;
        }
    }
    for (int i = 0; i < m; ++i) gorder[g0 + i] = idx[i];
}

__global__ void k_solver_perm(const int32_t* perm, const int32_t* gorder, int64_t n, int G, int32_t* rperm,
                              int32_t* riperm)
{
    const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n) return;
    const int64_t src = (int64_t)gorder[row / G] * G + row % G;   // a row < n of a full group, or the tail
    const int32_t p = perm[src];
    rperm[row] = p;
    riperm[p] = (int32_t)row;
}

// widths of the slices: the largest union of their groups, rounded up to the column unroll
__global__ void k_slice_width(const int32_t* ucount, const int32_t* gorder, int64_t ngroups, int gpw, int64_t nslices,
                              int64_t* entries)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslices) return;
    int w = 0;
    for (int j = 0; j < gpw; ++j) {
        const int64_t g = s * gpw + j;
        if (g < ngroups) {
            const int u = ucount[gorder[g]];
            w = u > w ? u : w;
        }
    }
    w = (w + kColUnroll - 1) / kColUnroll * kColUnroll;
    entries[s] = (int64_t)w * gpw;
}

template <typename HV>
__device__ __forceinline__ HV neg_hop(double2 h);
template <> __device__ __forceinline__ float neg_hop<float>(double2 h) { return (float)(-h.x); }
template <> __device__ __forceinline__ double neg_hop<double>(double2 h) { return -h.x; }
template <> __device__ __forceinline__ float2 neg_hop<float2>(double2 h) { return make_float2((float)(-h.x), (float)(-h.y)); }
template <> __device__ __forceinline__ double2 neg_hop<double2>(double2 h) { return make_double2(-h.x, -h.y); }
// field-batched value of one entry: the negated field-free hopping (real) and its phase per flux quantum
template <typename HV> __device__ __forceinline__ HV field_val(double2 h, uint64_t tau);
template <> __device__ __forceinline__ FieldVal<float> field_val<FieldVal<float>>(double2 h, uint64_t tau)
{
    return FieldVal<float>{(float)(-h.x), (uint32_t)((tau + 0x80000000ull) >> 32)};
}
template <> __device__ __forceinline__ FieldVal<double> field_val<FieldVal<double>>(double2 h, uint64_t tau)
{
    return FieldVal<double>{-h.x, tau};
}
__device__ __forceinline__ void add_to(float& a, float b) { a += b; }
__device__ __forceinline__ void add_to(double& a, double b) { a += b; }
__device__ __forceinline__ void add_to(float2& a, float2 b) { a.x += b.x; a.y += b.y; }
__device__ __forceinline__ void add_to(double2& a, double2 b) { a.x += b.x; a.y += b.y; }

// One thread per group (solver order): union columns, padding columns, values (the records must be
// zeroed), on-site terms.  An entry that repeats a column of its row (two periodic images of one atom)
// is added to the same value.
// FIELD: values FieldVal from the field-free hoppings and tau (each column at most once per row).
template <typename HV, typename DV, bool FIELD = false>
__global__ void k_fill_groups(const int32_t* nneigh, const int32_t* nlist, const double2* hopp, const double* h0,
                              const int32_t* rperm, const int32_t* riperm, const int32_t* gorder, const int32_t* ucount,
                              const int64_t* ustart, const uint64_t* ukeys, int64_t n, int32_t max_neigh, int G,
                              int gpw, int64_t ngroups, int64_t nslices, const int64_t* slice_ptr, unsigned char* mat,
                              DV* h0p, const uint64_t* tau = nullptr)
{
    const int64_t ng = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (ng >= nslices * gpw) return;
    const int64_t s = ng / gpw;
    const int j = (int)(ng % gpw);
    const int64_t base = slice_ptr[s];
    const int w = (int)((slice_ptr[s + 1] - base) / gpw);
    unsigned char* rec = mat + base * (int64_t)(sizeof(int32_t) + G * sizeof(HV));
    int32_t* col = reinterpret_cast<int32_t*>(rec);
    HV* val = reinterpret_cast<HV*>(rec + (size_t)w * gpw * sizeof(int32_t));
    const int64_t row0 = ng * G;
    int u = 0;
    const uint64_t* ul = nullptr;
    if (ng < ngroups) {
        const int32_t og = gorder[ng];
        u = ucount[og];
        ul = ukeys + ustart[og];
    }
    for (int k = 0; k < u; ++k) col[rec_slot(k, j, gpw)] = riperm[(uint32_t)ul[k]];
    for (int k = u; k < w; ++k) col[rec_slot(k, j, gpw)] = (int32_t)row0;
    for (int rr = 0; rr < G; ++rr) {
        const int64_t row = row0 + rr;
        if (row >= n) {
            h0p[row] = (DV)0;
            continue;
        }
        const int64_t p = rperm[row];
        h0p[row] = (DV)h0[p];
        const int kk = nneigh[p];
        for (int e = 0; e < kk; ++e) {
            const uint32_t rc = (uint32_t)(nlist[p * max_neigh + e] - 1);
            int lo = 0, hi = u;   // lower bound of rc among the group's sorted union columns
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if ((uint32_t)ul[mid] < rc) lo = mid + 1;
                else hi = mid;
            }
            if constexpr (FIELD) val[val_slot(lo, j, gpw, G, (int)sizeof(HV)) + rr] = field_val<HV>(hopp[p * max_neigh + e], tau[p * max_neigh + e]);
            else add_to(val[val_slot(lo, j, gpw, G, (int)sizeof(HV)) + rr], neg_hop<HV>(hopp[p * max_neigh + e]));
        }
    }
}

// (row, column) keys of all entries in the reference order, to find rows that hold two periodic images
// of one neighbour (the field-batched layout cannot merge them: their phases differ)
__global__ void k_row_keys(const int32_t* nneigh, const int32_t* nlist, int64_t n, int32_t max_neigh,
                           const int64_t* off, uint64_t* keys)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int e = 0; e < nneigh[i]; ++e)
        keys[off[i] + e] = ((uint64_t)i << 32) | (uint32_t)(nlist[i * max_neigh + e] - 1);
}

// bytes of the largest slice record
__global__ void k_max_record(const int64_t* slice_ptr, int64_t nslices, int64_t entry_bytes,
                             unsigned long long* out)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nslices) atomicMax(out, (unsigned long long)((slice_ptr[s + 1] - slice_ptr[s]) * entry_bytes));
}

// Default rows per group from the mean entries per row and the tile width R (measured with the autotuner
// on B200: graphene-like rows of about 3 entries gather too little per slice with one or two vectors, and
// groups of 4 rows share their union columns; bilayers with tens of interlayer entries share columns
// between pairs of rows once several vectors amortise the union's padding).
int auto_group(const gbn_ctx* c, int R, int prec)
{
    const double per_row = c->n > 0 ? (double)c->total / (double)c->n : 0.0;
    // one vector on a low-degree cell: in FP64 one row per group with 8 columns in flight and registers for
    // three blocks per SM (1.28M-atom graphene: 53.1 us per step against 73.4 us at four rows per group), in
    // mixed precision two rows per group (35.6 against 45.2 us)
    if (per_row < 8.0 && R == 1) return prec == GBN_FP64 ? 1 : 2;
    if (per_row < 8.0) return R <= 2 ? 4 : (R <= 4 ? 2 : 1);
    return R == 1 ? 1 : 2;
}

// ---------------------------------------------------------------------------- field tile table
// One warp per slice: the column indices are copied, and every FieldVal (h, tau) becomes, for each slot q,
// h exp(2 pi i frac(m_q tau)) with m_q the slot's flux quanta, stored at [entry][slot][G] so that the TPR
// threads of a row group read their slots' values from one contiguous piece: the turn fraction m_q tau wraps exactly in
// integer arithmetic and its angle is evaluated by sincospi in FP64, then rounded once to the storage type.
template <typename VT>
__global__ void k_field_table(const int64_t* __restrict__ slice_ptr, int64_t nslices, int gpw, int G, int slots,
                              const unsigned char* __restrict__ mat, int64_t eb, unsigned char* __restrict__ tab,
                              int64_t teb, const int32_t* __restrict__ slot_m)
{
    using C2 = typename V2<VT>::t;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t s = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); s < nslices; s += warps) {
        const int64_t base = slice_ptr[s], nent = slice_ptr[s + 1] - base;
        const int32_t* ci = reinterpret_cast<const int32_t*>(mat + base * eb);
        const FieldVal<VT>* vi = reinterpret_cast<const FieldVal<VT>*>(mat + base * eb + nent * 4);
        int32_t* co = reinterpret_cast<int32_t*>(tab + base * teb);
        C2* vo = reinterpret_cast<C2*>(tab + base * teb + nent * 4);
        for (int64_t k = lane; k < nent; k += 32) co[k] = ci[k];
        const int64_t nval = nent * G;
        for (int64_t k = lane; k < nval; k += 32) {   // value k = (entry, g): out at (entry, slot q, g)
            const FieldVal<VT> v = vi[k];
            const int64_t ent = k / G, g = k % G;
            for (int q = 0; q < slots; ++q) {
                double sn, cs;
                if constexpr (sizeof(VT) == 4) {
                    const uint32_t u = v.t * (uint32_t)(int64_t)slot_m[q];
                    sincospi((double)(int32_t)u * 4.656612873077393e-10, &sn, &cs);   // 2^-31
                } else {
                    const uint64_t u = v.t * (uint64_t)(int64_t)slot_m[q];
                    sincospi((double)(int64_t)u * 1.0842021724855044e-19, &sn, &cs);   // 2^-63
                }
                C2 o;
                o.x = (VT)((double)v.h * cs);
                o.y = (VT)((double)v.h * sn);
                vo[(ent * slots + q) * G + g] = o;
            }
        }
    }
}

int build_field_table(gbn_ctx* c, int slots, const int32_t* d_slot_m)
{
    Ell& E = c->ell;
    if (!E.valid || !E.field) return fail(c, GBN_ERR_STATE, "internal: no field-batched layout for a tile table");
    const int csz = E.prec == GBN_MIXED ? (int)sizeof(float2) : (int)sizeof(double2);
    const int64_t teb = 4 + (int64_t)slots * E.G * csz;
    GBN_CK(c, E.ftab.ensure((size_t)(E.nnz_stored * teb)));
    const int blk = 256;
    const int64_t grid = std::min<int64_t>((E.nslices + (blk / 32) - 1) / (blk / 32), (int64_t)c->num_sms * 16);
    if (E.prec == GBN_MIXED)
        k_field_table<float><<<(unsigned)std::max<int64_t>(grid, 1), blk, 0, c->stream>>>(
            E.slice_ptr.as<int64_t>(), E.nslices, E.gpw, E.G, slots, E.mat.as<unsigned char>(), E.entry_bytes,
            E.ftab.as<unsigned char>(), teb, d_slot_m);
    else
        k_field_table<double><<<(unsigned)std::max<int64_t>(grid, 1), blk, 0, c->stream>>>(
            E.slice_ptr.as<int64_t>(), E.nslices, E.gpw, E.G, slots, E.mat.as<unsigned char>(), E.entry_bytes,
            E.ftab.as<unsigned char>(), teb, d_slot_m);
    GBN_CK_LAUNCH(c);
    E.ftab_slots = slots;
    E.ftab_entry_bytes = (int)teb;
    E.ftab_valid = true;
    return GBN_OK;
}

// ---------------------------------------------------------------------------- tiles
// Greedy tiling of the slices in row order: a tile takes slices while the distinct rows its records gather
// (padding columns included) stay within hmax; a slice that alone exceeds hmax makes the layout untileable
// at that hmax.  The halo rows are numbered in order of first use and every column index of the tile's
// records is replaced by that number (tmat).  Host work O(entries), once per layout and hmax.
int build_tiles(gbn_ctx* c, int hmax)
{
    Ell& E = c->ell;
    if (!E.valid || E.field) return fail(c, GBN_ERR_STATE, "internal: tiles need a valid layout without fields");
    if (hmax < 1) return fail(c, GBN_ERR_ARG, "internal: tile halo limit must be positive");
    const int64_t ns = E.nslices, eb = E.entry_bytes;
    std::vector<int64_t> sp((size_t)ns + 1);
    GBN_CK(c, cudaMemcpyAsync(sp.data(), E.slice_ptr.p, sizeof(int64_t) * sp.size(), cudaMemcpyDeviceToHost, c->stream));
    const size_t mbytes = (size_t)(E.nnz_stored * eb);
    std::vector<unsigned char> m(mbytes ? mbytes : 1);
    if (mbytes) GBN_CK(c, cudaMemcpyAsync(m.data(), E.mat.p, mbytes, cudaMemcpyDeviceToHost, c->stream));
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    std::vector<int32_t> stamp((size_t)E.npad, -1), seen((size_t)E.npad, -1), local((size_t)E.npad, 0);
    std::vector<int64_t> tslice{0}, hptr{0};
    std::vector<int32_t> halo;
    int32_t t = 0, h = 0;
    for (int64_t s = 0; s < ns; ++s) {
        int32_t* col = reinterpret_cast<int32_t*>(m.data() + sp[(size_t)s] * eb);
        const int64_t nent = sp[(size_t)s + 1] - sp[(size_t)s];
        int32_t fresh = 0, distinct = 0;   // rows of this slice not yet in the tile's halo; all its rows
        for (int64_t k = 0; k < nent; ++k) {
            const int32_t cc = col[k];
            if (seen[(size_t)cc] != (int32_t)s) {
                seen[(size_t)cc] = (int32_t)s;
                ++distinct;
                if (stamp[(size_t)cc] != t) ++fresh;
            }
        }
        if (distinct > hmax) return fail(c, GBN_ERR_ARG, "internal: a slice gathers more rows than a tile holds");
        if (h + fresh > hmax) {   // close the tile before this slice
            tslice.push_back(s);
            hptr.push_back((int64_t)halo.size());
            ++t;
            h = 0;
        }
        for (int64_t k = 0; k < nent; ++k) {
            const int32_t cc = col[k];
            if (stamp[(size_t)cc] != t) {
                stamp[(size_t)cc] = t;
                local[(size_t)cc] = h++;
                halo.push_back(cc);
            }
            col[k] = local[(size_t)cc];
        }
    }
    tslice.push_back(ns);
    hptr.push_back((int64_t)halo.size());
    E.ntiles = (int64_t)tslice.size() - 1;
    GBN_CK(c, E.tile_slice.ensure(sizeof(int64_t) * tslice.size()));
    GBN_CK(c, E.halo_ptr.ensure(sizeof(int64_t) * hptr.size()));
    GBN_CK(c, E.halo.ensure(sizeof(int32_t) * (halo.size() ? halo.size() : 1)));
    GBN_CK(c, E.tmat.ensure(m.size()));
    GBN_CK(c, cudaMemcpyAsync(E.tile_slice.p, tslice.data(), sizeof(int64_t) * tslice.size(), cudaMemcpyHostToDevice,
                              c->stream));
    GBN_CK(c, cudaMemcpyAsync(E.halo_ptr.p, hptr.data(), sizeof(int64_t) * hptr.size(), cudaMemcpyHostToDevice,
                              c->stream));
    if (!halo.empty())
        GBN_CK(c, cudaMemcpyAsync(E.halo.p, halo.data(), sizeof(int32_t) * halo.size(), cudaMemcpyHostToDevice,
                                  c->stream));
    GBN_CK(c, cudaMemcpyAsync(E.tmat.p, m.data(), m.size(), cudaMemcpyHostToDevice, c->stream));
    GBN_CK(c, cudaStreamSynchronize(c->stream));   // the host buffers go out of scope
    E.tile_hmax = hmax;
    E.tiles_valid = true;
    return GBN_OK;
}

int build_ell(gbn_ctx* c, int prec, int G, int gpw, bool field)
{
    if (!c->have_ham) return fail(c, GBN_ERR_STATE, "no Hamiltonian loaded");
    if (G != 1 && G != 2 && G != 4) return fail(c, GBN_ERR_ARG, "rows per group must be 1, 2 or 4");
    if (!c->perm.p) {
        const int rc = build_identity_perm(c);
        if (rc) return rc;
    }
    Ell& E = c->ell;
    E.valid = false;
    E.ftab_valid = false;
    E.tiles_valid = false;
    E.dval_dir = 0;
    E.G = G;
    E.gpw = gpw;
    E.prec = prec;
    E.cplx = c->ham_complex;
    E.field = field;
    if (field && (c->ham_complex || !c->ptau.p))
        return fail(c, GBN_ERR_STATE, "batched fields need the field-free assembled Hamiltonian and its phases");
    const int64_t n = c->n;
    E.ngroups = (n + G - 1) / G;
    E.nslices = (E.ngroups + gpw - 1) / gpw;
    E.npad = E.nslices * gpw * G;
    const unsigned grn = (unsigned)((n + 255) / 256);
    const int32_t* nn = c->nneigh.as<int32_t>();
    const int32_t* nl = c->nlist.as<int32_t>();
    auto pol = thrust::cuda::par.on(c->stream);

    // entry keys (group, reference column), sorted and made unique: the union of every group
    DevBuf off, keys, ucount, ustart, gorder, maxbuf;
    GBN_CK(c, off.ensure(sizeof(int64_t) * (n + 1)));
    GBN_CK(c, cudaMemsetAsync(off.as<int64_t>() + n, 0, sizeof(int64_t), c->stream));
    k_row_counts<<<grn, 256, 0, c->stream>>>(nn, c->perm.as<int32_t>(), n, off.as<int64_t>());
    GBN_CK_LAUNCH(c);
    thrust::device_ptr<int64_t> op(off.as<int64_t>());
    thrust::exclusive_scan(pol, op, op + n + 1, op);
    int64_t nnz = 0;
    GBN_CK(c, cudaMemcpyAsync(&nnz, off.as<int64_t>() + n, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    GBN_CK(c, keys.ensure(sizeof(uint64_t) * (size_t)(nnz > 0 ? nnz : 1)));
    if (field && nnz > 0) {   // every (row, column) at most once
        DevBuf roff;
        GBN_CK(c, roff.ensure(sizeof(int64_t) * (n + 1)));
        GBN_CK(c, cudaMemsetAsync(roff.as<int64_t>() + n, 0, sizeof(int64_t), c->stream));
        thrust::device_ptr<const int32_t> np(nn);
        thrust::device_ptr<int64_t> rp(roff.as<int64_t>());
        thrust::transform(pol, np, np + n, rp, [] __device__(int32_t v) { return (int64_t)v; });
        thrust::exclusive_scan(pol, rp, rp + n + 1, rp);
        k_row_keys<<<grn, 256, 0, c->stream>>>(nn, nl, n, c->max_neigh, roff.as<int64_t>(), keys.as<uint64_t>());
        GBN_CK_LAUNCH(c);
        thrust::device_ptr<uint64_t> kq(keys.as<uint64_t>());
        thrust::sort(pol, kq, kq + nnz);
        const int64_t nuniq = thrust::unique(pol, kq, kq + nnz) - kq;
        c->launches += 6;
        if (nuniq != nnz)
            return fail(c, GBN_ERR_ARG, "a row holds two periodic images of one neighbour: the cell is too small for "
                                        "batched fields (use gbn_peierls per field)");
    }
    k_group_keys<<<grn, 256, 0, c->stream>>>(nn, nl, c->perm.as<int32_t>(), n, c->max_neigh, G, off.as<int64_t>(),
                                             keys.as<uint64_t>());
    GBN_CK_LAUNCH(c);
    thrust::device_ptr<uint64_t> kp(keys.as<uint64_t>());
    thrust::sort(pol, kp, kp + nnz);
    const int64_t nu = thrust::unique(pol, kp, kp + nnz) - kp;
    c->launches += 8;  // scan, sort and unique passes issued by thrust (setup only)
    off.release();
    GBN_CK(c, ucount.ensure(sizeof(int32_t) * (size_t)E.ngroups));
    GBN_CK(c, cudaMemsetAsync(ucount.p, 0, sizeof(int32_t) * (size_t)E.ngroups, c->stream));
    if (nu > 0) {
        k_union_counts<<<(unsigned)((nu + 255) / 256), 256, 0, c->stream>>>(keys.as<uint64_t>(), nu, ucount.as<int32_t>());
        GBN_CK_LAUNCH(c);
    }
    GBN_CK(c, ustart.ensure(sizeof(int64_t) * (size_t)(E.ngroups + 1)));
    {
        thrust::device_ptr<int32_t> up(ucount.as<int32_t>());
        thrust::device_ptr<int64_t> usp(ustart.as<int64_t>());
        GBN_CK(c, cudaMemsetAsync(ustart.as<int64_t>() + E.ngroups, 0, sizeof(int64_t), c->stream));
        thrust::exclusive_scan(pol, up, up + E.ngroups, usp, (int64_t)0);
    }

    // solver row order: groups reordered by union size inside small windows
    GBN_CK(c, gorder.ensure(sizeof(int32_t) * (size_t)E.ngroups));
    const int64_t nwin = (E.ngroups + kSortWindow - 1) / kSortWindow;
    k_group_order<<<(unsigned)((nwin + 127) / 128), 128, 0, c->stream>>>(ucount.as<int32_t>(), E.ngroups, n / G,
                                                                         gorder.as<int32_t>());
    GBN_CK_LAUNCH(c);
    GBN_CK(c, E.rperm.ensure(sizeof(int32_t) * n));
    GBN_CK(c, E.riperm.ensure(sizeof(int32_t) * n));
    k_solver_perm<<<grn, 256, 0, c->stream>>>(c->perm.as<int32_t>(), gorder.as<int32_t>(), n, G, E.rperm.as<int32_t>(),
                                              E.riperm.as<int32_t>());
    GBN_CK_LAUNCH(c);

    // slices
    GBN_CK(c, E.slice_ptr.ensure(sizeof(int64_t) * (size_t)(E.nslices + 1)));
    int64_t* sp = E.slice_ptr.as<int64_t>();
    GBN_CK(c, cudaMemsetAsync(sp + E.nslices, 0, sizeof(int64_t), c->stream));
    k_slice_width<<<(unsigned)((E.nslices + 255) / 256), 256, 0, c->stream>>>(ucount.as<int32_t>(), gorder.as<int32_t>(),
                                                                            E.ngroups, gpw, E.nslices, sp);
    GBN_CK_LAUNCH(c);
    thrust::device_ptr<int64_t> tp(sp);
    thrust::exclusive_scan(pol, tp, tp + E.nslices + 1, tp);
    GBN_CK(c, cudaMemcpyAsync(&E.nnz_stored, sp + E.nslices, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
    GBN_CK(c, cudaStreamSynchronize(c->stream));

    size_t vsz;
    if (field) vsz = prec == GBN_MIXED ? sizeof(FieldVal<float>) : sizeof(FieldVal<double>);
    else if (prec == GBN_MIXED) vsz = E.cplx ? sizeof(float2) : sizeof(float);
    else vsz = E.cplx ? sizeof(double2) : sizeof(double);
    const size_t eb = sizeof(int32_t) + vsz * G;
    const size_t ne = (size_t)(E.nnz_stored > 0 ? E.nnz_stored : 1);
    GBN_CK(c, E.mat.ensure(eb * ne));
    GBN_CK(c, cudaMemsetAsync(E.mat.p, 0, eb * ne, c->stream));
    GBN_CK(c, E.h0.ensure((prec == GBN_MIXED ? sizeof(float) : sizeof(double)) * (size_t)E.npad));
    const unsigned grg = (unsigned)((E.nslices * gpw + 127) / 128);
    const double2* hp = c->hopp.as<double2>();
    const double* h0 = c->h0.as<double>();
#define GBN_FILL(HV, DV)                                                                                          \
    k_fill_groups<HV, DV><<<grg, 128, 0, c->stream>>>(nn, nl, hp, h0, E.rperm.as<int32_t>(), E.riperm.as<int32_t>(), \
                                                      gorder.as<int32_t>(), ucount.as<int32_t>(), ustart.as<int64_t>(), \
                                                      keys.as<uint64_t>(), n, c->max_neigh, G, gpw, E.ngroups,         \
                                                      E.nslices, sp, E.mat.as<unsigned char>(), E.h0.as<DV>())
    if (field) {
        if (prec == GBN_MIXED)
            k_fill_groups<FieldVal<float>, float, true><<<grg, 128, 0, c->stream>>>(
                nn, nl, hp, h0, E.rperm.as<int32_t>(), E.riperm.as<int32_t>(), gorder.as<int32_t>(), ucount.as<int32_t>(),
                ustart.as<int64_t>(), keys.as<uint64_t>(), n, c->max_neigh, G, gpw, E.ngroups, E.nslices, sp,
                E.mat.as<unsigned char>(), E.h0.as<float>(), c->ptau.as<uint64_t>());
        else
            k_fill_groups<FieldVal<double>, double, true><<<grg, 128, 0, c->stream>>>(
                nn, nl, hp, h0, E.rperm.as<int32_t>(), E.riperm.as<int32_t>(), gorder.as<int32_t>(), ucount.as<int32_t>(),
                ustart.as<int64_t>(), keys.as<uint64_t>(), n, c->max_neigh, G, gpw, E.ngroups, E.nslices, sp,
                E.mat.as<unsigned char>(), E.h0.as<double>(), c->ptau.as<uint64_t>());
    } else if (prec == GBN_MIXED) {
        if (E.cplx) GBN_FILL(float2, float);
        else GBN_FILL(float, float);
    } else {
        if (E.cplx) GBN_FILL(double2, double);
        else GBN_FILL(double, double);
    }
#undef GBN_FILL
    GBN_CK_LAUNCH(c);
    GBN_CK(c, maxbuf.ensure(sizeof(unsigned long long)));
    unsigned long long* dmax = maxbuf.as<unsigned long long>();
    GBN_CK(c, cudaMemsetAsync(dmax, 0, sizeof(unsigned long long), c->stream));
    k_max_record<<<(unsigned)((E.nslices + 255) / 256), 256, 0, c->stream>>>(sp, E.nslices, (int64_t)eb, dmax);
    GBN_CK_LAUNCH(c);
    unsigned long long mr = 0;
    GBN_CK(c, cudaMemcpyAsync(&mr, dmax, sizeof(mr), cudaMemcpyDeviceToHost, c->stream));
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    E.max_record = (int64_t)mr;
    E.entry_bytes = (int)eb;
    {   // staging buffer size: the 99.5th percentile of the record sizes
        std::vector<int64_t> hsp((size_t)E.nslices + 1);
        GBN_CK(c, cudaMemcpyAsync(hsp.data(), sp, sizeof(int64_t) * hsp.size(), cudaMemcpyDeviceToHost, c->stream));
        GBN_CK(c, cudaStreamSynchronize(c->stream));
        std::vector<int64_t> rec((size_t)E.nslices);
        for (int64_t i = 0; i < E.nslices; ++i) rec[(size_t)i] = (hsp[(size_t)i + 1] - hsp[(size_t)i]) * (int64_t)eb;
        if (!rec.empty()) {
            std::sort(rec.begin(), rec.end());
            const double pct[4] = {0.995, 0.99, 0.95, 0.90};
            for (int i = 0; i < 4; ++i) {
                const size_t k = std::min(rec.size() - 1, (size_t)((double)rec.size() * pct[i]));
                E.cap_pct[i] = (rec[k] + 15) / 16 * 16;
            }
            E.cap_record = E.cap_pct[0];
        } else {
            E.cap_record = 0;
            for (int i = 0; i < 4; ++i) E.cap_pct[i] = 0;
        }
    }
    E.val_size = (int)vsz;
    E.valid = true;
    return GBN_OK;
}

}  // namespace gbn
