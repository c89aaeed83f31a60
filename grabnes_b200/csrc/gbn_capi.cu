// C ABI of libgrabnes_gpu (declared in include/grabnes_gpu.h): context management, argument
// checking, host<->device copies, tiling of many right-hand sides.  No function aborts; every error is
// returned as a GBN_ERR_* code with its text in gbn_last_error().
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <string>
#include <vector>

#include "gbn_internal.cuh"

namespace gbn {

int fail(gbn_ctx* c, int code, const std::string& msg)
{
    if (c) c->err = msg;
    return code;
}

int cuda_fail(gbn_ctx* c, cudaError_t e, const char* what)
{
    if (c) c->err = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
    return (e == cudaErrorMemoryAllocation) ? GBN_ERR_ALLOC : GBN_ERR_CUDA;
}

static int tile_width(int nrhs)
{
    int t = 1;
    while (t < nrhs && t < 32) t <<= 1;
    return t;
}

// Runs the recursion for all right-hand sides in tiles of at most 32; start(r0, cnt) writes the start
// vectors of right-hand sides r0 .. r0 + cnt - 1 into the tile (after lanczos_prepare).
template <typename Start>
static int run_tiles(gbn_ctx* c, int prec, int nrhs, Start&& start, const int32_t* nsteps, int32_t nmax, double* a,
                     double* b, bool field = false)
{
    const int T = tile_width(nrhs);
    int rc = lanczos_prepare(c, prec, T, field);
    if (rc) return rc;
    double step_ms = 0.0, spmm_sum = 0.0, upd_sum = 0.0;
    int64_t launches = 0;
    int tiles = 0;
    std::vector<double> hab;
    for (int r0 = 0; r0 < nrhs; r0 += T) {
        const int cnt = std::min(T, nrhs - r0);
        int32_t nt = 0;
        for (int r = r0; r < r0 + cnt; ++r) nt = std::max(nt, nsteps ? nsteps[r] : nmax);
        rc = start(r0, cnt);
        if (rc) return rc;
        rc = lanczos_run(c, nt);
        if (rc) return rc;
        step_ms += c->timing.step_ms;
        launches += c->timing.step_launches;
        spmm_sum += c->timing.spmm_ms_avg;
        upd_sum += c->timing.update_ms_avg;
        ++tiles;
        hab.resize((size_t)2 * T * nt);
        GBN_CK(c, cudaMemcpyAsync(hab.data(), c->ab.p, sizeof(double) * hab.size(), cudaMemcpyDeviceToHost, c->stream));
        GBN_CK(c, cudaStreamSynchronize(c->stream));
        for (int r = 0; r < cnt; ++r) {
            memcpy(a + (size_t)(r0 + r) * nmax, hab.data() + (size_t)r * nt, sizeof(double) * nt);
            memcpy(b + (size_t)(r0 + r) * nmax, hab.data() + (size_t)T * nt + (size_t)r * nt, sizeof(double) * nt);
        }
    }
    c->timing.step_ms = step_ms;
    c->timing.step_launches = launches;
    c->timing.spmm_ms_avg = tiles ? spmm_sum / tiles : 0.0;
    c->timing.update_ms_avg = tiles ? upd_sum / tiles : 0.0;
    return GBN_OK;
}

// Inputs are either complex start vectors (psi) or uniform draws (phases), [nrhs][n] on the host.
static int run_tiled(gbn_ctx* c, int prec, int nrhs, const double* host_in, bool phases, const int32_t* nsteps,
                     int32_t nmax, double* a, double* b)
{
    const size_t per = (size_t)c->n * (phases ? 1 : 2);
    GBN_CK(c, c->upload.ensure(sizeof(double) * per * tile_width(nrhs)));
    return run_tiles(
        c, prec, nrhs,
        [&](int r0, int cnt) -> int {
            GBN_CK(c, cudaMemcpyAsync(c->upload.p, host_in + per * r0, sizeof(double) * per * cnt,
                                      cudaMemcpyHostToDevice, c->stream));
            return phases ? lanczos_start_from_phases(c, c->upload.as<double>(), cnt)
                          : lanczos_start_from_psi(c, c->upload.as<double>(), cnt);
        },
        nsteps, nmax, a, b);
}

static int check_solver_args(gbn_ctx* c, int32_t precision, int32_t nrhs, const void* in, const int32_t* nsteps,
                             int32_t nmax, const double* a, const double* b)
{
    if (!c->have_ham) return fail(c, GBN_ERR_STATE, "no Hamiltonian: call gbn_load_hamiltonian or gbn_assemble first");
    if (precision != GBN_FP64 && precision != GBN_MIXED) return fail(c, GBN_ERR_ARG, "precision must be GBN_FP64 or GBN_MIXED");
    if (nrhs < 1) return fail(c, GBN_ERR_ARG, "nrhs must be at least 1");
    if (nmax < 1) return fail(c, GBN_ERR_ARG, "nmax must be at least 1");
    if (!in || !a || !b) return fail(c, GBN_ERR_ARG, "NULL input or output array");
    if (nsteps)
        for (int r = 0; r < nrhs; ++r)
            if (nsteps[r] < 1 || nsteps[r] > nmax) return fail(c, GBN_ERR_ARG, "nsteps[r] must be in 1..nmax");
    return GBN_OK;
}

}  // namespace gbn

using namespace gbn;

extern "C" {

const char* gbn_version(void) { return "grabnes_b200 0.1 (sm_100a)"; }

int gbn_create(gbn_ctx** out, int32_t device)
{
    if (!out) return GBN_ERR_ARG;
    *out = nullptr;
    gbn_ctx* c = new (std::nothrow) gbn_ctx();
    if (!c) return GBN_ERR_ALLOC;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        delete c;
        return GBN_ERR_CUDA;
    }
    if (device < 0 || device >= ndev) {
        delete c;
        return GBN_ERR_ARG;
    }
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return GBN_ERR_CUDA;
    }
    c->own_stream = true;
    *out = c;
    return GBN_OK;
}

int gbn_destroy(gbn_ctx* c)
{
    if (!c) return GBN_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    DevBuf* bufs[] = {&c->rat, &c->species, &c->layer, &c->nneigh, &c->nlist, &c->neighd, &c->ncell, &c->h0,
                      &c->hopp, &c->rat_hop, &c->perm, &c->iperm, &c->ell.slice_ptr, &c->ell.mat,
                      &c->ell.h0, &c->ell.rperm, &c->ell.riperm, &c->ell.dval, &c->partials, &c->scal, &c->counter, &c->ab, &c->upload,
                      &c->h0_bottom, &c->dimer};
    for (DevBuf* b : bufs) b->release();
    for (auto& v : c->vec) v.release();
    for (auto& v : c->cheb) v.release();
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    for (auto& e : c->kev)
        if (e) cudaEventDestroy(e);
    if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return GBN_OK;
}

const char* gbn_last_error(const gbn_ctx* c) { return c ? c->err.c_str() : "no context"; }

int gbn_set_stream(gbn_ctx* c, void* s)
{
    if (!c) return GBN_ERR_ARG;
    cudaSetDevice(c->device);
    if (c->own_stream && c->stream) cudaStreamSynchronize(c->stream);
    if (s) {
        if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
        c->stream = static_cast<cudaStream_t>(s);
        c->own_stream = false;
    } else if (!c->own_stream) {
        GBN_CK(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->own_stream = true;
    }
    return GBN_OK;
}

int64_t gbn_launch_count(const gbn_ctx* c) { return c ? c->launches : 0; }

int gbn_last_timing(const gbn_ctx* c, double* ms, int64_t* launches)
{
    if (!c) return GBN_ERR_ARG;
    if (ms) *ms = c->timing.step_ms;
    if (launches) *launches = c->timing.step_launches;
    return GBN_OK;
}

int gbn_set_tuning(gbn_ctx* c, int32_t rhs_per_thread, int32_t blocks_per_sm, int32_t rows_per_group, int32_t staged,
                   int32_t prefetch)
{
    if (!c) return GBN_ERR_ARG;
    if (rhs_per_thread < 0 || rhs_per_thread > 4 || blocks_per_sm < 0 || blocks_per_sm > 32 ||
        (rows_per_group != 0 && rows_per_group != 1 && rows_per_group != 2 && rows_per_group != 4) || staged < -1 ||
        staged > 1 || prefetch < -1 || prefetch > 7)
        return fail(c, GBN_ERR_ARG, "tuning values out of range");
    c->tune_rpt = rhs_per_thread;
    c->tune_blocks_per_sm = blocks_per_sm;
    c->tune_group = rows_per_group;
    c->tune_staged = staged;
    c->tune_prefetch = prefetch;   // a layout of other rows per group or threads per group is rebuilt when used
    return GBN_OK;
}

int gbn_set_kernel_variant(gbn_ctx* c, int32_t col_unroll, int32_t stage_values, int32_t min_blocks,
                           int32_t field_table, int32_t tiled, int32_t fused)
{
    if (!c) return GBN_ERR_ARG;
    if ((col_unroll != 0 && col_unroll != 4 && col_unroll != 8) || stage_values < -1 || stage_values > 1 ||
        (min_blocks < 0 || min_blocks > 3) || field_table < -1 || field_table > 1 || tiled < -1 || tiled > 1 ||
        fused < -1 || fused > 1)
        return fail(c, GBN_ERR_ARG, "kernel variant out of range");
    c->tune_fused = fused;
    c->tune_tiled = tiled;
    c->tune_unroll = col_unroll;
    c->tune_stage_values = stage_values;
    c->tune_min_blocks = min_blocks;
    c->tune_field_table = field_table;
    return GBN_OK;
}

int gbn_last_kernel_timing(const gbn_ctx* c, double* spmm_ms, double* update_ms)
{
    if (!c) return GBN_ERR_ARG;
    if (spmm_ms) *spmm_ms = c->timing.spmm_ms_avg;
    if (update_ms) *update_ms = c->timing.update_ms_avg;
    return GBN_OK;
}

int gbn_set_geometry(gbn_ctx* c, int64_t n, const double* rat, const int32_t* species, const int32_t* layer,
                     const double* ucell)
{
    if (!c) return GBN_ERR_ARG;
    if (n < 1 || n >= (int64_t)1 << 31) return fail(c, GBN_ERR_ARG, "number of atoms must be in 1..2^31-1");
    if (!rat || !species || !layer || !ucell) return fail(c, GBN_ERR_ARG, "NULL geometry array");
    cudaSetDevice(c->device);
    GBN_CK(c, c->rat.ensure(sizeof(double) * 3 * n));
    GBN_CK(c, c->species.ensure(sizeof(int32_t) * n));
    GBN_CK(c, c->layer.ensure(sizeof(int32_t) * n));
    GBN_CK(c, cudaMemcpyAsync(c->rat.p, rat, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->stream));
    GBN_CK(c, cudaMemcpyAsync(c->species.p, species, sizeof(int32_t) * n, cudaMemcpyHostToDevice, c->stream));
    GBN_CK(c, cudaMemcpyAsync(c->layer.p, layer, sizeof(int32_t) * n, cudaMemcpyHostToDevice, c->stream));
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    memcpy(c->ucell, ucell, sizeof(c->ucell));
    c->n = n;
    c->have_geometry = true;
    c->have_neigh = c->have_neighd = c->have_ham = false;
    c->ell.valid = false;
    return build_spatial_perm(c);
}

int gbn_neighbours(gbn_ctx* c, double cut2intra, double cut2inter, int32_t second_layer, int32_t* max_neigh,
                   int64_t* total)
{
    if (!c) return GBN_ERR_ARG;
    if (!c->have_geometry) return fail(c, GBN_ERR_STATE, "no geometry: call gbn_set_geometry first");
    if (!(cut2intra > 0.0) || !(cut2inter > 0.0)) return fail(c, GBN_ERR_ARG, "search radii must be positive");
    cudaSetDevice(c->device);
    const int rc = neigh_search(c, cut2intra, cut2inter, second_layer);
    if (rc) return rc;
    if (max_neigh) *max_neigh = c->max_neigh;
    if (total) *total = c->total;
    return GBN_OK;
}

int gbn_get_neighbours(gbn_ctx* c, int32_t* nneigh, int32_t* nlist, double* neighd, int32_t* ncell)
{
    if (!c) return GBN_ERR_ARG;
    if (!c->have_neigh) return fail(c, GBN_ERR_STATE, "no neighbour tables");
    cudaSetDevice(c->device);
    const size_t e = (size_t)c->n * c->max_neigh;
    if (nneigh) GBN_CK(c, cudaMemcpyAsync(nneigh, c->nneigh.p, sizeof(int32_t) * c->n, cudaMemcpyDeviceToHost, c->stream));
    if (nlist) GBN_CK(c, cudaMemcpyAsync(nlist, c->nlist.p, sizeof(int32_t) * e, cudaMemcpyDeviceToHost, c->stream));
    if (neighd) {
        if (!c->have_neighd) return fail(c, GBN_ERR_STATE, "no NeighD table");
        GBN_CK(c, cudaMemcpyAsync(neighd, c->neighd.p, sizeof(double) * 3 * e, cudaMemcpyDeviceToHost, c->stream));
    }
    if (ncell) {
        if (!c->ncell.p) return fail(c, GBN_ERR_STATE, "no neighCell table");
        GBN_CK(c, cudaMemcpyAsync(ncell, c->ncell.p, sizeof(int32_t) * 3 * e, cudaMemcpyDeviceToHost, c->stream));
    }
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    return GBN_OK;
}

int gbn_assemble(gbn_ctx* c, const gbn_model* m, const double* rat_on, const double* rat_hop, const double* uniform)
{
    if (!c || !m) return GBN_ERR_ARG;
    if (!c->have_neigh || !c->have_neighd) return fail(c, GBN_ERR_STATE, "no neighbour tables: call gbn_neighbours first");
    if (m->tbnn < 1 || m->tbnn > 8) return fail(c, GBN_ERR_ARG, "tbnn must be in 1..8");
    if (m->anderson && !uniform) return fail(c, GBN_ERR_ARG, "Anderson disorder needs the uniform draws");
    if (m->encapsulated && m->bernal != 1 && m->bernal != 2)
        return fail(c, GBN_ERR_ARG, "the encapsulated bilayer needs bernal 1 (vertical pairs) or 2 (bilayer F2G2 set)");
    if (m->encapsulated && !m->rotate_first && m->eps == 0.0 && (m->moire_onsite || m->moire_offdiag))
        return fail(c, GBN_ERR_ARG, "the top layer's shift without rotate-first divides by the lattice mismatch");
    if (m->second_moire && !m->rotate_first &&
        ((m->twisted2 && m->moire_onsite && m->eps == 0.0) ||
         (m->moire_offdiag && (m->eps == 0.0 || m->eps_factor == 0.0))))
        return fail(c, GBN_ERR_ARG, "the second moire without SecondMoireRotateFirst divides by the lattice mismatch");
    cudaSetDevice(c->device);
    DevBuf ron, uni;
    const double* d_on = c->rat.as<double>();
    const double* d_hop = c->rat.as<double>();
    if (rat_on) {
        GBN_CK(c, ron.ensure(sizeof(double) * 3 * c->n));
        GBN_CK(c, cudaMemcpyAsync(ron.p, rat_on, sizeof(double) * 3 * c->n, cudaMemcpyHostToDevice, c->stream));
        d_on = ron.as<double>();
    }
    GBN_CK(c, c->rat_hop.ensure(sizeof(double) * 3 * c->n));
    if (rat_hop)
        GBN_CK(c, cudaMemcpyAsync(c->rat_hop.p, rat_hop, sizeof(double) * 3 * c->n, cudaMemcpyHostToDevice, c->stream));
    else
        GBN_CK(c, cudaMemcpyAsync(c->rat_hop.p, c->rat.p, sizeof(double) * 3 * c->n, cudaMemcpyDeviceToDevice, c->stream));
    d_hop = c->rat_hop.as<double>();
    const double* d_uni = nullptr;
    if (m->anderson) {
        GBN_CK(c, uni.ensure(sizeof(double) * c->n));
        GBN_CK(c, cudaMemcpyAsync(uni.p, uniform, sizeof(double) * c->n, cudaMemcpyHostToDevice, c->stream));
        d_uni = uni.as<double>();
    }
    const int rc = assemble(c, m, d_on, d_hop, d_uni);
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    return rc;
}

int gbn_peierls(gbn_ctx* c, double flux)
{
    if (!c) return GBN_ERR_ARG;
    if (!c->have_ham || !c->ncell.p || !c->rat_hop.p)
        return fail(c, GBN_ERR_STATE, "Peierls phases need an assembled Hamiltonian (gbn_assemble)");
    cudaSetDevice(c->device);
    return peierls(c, flux);
}

int gbn_get_hamiltonian(gbn_ctx* c, double* h0, double* hopp)
{
    if (!c) return GBN_ERR_ARG;
    if (!c->have_ham) return fail(c, GBN_ERR_STATE, "no Hamiltonian");
    cudaSetDevice(c->device);
    if (h0) GBN_CK(c, cudaMemcpyAsync(h0, c->h0.p, sizeof(double) * c->n, cudaMemcpyDeviceToHost, c->stream));
    if (hopp)
        GBN_CK(c, cudaMemcpyAsync(hopp, c->hopp.p, sizeof(double2) * (size_t)c->n * c->max_neigh, cudaMemcpyDeviceToHost,
                                  c->stream));
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    return GBN_OK;
}

int gbn_get_onsite_layers(gbn_ctx* c, double* bottom, double* top)
{
    if (!c) return GBN_ERR_ARG;
    if (!c->have_ham) return fail(c, GBN_ERR_STATE, "no Hamiltonian");
    cudaSetDevice(c->device);
    const size_t n = (size_t)c->n;
    if (bottom) {
        if (c->have_bottom)
            GBN_CK(c, cudaMemcpyAsync(bottom, c->h0_bottom.p, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
        else
            memset(bottom, 0, sizeof(double) * n);
    }
    if (top) {
        if (c->have_top) {
            std::vector<double> b(n);
            GBN_CK(c, cudaMemcpyAsync(top, c->h0.p, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
            GBN_CK(c, cudaMemcpyAsync(b.data(), c->h0_bottom.p, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
            GBN_CK(c, cudaStreamSynchronize(c->stream));
            for (size_t i = 0; i < n; ++i) top[i] = top[i] - b[i];   // H0Top = H0 - H0Bottom (ham.F90:3639)
        } else {
            memset(top, 0, sizeof(double) * n);
        }
    }
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    return GBN_OK;
}

int gbn_load_hamiltonian(gbn_ctx* c, int64_t n, int32_t max_neigh, const int32_t* nneigh, const int32_t* nlist,
                         const double* hopp, const double* h0)
{
    if (!c) return GBN_ERR_ARG;
    if (n < 1 || n >= (int64_t)1 << 31) return fail(c, GBN_ERR_ARG, "number of atoms must be in 1..2^31-1");
    if (max_neigh < 1) return fail(c, GBN_ERR_ARG, "max_neigh must be at least 1");
    if (!nneigh || !nlist || !hopp || !h0) return fail(c, GBN_ERR_ARG, "NULL Hamiltonian array");
    int64_t total = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (nneigh[i] < 0 || nneigh[i] > max_neigh) return fail(c, GBN_ERR_ARG, "Nneigh(i) outside 0..maxNeigh");
        total += nneigh[i];
        for (int32_t j = 0; j < nneigh[i]; ++j) {
            const int32_t m = nlist[i * max_neigh + j];
            if (m < 1 || m > n) return fail(c, GBN_ERR_ARG, "NList entry outside 1..N");
        }
    }
    bool cplx = false;
    const size_t e = (size_t)n * max_neigh;
    for (size_t k = 0; k < e && !cplx; ++k) cplx = hopp[2 * k + 1] != 0.0;
    cudaSetDevice(c->device);
    const bool same_atoms = c->have_geometry && c->n == n;
    GBN_CK(c, c->nneigh.ensure(sizeof(int32_t) * n));
    GBN_CK(c, c->nlist.ensure(sizeof(int32_t) * e));
    GBN_CK(c, c->hopp.ensure(sizeof(double2) * e));
    GBN_CK(c, c->h0.ensure(sizeof(double) * n));
    GBN_CK(c, cudaMemcpyAsync(c->nneigh.p, nneigh, sizeof(int32_t) * n, cudaMemcpyHostToDevice, c->stream));
    GBN_CK(c, cudaMemcpyAsync(c->nlist.p, nlist, sizeof(int32_t) * e, cudaMemcpyHostToDevice, c->stream));
    GBN_CK(c, cudaMemcpyAsync(c->hopp.p, hopp, sizeof(double2) * e, cudaMemcpyHostToDevice, c->stream));
    GBN_CK(c, cudaMemcpyAsync(c->h0.p, h0, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    if (!same_atoms) {
        c->have_geometry = false;
        c->n = n;
        const int rc = build_identity_perm(c);
        if (rc) return rc;
    }
    c->max_neigh = max_neigh;
    c->total = total;
    c->have_neigh = true;
    c->have_neighd = same_atoms && c->have_neighd;
    c->have_ham = true;
    c->have_bottom = c->have_top = false;
    c->ham_complex = cplx;
    c->ell.valid = false;
    return GBN_OK;
}

int gbn_check_hamiltonian(gbn_ctx* c, int64_t* counts, double* max_asym)
{
    if (!c || !counts || !max_asym) return GBN_ERR_ARG;
    cudaSetDevice(c->device);
    return check_hamiltonian(c, counts, max_asym);
}

int gbn_haldane(gbn_ctx* c, double aG, double t2, double phase, int32_t paper, uint32_t layer_mask)
{
    if (!c) return GBN_ERR_ARG;
    if (!(aG > 0.0)) return fail(c, GBN_ERR_ARG, "aG must be positive");
    cudaSetDevice(c->device);
    return haldane(c, aG, t2, phase, paper, layer_mask);
}

int gbn_set_images(gbn_ctx* c, const int32_t* ncell)
{
    if (!c || !ncell) return GBN_ERR_ARG;
    if (!c->have_neigh) return fail(c, GBN_ERR_STATE, "load the neighbour list first");
    if (!c->have_geometry) return fail(c, GBN_ERR_STATE, "the Peierls phases need the positions: gbn_set_geometry first");
    cudaSetDevice(c->device);
    const size_t e = (size_t)c->n * c->max_neigh;
    GBN_CK(c, c->ncell.ensure(sizeof(int32_t) * 3 * e));
    GBN_CK(c, cudaMemcpyAsync(c->ncell.p, ncell, sizeof(int32_t) * 3 * e, cudaMemcpyHostToDevice, c->stream));
    GBN_CK(c, c->rat_hop.ensure(sizeof(double) * 3 * (size_t)c->n));
    GBN_CK(c, cudaMemcpyAsync(c->rat_hop.p, c->rat.p, sizeof(double) * 3 * (size_t)c->n, cudaMemcpyDeviceToDevice,
                              c->stream));
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    return GBN_OK;
}

int gbn_set_neighd(gbn_ctx* c, const double* neighd)
{
    if (!c || !neighd) return GBN_ERR_ARG;
    if (!c->have_neigh) return fail(c, GBN_ERR_STATE, "load the neighbour list first");
    cudaSetDevice(c->device);
    const size_t e = (size_t)c->n * c->max_neigh;
    GBN_CK(c, c->neighd.ensure(sizeof(double) * 3 * e));
    GBN_CK(c, cudaMemcpyAsync(c->neighd.p, neighd, sizeof(double) * 3 * e, cudaMemcpyHostToDevice, c->stream));
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    c->have_neighd = true;
    return GBN_OK;
}

int gbn_lanczos(gbn_ctx* c, int32_t precision, int32_t nrhs, const double* psi0, const int32_t* nsteps, int32_t nmax,
                double* a, double* b)
{
    if (!c) return GBN_ERR_ARG;
    int rc = check_solver_args(c, precision, nrhs, psi0, nsteps, nmax, a, b);
    if (rc) return rc;
    cudaSetDevice(c->device);
    return run_tiled(c, precision, nrhs, psi0, false, nsteps, nmax, a, b);
}

int gbn_lanczos_phases(gbn_ctx* c, int32_t precision, int32_t nrhs, const double* u, const int32_t* nsteps,
                       int32_t nmax, double* a, double* b)
{
    if (!c) return GBN_ERR_ARG;
    int rc = check_solver_args(c, precision, nrhs, u, nsteps, nmax, a, b);
    if (rc) return rc;
    cudaSetDevice(c->device);
    return run_tiled(c, precision, nrhs, u, true, nsteps, nmax, a, b);
}

int gbn_lanczos_sites(gbn_ctx* c, int32_t precision, int32_t nsites, const int64_t* sites, const int32_t* nsteps,
                      int32_t nmax, double* a, double* b)
{
    if (!c) return GBN_ERR_ARG;
    int rc = check_solver_args(c, precision, nsites, sites, nsteps, nmax, a, b);
    if (rc) return rc;
    std::vector<int64_t> s0((size_t)nsites);
    for (int r = 0; r < nsites; ++r) {
        if (sites[r] < 1 || sites[r] > c->n) return fail(c, GBN_ERR_ARG, "site index out of 1..N");
        s0[(size_t)r] = sites[r] - 1;
    }
    cudaSetDevice(c->device);
    DevBuf d_site;
    GBN_CK(c, d_site.ensure(sizeof(int64_t) * (size_t)nsites));
    GBN_CK(c, cudaMemcpyAsync(d_site.p, s0.data(), sizeof(int64_t) * (size_t)nsites, cudaMemcpyHostToDevice,
                              c->stream));
    rc = run_tiles(
        c, precision, nsites,
        [&](int r0, int cnt) -> int { return lanczos_start_from_sites(c, d_site.as<int64_t>() + r0, cnt); }, nsteps,
        nmax, a, b);
    cudaStreamSynchronize(c->stream);
    return rc;
}

int gbn_lanczos_sets(gbn_ctx* c, int32_t precision, int32_t nsets, const int32_t* set_of_atom, const double* u,
                     const double* assumed, const int32_t* nsteps, int32_t nmax, double* a, double* b)
{
    if (!c) return GBN_ERR_ARG;
    int rc = check_solver_args(c, precision, nsets, set_of_atom, nsteps, nmax, a, b);
    if (rc) return rc;
    if (!u || !assumed) return fail(c, GBN_ERR_ARG, "NULL draws or assumed counts");
    const int64_t n = c->n;
    // draw of each atom: the k-th member of a set takes u[k] (each set reseeds the same stream)
    std::vector<int64_t> members((size_t)nsets, 0);
    std::vector<double> draw((size_t)n, 0.0);
    for (int64_t i = 0; i < n; ++i) {
        const int32_t s = set_of_atom[i];
        if (s < -1 || s >= nsets) return fail(c, GBN_ERR_ARG, "set_of_atom entries must be in -1..nsets-1");
        if (s >= 0) draw[(size_t)i] = u[members[(size_t)s]++];
    }
    for (int s = 0; s < nsets; ++s)
        if (!(assumed[s] > 0.0)) return fail(c, GBN_ERR_ARG, "assumed counts must be positive");
    // A set without atoms has a zero start vector and no DOS (the reference divides by its zero norm):
    // its a, b are NaN and the others run as a compact batch.
    std::vector<int32_t> slot((size_t)nsets, -1), owner;
    for (int s = 0; s < nsets; ++s)
        if (members[(size_t)s] > 0) {
            slot[(size_t)s] = (int32_t)owner.size();
            owner.push_back(s);
        }
    const int ne = (int)owner.size();
    for (int s = 0; s < nsets; ++s)
        if (slot[(size_t)s] < 0)
            for (int k = 0; k < nmax; ++k) a[(size_t)s * nmax + k] = b[(size_t)s * nmax + k] = NAN;
    if (ne == 0) return GBN_OK;
    std::vector<int32_t> so((size_t)n), ns;
    for (int64_t i = 0; i < n; ++i) so[(size_t)i] = set_of_atom[i] >= 0 ? slot[(size_t)set_of_atom[i]] : -1;
    // psi = e^(i th)/sqrt(M); the reference normalises when |<psi|psi> - 1| > 1e-6, <psi|psi> = count/M
    std::vector<double> den((size_t)2 * ne);
    for (int e = 0; e < ne; ++e) {
        const int s = owner[(size_t)e];
        const double nrm = (double)members[(size_t)s] / assumed[s];
        den[(size_t)2 * e] = sqrt(assumed[s]);
        den[(size_t)2 * e + 1] = fabs(nrm - 1.0) > 1.0e-6 ? sqrt(nrm) : 1.0;
        if (nsteps) ns.push_back(nsteps[s]);
    }
    cudaSetDevice(c->device);
    DevBuf d_set, d_draw, d_den;
    GBN_CK(c, d_set.ensure(sizeof(int32_t) * (size_t)n));
    GBN_CK(c, d_draw.ensure(sizeof(double) * (size_t)n));
    GBN_CK(c, d_den.ensure(sizeof(double) * den.size()));
    GBN_CK(c, cudaMemcpyAsync(d_set.p, so.data(), sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, c->stream));
    GBN_CK(c, cudaMemcpyAsync(d_draw.p, draw.data(), sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, c->stream));
    GBN_CK(c, cudaMemcpyAsync(d_den.p, den.data(), sizeof(double) * den.size(), cudaMemcpyHostToDevice, c->stream));
    std::vector<double> ae((size_t)ne * nmax), be((size_t)ne * nmax);
    rc = run_tiles(
        c, precision, ne,
        [&](int r0, int cnt) -> int {
            return lanczos_start_from_sets(c, d_set.as<int32_t>(), d_draw.as<double>(), d_den.as<double>(), r0, cnt);
        },
        nsteps ? ns.data() : nullptr, nmax, ae.data(), be.data());
    cudaStreamSynchronize(c->stream);   // the host vectors above must outlive the copies
    if (rc) return rc;
    for (int e = 0; e < ne; ++e) {
        memcpy(a + (size_t)owner[(size_t)e] * nmax, ae.data() + (size_t)e * nmax, sizeof(double) * nmax);
        memcpy(b + (size_t)owner[(size_t)e] * nmax, be.data() + (size_t)e * nmax, sizeof(double) * nmax);
    }
    return GBN_OK;
}

int gbn_lanczos_fields(gbn_ctx* c, int32_t precision, int32_t nfields, const int32_t* m, int32_t nvec, const double* u,
                       const int32_t* nsteps, int32_t nmax, double* a, double* b)
{
    if (!c) return GBN_ERR_ARG;
    if (nfields < 1 || nvec < 1 || !m) return fail(c, GBN_ERR_ARG, "nfields and nvec must be positive, m not NULL");
    const int64_t nr64 = (int64_t)nfields * nvec;
    if (nr64 > (int64_t)1 << 30) return fail(c, GBN_ERR_ARG, "too many right-hand sides");
    const int nrhs = (int)nr64;
    int rc = check_solver_args(c, precision, nrhs, u, nsteps, nmax, a, b);
    if (rc) return rc;
    if (c->has_field)
        return fail(c, GBN_ERR_STATE, "the hoppings already carry a field: assemble again without gbn_peierls");
    if (c->ham_complex)
        return fail(c, GBN_ERR_STATE, "batched fields need a Hamiltonian assembled on the device (gbn_assemble)");
    cudaSetDevice(c->device);
    rc = peierls_turns(c);
    if (rc) return rc;
    // the RPT right-hand sides of a thread share one field: RPT divides the vectors per field
    const int T = tile_width(nrhs);
    const int saved_rpt = c->tune_rpt;
    int rpt, tpr;
    split_rhs(precision, T, saved_rpt, &rpt, &tpr);
    while (nvec % rpt) rpt >>= 1;
    // run order: within a field its vectors by decreasing length, in chunks of RPT; chunks by decreasing
    // length, so that a tile's vectors end close together (a tile runs to its longest vector)
    auto len = [&](int r) { return nsteps ? nsteps[r] : nmax; };
    std::vector<std::pair<int32_t, int32_t>> chunks;   // (length of the chunk's first vector, first slot)
    std::vector<int32_t> sorted((size_t)nrhs);
    for (int f = 0; f < nfields; ++f) {
        int32_t* v = sorted.data() + (size_t)f * nvec;
        for (int k = 0; k < nvec; ++k) v[k] = f * nvec + k;
        std::stable_sort(v, v + nvec, [&](int32_t x, int32_t y) { return len(x) > len(y); });
        for (int k = 0; k < nvec; k += rpt) chunks.push_back({len(v[k]), f * nvec + k});
    }
    std::stable_sort(chunks.begin(), chunks.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
    std::vector<int32_t> order, ns_run, fm_run;
    for (const auto& ch : chunks)
        for (int k = 0; k < rpt; ++k) {
            const int32_t r = sorted[(size_t)ch.second + k];
            order.push_back(r);
            ns_run.push_back(len(r));
            fm_run.push_back(m[r / nvec]);
        }
    const int64_t n = c->n;
    GBN_CK(c, c->upload.ensure(sizeof(double) * (size_t)n * T));
    std::vector<double> ar((size_t)nrhs * nmax), br((size_t)nrhs * nmax);
    c->tune_rpt = rpt;
    split_rhs(precision, T, rpt, &rpt, &tpr);   // the split the tile's kernel uses
    GBN_CK(c, c->field_m.ensure(sizeof(int32_t) * (size_t)(T + tpr)));
    std::vector<int32_t> fm((size_t)(T + tpr));
    rc = run_tiles(
        c, precision, nrhs,
        [&](int r0, int cnt) -> int {
            for (int r = 0; r < cnt; ++r)
                GBN_CK(c, cudaMemcpyAsync(c->upload.as<double>() + (size_t)r * n, u + (size_t)order[(size_t)(r0 + r)] * n,
                                          sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, c->stream));
            for (int r = 0; r < T; ++r) fm[(size_t)r] = fm_run[(size_t)(r0 + (r < cnt ? r : 0))];
            // the flux quanta of each thread slot of a row group (the slot's RPT right-hand sides share one
            // field) follow those of the right-hand sides: fm[T + q] = fm[q RPT]
            for (int q = 0; q < tpr; ++q) fm[(size_t)T + q] = fm[(size_t)q * rpt];
            GBN_CK(c, cudaMemcpyAsync(c->field_m.p, fm.data(), sizeof(int32_t) * fm.size(), cudaMemcpyHostToDevice,
                                      c->stream));
            if (c->tune_field_table == 1) {   // the tile's rotations, once for all its steps
                const int rc2 = build_field_table(c, tpr, c->field_m.as<int32_t>() + T);
                if (rc2) return rc2;
            }
            return lanczos_start_from_phases(c, c->upload.as<double>(), cnt);
        },
        ns_run.data(), nmax, ar.data(), br.data(), true);
    c->tune_rpt = saved_rpt;
    c->staged = false;
    if (rc) return rc;
    for (int r = 0; r < nrhs; ++r) {
        memcpy(a + (size_t)order[(size_t)r] * nmax, ar.data() + (size_t)r * nmax, sizeof(double) * nmax);
        memcpy(b + (size_t)order[(size_t)r] * nmax, br.data() + (size_t)r * nmax, sizeof(double) * nmax);
    }
    return GBN_OK;
}

int gbn_stage_phases(gbn_ctx* c, int32_t precision, int32_t nrhs, const double* u)
{
    if (!c) return GBN_ERR_ARG;
    if (!c->have_ham) return fail(c, GBN_ERR_STATE, "no Hamiltonian");
    if (!u) return fail(c, GBN_ERR_ARG, "NULL draws");
    if (precision != GBN_FP64 && precision != GBN_MIXED) return fail(c, GBN_ERR_ARG, "bad precision");
    if (nrhs != 1 && nrhs != 2 && nrhs != 4 && nrhs != 8 && nrhs != 16 && nrhs != 32)
        return fail(c, GBN_ERR_ARG, "staged runs take 1, 2, 4, 8, 16 or 32 vectors");
    cudaSetDevice(c->device);
    int rc = lanczos_prepare(c, precision, nrhs);
    if (rc) return rc;
    GBN_CK(c, c->upload.ensure(sizeof(double) * (size_t)c->n * nrhs));
    GBN_CK(c, cudaMemcpyAsync(c->upload.p, u, sizeof(double) * (size_t)c->n * nrhs, cudaMemcpyHostToDevice, c->stream));
    rc = lanczos_start_from_phases(c, c->upload.as<double>(), nrhs);
    if (rc) return rc;
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    c->staged = true;
    return GBN_OK;
}

int gbn_run_staged(gbn_ctx* c, int32_t nmax, double* a, double* b)
{
    if (!c) return GBN_ERR_ARG;
    if (!c->staged) return fail(c, GBN_ERR_STATE, "nothing staged: call gbn_stage_phases first");
    if (nmax < 1) return fail(c, GBN_ERR_ARG, "nmax must be at least 1");
    cudaSetDevice(c->device);
    int rc = GBN_OK;
    // the layout matches the current Hamiltonian and tuning (rebuilt only when either changed since staging)
    rc = lanczos_prepare(c, c->prec, c->nrhs);
    if (rc) return rc;
    // the start vectors are rebuilt from the staged draws so that every run starts from them
    rc = lanczos_start_from_phases(c, c->upload.as<double>(), c->nrhs);
    if (rc) return rc;
    rc = lanczos_run(c, nmax);
    if (rc) return rc;
    if (a && b) {
        GBN_CK(c, cudaMemcpyAsync(a, c->ab.p, sizeof(double) * (size_t)c->nrhs * nmax, cudaMemcpyDeviceToHost, c->stream));
        GBN_CK(c, cudaMemcpyAsync(b, c->ab.as<double>() + (size_t)c->nrhs * nmax, sizeof(double) * (size_t)c->nrhs * nmax,
                                  cudaMemcpyDeviceToHost, c->stream));
        GBN_CK(c, cudaStreamSynchronize(c->stream));
    }
    return GBN_OK;
}

int gbn_cf_dos(gbn_ctx* c, int32_t nrhs, const double* a, const double* b, const int32_t* nsteps, int32_t nmax,
               double eta, int32_t n_en, double emin, double emax, const double* norm, double* energy, double* dos)
{
    if (!c) return GBN_ERR_ARG;
    if (nrhs < 1 || nmax < 1 || n_en < 1 || !a || !b || !dos) return fail(c, GBN_ERR_ARG, "bad continued-fraction arguments");
    if (!(eta > 0.0)) return fail(c, GBN_ERR_ARG, "eta must be positive");
    if (nsteps)
        for (int r = 0; r < nrhs; ++r)
            if (nsteps[r] < 1 || nsteps[r] > nmax) return fail(c, GBN_ERR_ARG, "nsteps[r] must be in 1..nmax");
    cudaSetDevice(c->device);
    const size_t nab = (size_t)nrhs * nmax, nd = (size_t)nrhs * (n_en + 1);
    DevBuf da, db, dn, dno, dd;
    GBN_CK(c, da.ensure(sizeof(double) * nab));
    GBN_CK(c, db.ensure(sizeof(double) * nab));
    GBN_CK(c, dd.ensure(sizeof(double) * nd));
    GBN_CK(c, cudaMemcpyAsync(da.p, a, sizeof(double) * nab, cudaMemcpyHostToDevice, c->stream));
    GBN_CK(c, cudaMemcpyAsync(db.p, b, sizeof(double) * nab, cudaMemcpyHostToDevice, c->stream));
    if (nsteps) {
        GBN_CK(c, dn.ensure(sizeof(int32_t) * nrhs));
        GBN_CK(c, cudaMemcpyAsync(dn.p, nsteps, sizeof(int32_t) * nrhs, cudaMemcpyHostToDevice, c->stream));
    }
    if (norm) {
        GBN_CK(c, dno.ensure(sizeof(double) * nrhs));
        GBN_CK(c, cudaMemcpyAsync(dno.p, norm, sizeof(double) * nrhs, cudaMemcpyHostToDevice, c->stream));
    }
    int rc = cf_dos(c, nrhs, da.as<double>(), db.as<double>(), nsteps ? dn.as<int32_t>() : nullptr, nmax, eta, n_en, emin,
                    emax, norm ? dno.as<double>() : nullptr, dd.as<double>());
    if (rc) return rc;
    GBN_CK(c, cudaMemcpyAsync(dos, dd.p, sizeof(double) * nd, cudaMemcpyDeviceToHost, c->stream));
    GBN_CK(c, cudaStreamSynchronize(c->stream));
    if (energy) {
        const double de = (emax - emin) / n_en;
        for (int k = 0; k <= n_en; ++k) energy[k] = emin + (double)k * de;
    }
    return GBN_OK;
}

int gbn_cheb_evolve(gbn_ctx* c, int32_t precision, int32_t nrhs, const double* coef, int32_t npol, double ac, double bc,
                    double* z)
{
    if (!c) return GBN_ERR_ARG;
    cudaSetDevice(c->device);
    return cheb_evolve(c, precision, nrhs, coef, npol, ac, bc, z);
}

int gbn_kubo_evol(gbn_ctx* c, int32_t precision, int32_t nrhs, const double* coef, int32_t npol, double ac, double bc,
                  int32_t dir, double* psi, double* zupsi)
{
    if (!c) return GBN_ERR_ARG;
    if (!c->have_ham) return fail(c, GBN_ERR_STATE, "no Hamiltonian");
    if (!c->have_neighd) return fail(c, GBN_ERR_STATE, "KuboEvol needs NeighD (gbn_neighbours or gbn_set_neighd)");
    if (dir != 1 && dir != 2) return fail(c, GBN_ERR_ARG, "dir must be 1 (x) or 2 (y)");
    if (nrhs < 1 || npol < 1 || !coef || !psi || !zupsi || !(bc > 0.0)) return fail(c, GBN_ERR_ARG, "bad KuboEvol arguments");
    cudaSetDevice(c->device);
    return kubo_evol(c, precision, nrhs, coef, npol, ac, bc, dir, psi, zupsi);
}

int gbn_kubo_tevol(gbn_ctx* c, int32_t precision, int32_t nrhs, const double* coef, int32_t npol, double ac, double bc,
                   int32_t dir, int32_t nt, int32_t nwr, int32_t nrecurs, double* psi, double* zupsi, double* norms,
                   double* a, double* b)
{
    if (!c) return GBN_ERR_ARG;
    if (!c->have_ham) return fail(c, GBN_ERR_STATE, "no Hamiltonian");
    if (precision != GBN_FP64 && precision != GBN_MIXED) return fail(c, GBN_ERR_ARG, "bad precision");
    if (nrhs < 1 || npol < 1 || !coef || !psi || !zupsi || !(bc > 0.0) || !isfinite(ac) || nt < 0 || nwr < 1 ||
        nrecurs < 1)
        return fail(c, GBN_ERR_ARG, "bad KuboTEvol arguments");
    if (nt / nwr > 0 && (!norms || !a || !b)) return fail(c, GBN_ERR_ARG, "NULL output arrays");
    cudaSetDevice(c->device);
    return kubo_tevol(c, precision, nrhs, coef, npol, ac, bc, dir, nt, nwr, nrecurs, psi, zupsi, norms, a, b);
}

int gbn_dos_gradient(gbn_ctx* c, const gbn_model* model, double g0, const double* u, int32_t nrecurs, int32_t checkpoint,
                     double eta, int32_t n_en, double emin, double emax, const double* target, double* loss, double* grad,
                     double* dos, double* a, double* b)
{
    if (!c) return GBN_ERR_ARG;
    cudaSetDevice(c->device);
    return dos_gradient(c, GBN_FP64, model, g0, u, nrecurs, checkpoint, eta, n_en, emin, emax, target, loss, grad,
                        dos, a, b);
}

int gbn_dos_gradient_prec(gbn_ctx* c, int32_t precision, const gbn_model* model, double g0, const double* u,
                          int32_t nrecurs, int32_t checkpoint, double eta, int32_t n_en, double emin, double emax,
                          const double* target, double* loss, double* grad, double* dos, double* a, double* b)
{
    if (!c) return GBN_ERR_ARG;
    cudaSetDevice(c->device);
    return dos_gradient(c, precision, model, g0, u, nrecurs, checkpoint, eta, n_en, emin, emax, target, loss, grad,
                        dos, a, b);
}

}  // extern "C"
