// Internal declarations of libgrabnes_gpu: context, device buffers, error plumbing.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/grabnes_gpu.h"

namespace gbn {

// Device allocation that grows on demand; freed by release() or when it goes out of scope.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    cudaError_t ensure(size_t need) {
        if (need <= bytes && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, need ? need : 16);
        if (e == cudaSuccess) bytes = need ? need : 16;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

// Grouped sliced ELL of the permuted Hamiltonian.  Rows are taken in groups of G consecutive rows
// (neighbouring atoms in the solver's row order); a group stores the union of its rows' neighbour
// columns once, with G values per union column (zero where a row has no such neighbour), so a
// gathered vector row serves all G rows.  gpw groups form a slice (the groups one warp processes
// together).  A slice is one contiguous record in `mat`, starting at byte slice_ptr[s] * entry_bytes
// (entry_bytes = 4 + G * val_size; slice_ptr counts union entries, w * gpw per slice):
//     int32 col[w/4][gpw][4]   then   value val[w/4][gpw][4] (one FP32 value per column) or val[w][gpw][G]
// (blocks of four union columns; in a block each group's four columns are contiguous: rec_slot, val_slot).
// Slice widths w are multiples of 4 (records are multiples of 16 bytes and start on 16-byte
// boundaries); padding columns point at the group's first row with zero values.  Values are stored
// NEGATED (-hopp = +t/g0), so that (H x)_i = h0_i x_i + sum val * x.  G = 1 is the plain sliced ELL.
struct Ell {
    int G = 0;               // rows per group
    int gpw = 0;             // groups per slice
    int prec = -1;           // GBN_FP64 / GBN_MIXED
    bool cplx = false;       // complex values stored
    int64_t ngroups = 0;
    int64_t nslices = 0;
    int64_t npad = 0;        // nslices * gpw * G rows (vectors are allocated for npad rows)
    int64_t nnz_stored = 0;  // union entries including padding
    DevBuf slice_ptr;        // int64 [nslices + 1]
    DevBuf mat;              // slice records
    DevBuf h0;               // float | double [npad]
    DevBuf rperm, riperm;    // solver row order: rperm[row] = reference atom (row < n), riperm inverse
    int val_size = 0;        // bytes per stored value
    int entry_bytes = 0;     // 4 + G * val_size
    DevBuf dval;             // d * val per stored value (KuboEvol's commutator), same indexing as the values
    int dval_dir = 0;        // NeighD component of dval (1 = x, 2 = y; 0 = not built)
    int64_t max_record = 0;  // bytes of the largest slice record
    int64_t cap_record = 0;  // staging buffer size: 99.5 % of the records fit (larger ones are read in place)
    int64_t cap_pct[4] = {0, 0, 0, 0};   // record sizes at the 99.5th, 99th, 95th and 90th percentiles
    bool field = false;      // field-batched values: field-free hopping and Peierls phase per flux quantum
    // Field-batched tile table: the records with each value rotated for the fields of the tile's thread
    // slots (slot q of a row group = its q-th thread's right-hand sides): the record's int32 columns, then
    // complex val[w][gpw][slots][G] in the order of the record's values (val_slot: field values are
    // column-major; slot q rotated by the field of slot q).  Rebuilt for every tile.
    DevBuf ftab;
    int ftab_slots = 0;
    int ftab_entry_bytes = 0;   // 4 + slots * G * complex bytes
    bool ftab_valid = false;
    // Tiles of consecutive slices for the tile-local product: tile t holds slices
    // [tile_slice[t], tile_slice[t+1]) and gathers only the rows halo[halo_ptr[t] .. halo_ptr[t+1]) (at most
    // tile_hmax, in order of first use); tmat is mat with every column index replaced by its position in
    // the tile's halo list, so that a tile's gathers read a copy of those rows in shared memory.
    DevBuf tile_slice, halo_ptr, halo, tmat;
    int64_t ntiles = 0;
    int tile_hmax = 0;
    bool tiles_valid = false;
    bool valid = false;
};

// unroll of the union-column loop (slice widths are multiples of it)
constexpr int kColUnroll = 4;

// Entry position of union column k of group j in a slice record of gpw groups.  The record holds its
// columns in blocks of kColUnroll; inside a block each group's kColUnroll indices are contiguous (16
// bytes), so a thread reads a block's indices with one 16-byte load and a warp's groups read one block
// from consecutive 16-byte pieces.
__host__ __device__ __forceinline__ int64_t rec_slot(int k, int j, int gpw)
{
    return (int64_t)(k / kColUnroll) * kColUnroll * gpw + (int64_t)j * kColUnroll + k % kColUnroll;
}

// The values follow rec_slot's order only where a group's values of one column take 4 bytes (one FP32
// value, G = 1: a block's four are one 16-byte load).  Wider values stay column-major, val[w][gpw][G]:
// read one column at a time, the groups of a warp then touch consecutive bytes and distinct banks,
// where rec_slot's order would put them 4 columns apart (2- to 8-way bank conflicts).
__host__ __device__ __forceinline__ constexpr bool block_vals(int G, int val_bytes) { return G * val_bytes == 4; }
// Position (in values) of the first of the G values of union column k of group j.
__host__ __device__ __forceinline__ int64_t val_slot(int k, int j, int gpw, int G, int val_bytes)
{
    return block_vals(G, val_bytes) ? rec_slot(k, j, gpw) : ((int64_t)k * gpw + j) * G;
}

struct Timing {
    double step_ms = 0.0;        // whole recursion loop of the last call
    int64_t step_launches = 0;   // recursion steps of the last call
    double update_ms_avg = 0.0;  // per-launch duration of the update kernel (first steps)
    double spmm_ms_avg = 0.0;    // per-launch duration of the sparse-product kernel (first steps)
};

constexpr int kTimedSteps = 64;
// steps per CUDA-graph replay of the recursion loop (even: the two x buffers alternate with the step)
constexpr int kGraphSteps = 32;

}  // namespace gbn

struct gbn_ctx {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;
    int64_t launches = 0;

    // geometry (reference order)
    int64_t n = 0;
    double ucell[9] = {0};
    gbn::DevBuf rat, species, layer;  // double[3n], int32[n], int32[n]
    bool have_geometry = false;

    // neighbour tables (reference layout)
    int32_t max_neigh = 0;
    int64_t total = 0;
    gbn::DevBuf nneigh, nlist, neighd, ncell;
    bool have_neigh = false;
    bool have_neighd = false;

    // Hamiltonian (reference layout, FP64)
    gbn::DevBuf h0, hopp;  // double[n], double2[n*max_neigh]
    gbn::DevBuf rat_hop;   // positions used for the Peierls phases
    gbn::DevBuf h0_bottom; // double[n]: H0 after the first moire's terms (moire branch only)
    bool have_bottom = false;   // the assembled model ran the moire branch (h0_bottom is set)
    bool have_top = false;      // ... and the second moire (H0Top = H0 - H0Bottom)
    gbn::DevBuf dimer;          // int8 [n] dimer sites of the Bernal interlayer branch, then a 64-bit count
    int bernal_used = 0;        // the encapsulated bilayer's interlayer branch of the last assembly (0: none)
    bool have_ham = false;
    bool ham_complex = false;
    bool has_field = false;   // gbn_peierls has been applied to the assembled hoppings
    gbn::DevBuf ptau;         // uint64 [n*max_neigh]: Peierls phase per flux quantum, fraction of a turn * 2^64
    gbn::DevBuf field_m;      // int32 [R]: flux quanta of each right-hand side of a field-batched tile

    // row permutation used by the solver: perm[new] = reference index, iperm[reference] = new
    gbn::DevBuf perm, iperm;
    bool perm_spatial = false;

    gbn::Ell ell;

    // recursion state
    int prec = -1;
    int nrhs = 0;
    gbn::DevBuf vec[4];      // v, x_prev, x_cur (ping-pong of the x pair)
    gbn::DevBuf partials;    // double [blocks][R]
    gbn::DevBuf scal;        // double [R][4]: a, norms of the current and the previous carried vector
    gbn::DevBuf counter;     // uint32 block counter + int32 step index + int32 flag
    gbn::DevBuf ab;          // double [2][R][nmax]
    gbn::DevBuf upload;      // staging of host inputs
    int32_t staged_nmax = 0;
    bool staged = false;
    gbn::Timing timing;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t kev[3 * gbn::kTimedSteps] = {};

    // tuning of the recursion kernels (0 = automatic)
    int tune_rpt = 0;            // right-hand sides per thread
    int tune_blocks_per_sm = 0;  // cap on resident blocks per SM
    int tune_group = 0;          // rows per group of the matrix layout (1, 2, 4)
    int tune_staged = -1;        // matrix records staged in shared memory by bulk copies (-1 auto, 0 no, 1 yes)
    int tune_prefetch = -1;      // staged kernel: prefetch the gather rows of a slice (0 no, 1 to L2, 2 to L1)
                                 // or the rows of its epilogue (3 to L1, 4 to L2; -1 = 4)
    int tune_unroll = 0;         // union columns in flight per batch of the product (4, 8; 0 = automatic)
    int tune_stage_values = -1;  // staged records carry the values (1) or only the column indices (0); -1 auto
    int tune_min_blocks = 0;     // product kernel compiled for 1 or 3 resident blocks per SM (0 = 1)
    int tune_tiled = -1;         // tile-local product (halo rows in shared memory): 1 yes, 0 no, -1 default (no)
    int tune_fused = -1;         // the update folded into the product: 1 yes, 0 no, -1 default (no)
    int tune_field_table = -1;   // batched fields: rotations tabulated per tile (1) or on the fly (0, -1 default)
    bool last_staged = false;    // the last recursion used the staged kernel

    // Chebyshev work vectors
    gbn::DevBuf cheb[8];

    // the recursion loop's CUDA graph (kGraphSteps steps) and the launch configuration it was captured with
    cudaGraphExec_t step_graph = nullptr;
    std::vector<unsigned char> step_graph_key;
    int64_t graph_replays = 0;   // graph launches of the last recursion
};

namespace gbn {

int fail(gbn_ctx* c, int code, const std::string& msg);
int cuda_fail(gbn_ctx* c, cudaError_t e, const char* what);

#define GBN_CK(ctx, call)                                                   \
    do {                                                                    \
        cudaError_t e__ = (call);                                           \
        if (e__ != cudaSuccess) return gbn::cuda_fail((ctx), e__, #call);  \
    } while (0)

#define GBN_CK_LAUNCH(ctx)                                                          \
    do {                                                                            \
        (ctx)->launches++;                                                          \
        cudaError_t e__ = cudaGetLastError();                                       \
        if (e__ != cudaSuccess) return gbn::cuda_fail((ctx), e__, "kernel launch"); \
    } while (0)

// layout / permutation (gbn_layout.cu)
int build_identity_perm(gbn_ctx* c);
int build_spatial_perm(gbn_ctx* c);
// field: the field-batched values (FieldVal: field-free hopping and c->ptau), for gbn_lanczos_fields
int build_ell(gbn_ctx* c, int prec, int G, int gpw, bool field = false);
int auto_group(const gbn_ctx* c, int R, int prec);   // default rows per group for a tile of R vectors
// the tile table of the field-batched layout for the flux quanta of each thread slot (d_slot_m [slots])
int build_field_table(gbn_ctx* c, int slots, const int32_t* d_slot_m);
// tiles of the layout whose halos have at most hmax rows (host pass over the records)
int build_tiles(gbn_ctx* c, int hmax);

// recursion (gbn_lanczos.cu)
int lanczos_prepare(gbn_ctx* c, int prec, int nrhs, bool field = false);
int lanczos_start_from_phases(gbn_ctx* c, const double* d_u, int nrhs_real);
int lanczos_start_from_psi(gbn_ctx* c, const double* d_psi, int nrhs_real);
int lanczos_start_from_sites(gbn_ctx* c, const int64_t* d_site, int nrhs_real);
int lanczos_start_from_sets(gbn_ctx* c, const int32_t* d_set, const double* d_draw, const double* d_den, int set0,
                            int nrhs_real);
int lanczos_run(gbn_ctx* c, int32_t nmax);
// right-hand sides per thread and threads per row group for a tile of R vectors
void split_rhs(int prec, int R, int want, int* rpt, int* tpr);

// continued fraction (gbn_cf.cu)
int cf_dos(gbn_ctx* c, int32_t nrhs, const double* d_a, const double* d_b, const int32_t* d_nsteps, int32_t nmax,
           double eta, int32_t n_en, double emin, double emax, const double* d_norm, double* d_dos);

// neighbour search and assembly (gbn_neigh.cu, gbn_model.cu)
int neigh_search(gbn_ctx* c, double cut2intra, double cut2inter, int32_t second_layer);
int assemble(gbn_ctx* c, const gbn_model* m, const double* d_rat_on, const double* d_rat_hop, const double* d_uniform);
int peierls(gbn_ctx* c, double flux);
int peierls_turns(gbn_ctx* c);
int haldane(gbn_ctx* c, double aG, double t2, double phase, int32_t paper, uint32_t layer_mask);
int check_hamiltonian(gbn_ctx* c, int64_t* out, double* max_asym);   // c->ptau from the positions, images and cell of the assembled model

// gradient of a DOS loss (gbn_adjoint.cu)
int dos_gradient(gbn_ctx* c, int32_t prec, const gbn_model* m, double g0, const double* u_host, int32_t K, int32_t C,
                 double eta, int32_t n_en, double emin, double emax, const double* target, double* loss_out,
                 double* grad, double* dos, double* a_out, double* b_out);

// Chebyshev (gbn_cheb.cu)
int cheb_evolve(gbn_ctx* c, int32_t prec, int32_t nrhs, const double* c_host, int32_t npol, double ac, double bc,
                double* z_host);
int kubo_evol(gbn_ctx* c, int32_t prec, int32_t nrhs, const double* c_host, int32_t npol, double ac, double bc,
              int32_t dir, double* psi_host, double* zupsi_host);
int kubo_tevol(gbn_ctx* c, int32_t prec, int32_t nrhs, const double* c_host, int32_t npol, double ac, double bc,
               int32_t dir, int32_t nt, int32_t nwr, int32_t nrecurs, double* psi_host, double* zupsi_host,
               double* norms, double* a_out, double* b_out);

inline int grid_for(gbn_ctx* c, int blocks_per_sm) { return c->num_sms * blocks_per_sm; }

}  // namespace gbn
