// gbn_lanczos_noalloc: the recursion of KuboRecursion for one start vector, for callers that cannot
// allocate device memory.
//
// Who needs it: a host program that hands all of a GPU's memory to its own pool allocator (a Fortran
// or C++ code that reserves the device up front, a framework whose caching allocator owns the card)
// leaves nothing for cudaMalloc, and cudaMalloc/cudaFree also synchronise the whole device, which a
// host that keeps other work in flight on that GPU may forbid.  Such a caller owns the Hamiltonian,
// the start vector and the coefficient arrays in device memory and passes them in; the three
// recursion vectors, the reduction partials and the block counter live in the file-scope array
// below instead of in memory this library would otherwise allocate per context.
//
// The array is a static __device__ object: every GPU that loads this library holds its
// kNaScratchBytes (about 48 MiB) until the process exits.  In host code its name is only a host-side
// stand-in, so the host asks the runtime for its device address once per device and context
// (cudaGetSymbolAddress, in na_scratch_on_current_device) and passes that address to the kernels.
//
// The recursion is the same three passes per step as the reference's KuboRecursion
// (lanczosKuboCode/Src/kubosubs.F90:26-138) on the reference's own neighbour-list layout:
//   a_n = Re <psi_n|H|psi_n>,  r = H psi_n - a_n psi_n - b_{n-1} psi_{n-1},  b_n = |r|,  psi_{n+1} = r / b_n
// with H psi = H0 psi - sum_j hopp(j) psi(NList(j)).  Sums are reduced in a fixed order (per-block
// partials, the last block adds them), so two calls on the same inputs give the same bits.
#include <cuda.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <mutex>

#include "../../include/grabnes_gpu.h"

namespace {

constexpr int kNaThreads = 256;
constexpr int kNaMaxBlocks = 148 * 8;
constexpr size_t kNaVecBytes = sizeof(double2) * (size_t)GBN_NOALLOC_MAX_ATOMS;
// psi_n, psi_{n-1}, H psi_n | partial sums | counter and error flags
constexpr size_t kNaScratchBytes = 3 * kNaVecBytes + sizeof(double) * kNaMaxBlocks + 256;

static __device__ __align__(256) unsigned char g_na_scratch[kNaScratchBytes];

struct NaScratch {
    double2* psin;
    double2* psinm1;
    double2* hv;
    double* partial;
    unsigned int* counter;  // counter[0]: blocks done with the current sum; counter[1]: error flags
};

NaScratch na_layout(unsigned char* base)
{
    NaScratch s;
    s.psin = reinterpret_cast<double2*>(base);
    s.psinm1 = reinterpret_cast<double2*>(base + kNaVecBytes);
    s.hv = reinterpret_cast<double2*>(base + 2 * kNaVecBytes);
    s.partial = reinterpret_cast<double*>(base + 3 * kNaVecBytes);
    s.counter = reinterpret_cast<unsigned int*>(base + 3 * kNaVecBytes + sizeof(double) * kNaMaxBlocks);
    return s;
}

constexpr unsigned kNaBadIndex = 1u;    // Nneigh or NList entry out of range (the access was skipped)
constexpr unsigned kNaBadNorm = 2u;     // b_n not finite or not positive

// Block sum in a fixed order; the last block to finish adds the block partials in index order and
// returns true in every thread of that block, with the total in *total.
__device__ bool na_grid_sum(double v, NaScratch s, double* total)
{
    __shared__ double warp_sums[kNaThreads / 32];
    __shared__ bool last;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kNaThreads / 32; ++w) t += warp_sums[w];
        s.partial[blockIdx.x] = t;
        __threadfence();
        last = atomicAdd(s.counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (unsigned blk = 0; blk < gridDim.x; ++blk) t += ((volatile double*)s.partial)[blk];
        *total = t;
        s.counter[0] = 0;  // ready for the next sum
    }
    return true;
}

__global__ void k_na_start(const double2* __restrict__ psi, int64_t n, NaScratch s)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        s.psin[i] = psi[i];
        s.psinm1[i] = make_double2(0.0, 0.0);
    }
}

// hv = H psi_n and a_n = Re <psi_n|hv>.
__global__ void __launch_bounds__(kNaThreads) k_na_apply(int64_t n, int32_t max_neigh, const int32_t* __restrict__ nneigh,
                                                        const int32_t* __restrict__ nlist, const double2* __restrict__ hopp,
                                                        const double* __restrict__ h0, NaScratch s, double* a, int it)
{
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 p = s.psin[i];
        double cr = h0[i] * p.x, ci = h0[i] * p.y;
        int32_t cnt = nneigh[i];
        if (cnt < 0 || cnt > max_neigh) {
            atomicOr(s.counter + 1, kNaBadIndex);
            cnt = 0;
        }
        const int64_t base = i * max_neigh;
        for (int32_t j = 0; j < cnt; ++j) {
            const int32_t m = nlist[base + j];
            if (m < 1 || m > n) {
                atomicOr(s.counter + 1, kNaBadIndex);
                continue;
            }
            const double2 t = hopp[base + j];
            const double2 x = s.psin[m - 1];
            cr -= t.x * x.x - t.y * x.y;
            ci -= t.x * x.y + t.y * x.x;
        }
        s.hv[i] = make_double2(cr, ci);
        acc += cr * p.x + ci * p.y;
    }
    double total;
    if (na_grid_sum(acc, s, &total) && threadIdx.x == 0) a[it] = total;
}

// r = hv - a_n psi_n - b_{n-1} psi_{n-1} (kept in hv) and b_n = |r|.
__global__ void __launch_bounds__(kNaThreads) k_na_residual(int64_t n, NaScratch s, const double* a, double* b, int it)
{
    const double an = a[it];
    const double bp = it > 0 ? b[it - 1] : 0.0;
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 h = s.hv[i], p = s.psin[i], q = s.psinm1[i];
        const double cr = (h.x - an * p.x) - bp * q.x;
        const double ci = (h.y - an * p.y) - bp * q.y;
        s.hv[i] = make_double2(cr, ci);
        acc += cr * cr + ci * ci;
    }
    double total;
    if (na_grid_sum(acc, s, &total) && threadIdx.x == 0) {
        const double bn = sqrt(fabs(total));
        b[it] = bn;
        if (!(bn > 0.0) || !isfinite(bn)) atomicOr(s.counter + 1, kNaBadNorm);
    }
}

// psi_{n-1} <- psi_n, psi_n <- r / b_n.
__global__ void k_na_shift(int64_t n, NaScratch s, const double* b, int it)
{
    const double bn = b[it];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 h = s.hv[i];
        s.psinm1[i] = s.psin[i];
        s.psin[i] = make_double2(h.x / bn, h.y / bn);
    }
}

constexpr int kNaMaxDevices = 64;
std::mutex g_na_mutex;
unsigned char* g_na_ptr[kNaMaxDevices];
unsigned long long g_na_ctx_id[kNaMaxDevices];   // unique id of the context the address belongs to

// Driver entry points reached through the runtime (no link to the driver library): the current context
// and its unique id, which CUDA never reuses, so that an address looked up before a device reset (which
// destroys the context and unloads this module from it) is not used afterwards.
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

bool current_context_id(unsigned long long* id)
{
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static bool looked = false;
    if (!looked) {
        looked = true;
        cudaDriverEntryPointQueryResult q1, q2;
        void* f1 = nullptr;
        void* f2 = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
            q2 == cudaDriverEntryPointSuccess) {
            get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
            get_id = reinterpret_cast<CtxGetIdFn>(f2);
        }
    }
    CUcontext ctx = nullptr;
    return get_current && get_id && get_current(&ctx) == CUDA_SUCCESS && ctx && get_id(ctx, id) == CUDA_SUCCESS;
}

// Device address of g_na_scratch on the current device.  It is looked up (cudaGetSymbolAddress, which
// may load this library's module into the context) on the first call for a device, and again when that
// device's context is a new one (after a reset); otherwise the cached address is used.  A caller that
// cannot tell the context's identity (driver entry points unavailable) gets a lookup on every call.
int na_scratch_on_current_device(unsigned char** out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return GBN_ERR_CUDA;
    if (dev < 0 || dev >= kNaMaxDevices) return GBN_ERR_ARG;
    if (cudaSetDevice(dev) != cudaSuccess) return GBN_ERR_CUDA;   // makes the device's context current
    unsigned long long id = 0;
    const bool have_id = current_context_id(&id);
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_ptr[dev] || !have_id || g_na_ctx_id[dev] != id) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_na_scratch) != cudaSuccess || !p) return GBN_ERR_CUDA;
        g_na_ptr[dev] = static_cast<unsigned char*>(p);
        g_na_ctx_id[dev] = have_id ? id : 0ull;
    }
    *out = g_na_ptr[dev];
    return GBN_OK;
}

}  // namespace

extern "C" int gbn_lanczos_noalloc(int64_t n, int32_t max_neigh, const int32_t* nneigh, const int32_t* nlist,
                                   const double* hopp, const double* h0, const double* psi, int32_t nrecurs,
                                   double* a, double* b, void* stream)
{
    if (n > GBN_NOALLOC_MAX_ATOMS) return GBN_ERR_LIMIT;
    if (n < 1 || max_neigh < 1 || nrecurs < 1) return GBN_ERR_ARG;
    if (!nneigh || !nlist || !hopp || !h0 || !psi || !a || !b) return GBN_ERR_ARG;
    if (((uintptr_t)hopp | (uintptr_t)psi) & 15) return GBN_ERR_ARG;  // read as 16-byte complex values
    unsigned char* base = nullptr;
    int rc = na_scratch_on_current_device(&base);
    if (rc) return rc;
    const NaScratch s = na_layout(base);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // The array keeps the previous call's contents: the counter and the error flags must start at 0.
    if (cudaMemsetAsync(s.counter, 0, 2 * sizeof(unsigned int), st) != cudaSuccess) return GBN_ERR_CUDA;
    const int blocks = (int)((n + kNaThreads - 1) / kNaThreads < kNaMaxBlocks ? (n + kNaThreads - 1) / kNaThreads
                                                                              : kNaMaxBlocks);
    k_na_start<<<blocks, kNaThreads, 0, st>>>(reinterpret_cast<const double2*>(psi), n, s);
    for (int it = 0; it < nrecurs; ++it) {
        k_na_apply<<<blocks, kNaThreads, 0, st>>>(n, max_neigh, nneigh, nlist, reinterpret_cast<const double2*>(hopp),
                                                  h0, s, a, it);
        k_na_residual<<<blocks, kNaThreads, 0, st>>>(n, s, a, b, it);
        k_na_shift<<<blocks, kNaThreads, 0, st>>>(n, s, b, it);
    }
    if (cudaGetLastError() != cudaSuccess) return GBN_ERR_CUDA;
    unsigned int flags = 0;
    if (cudaMemcpyAsync(&flags, s.counter + 1, sizeof(flags), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return GBN_ERR_CUDA;
    if (flags & kNaBadIndex) return GBN_ERR_ARG;
    if (flags & kNaBadNorm) return GBN_ERR_NUMERIC;
    return GBN_OK;
}
