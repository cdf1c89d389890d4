// sc_compliance_noalloc: the compliance C = f . u of motions the caller already holds
// on the device, computed without allocating any device memory.
//
// Who needs it: a host engine that owns all of the GPU's memory through its own arena
// (a game or simulation that budgets VRAM up front), code that runs while the caller is
// capturing a CUDA graph, and per-frame loops where cudaMalloc's implicit device
// synchronisation would stall the frame. They cannot let the library call cudaMalloc,
// so every other entry point, which takes its work memory from the device pool, is
// closed to them.
//
// The reduction is a deterministic two-stage sum of its own: fixed 8192-value chunks,
// a fixed-order tree inside each chunk, and the chunks' partial sums added by one block
// in a fixed order (strided runs, then a tree). It is not the solver's dot-product sum
// (whose chunks follow the pieces), so the two agree to rounding, not bit for bit. Its
// per-chunk partial sums live in one file-scope device array instead of allocated
// scratch. That array is process-wide: every GPU that loads this library holds its
// 512 KB until the process exits, every call shares it, and it keeps the last call's
// partial sums (each call overwrites the ones it reads before reading them, so nothing
// has to start at zero). Two calls whose kernels overlap on the GPU (different streams,
// no ordering between them) race on it and may return wrong sums: order such calls on
// one stream, or wait for one before starting the other.
//
// The array's device address belongs to the CUDA context that is current, not to the
// device number: an engine may make its own context current or reset the device between
// calls. So each call looks the address up again (cudaGetSymbolAddress, which allocates
// nothing) in the caller's current context, with the caller's device current.
#include <cuda_runtime.h>

#include "../../include/statics_cuda.h"
#include "common.cuh"

namespace sc {
namespace {

constexpr int NOALLOC_BLOCK = 256;
constexpr int64_t NOALLOC_CHUNK = 8192;      // values reduced by one block
constexpr int64_t NOALLOC_PARTIALS = 65536;  // 512 KB of partial sums

static __device__ __align__(256) double g_noalloc_partials[NOALLOC_PARTIALS];

__global__ void __launch_bounds__(NOALLOC_BLOCK) k_noalloc_chunks(const double* __restrict__ f,
                                                                  const double* __restrict__ u, int64_t n,
                                                                  double* __restrict__ partial) {
    int64_t lo = blockIdx.x * NOALLOC_CHUNK;
    int64_t hi = lo + NOALLOC_CHUNK < n ? lo + NOALLOC_CHUNK : n;
    double s = 0.0;
    for (int64_t i = lo + threadIdx.x; i < hi; i += NOALLOC_BLOCK) s = fma(f[i], u[i], s);
    __shared__ double red[NOALLOC_BLOCK];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = NOALLOC_BLOCK / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// The chunks' partial sums, by one block: thread t adds chunks t, t + 256, ... in order,
// then a fixed-order tree (deterministic).
__global__ void __launch_bounds__(NOALLOC_BLOCK) k_noalloc_total(const double* __restrict__ partial, int64_t chunks,
                                                                 double* __restrict__ out) {
    double s = 0.0;
    for (int64_t c = threadIdx.x; c < chunks; c += NOALLOC_BLOCK) s += partial[c];
    __shared__ double red[NOALLOC_BLOCK];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = NOALLOC_BLOCK / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

}  // namespace
}  // namespace sc

extern "C" sc_status sc_compliance_noalloc(const double* loads, const double* motions, int64_t n_values,
                                           double* compliance, void* stream) {
    using namespace sc;
    if (!loads || !motions || !compliance || n_values < 0) return SC_BAD_INPUT;
    if (n_values > SC_NOALLOC_MAX_VALUES) return SC_BAD_INPUT;
    // the array's address in the current context (on the host, g_noalloc_partials names
    // a host-side stand-in, never handed to a kernel)
    void* addr = nullptr;
    if (cudaGetSymbolAddress(&addr, g_noalloc_partials) != cudaSuccess || !addr) return SC_CUDA;
    double* partial = static_cast<double*>(addr);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int64_t chunks = (n_values + NOALLOC_CHUNK - 1) / NOALLOC_CHUNK;
    // launched through cudaLaunchKernel, whose return value is this launch's own result:
    // an error the caller left pending is neither consumed nor reported here
    if (chunks > 0) {
        void* args[] = {(void*)&loads, (void*)&motions, (void*)&n_values, (void*)&partial};
        if (cudaLaunchKernel((const void*)k_noalloc_chunks, dim3((unsigned)chunks), dim3(NOALLOC_BLOCK), args, 0, st) !=
            cudaSuccess)
            return SC_CUDA;
        g_launches.fetch_add(1, std::memory_order_relaxed);
    }
    void* targs[] = {(void*)&partial, (void*)&chunks, (void*)&compliance};
    if (cudaLaunchKernel((const void*)k_noalloc_total, dim3(1), dim3(NOALLOC_BLOCK), targs, 0, st) != cudaSuccess)
        return SC_CUDA;
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return SC_OK;
}

static_assert(SC_NOALLOC_MAX_VALUES == sc::NOALLOC_CHUNK * sc::NOALLOC_PARTIALS,
              "the header's limit is the partial-sum array's capacity");
