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
// The reduction is the same deterministic two-stage sum the solver uses for its dot
// products (fixed chunks, fixed-order tree in each chunk, chunks summed in order); its
// per-chunk partial sums live in one file-scope device array instead of allocated
// scratch. That array is process-wide: every GPU that loads this library holds its
// 512 KB until the process exits, every call shares it, and it keeps the last call's
// partial sums (each call overwrites the ones it reads before reading them, so nothing
// has to start at zero). Two calls whose kernels overlap on the GPU (different streams,
// no ordering between them) race on it and may return wrong sums: order such calls on
// one stream, or wait for one before starting the other.
#include <cuda_runtime.h>

#include <mutex>

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

// The chunks' partial sums added in chunk order by one thread (deterministic).
__global__ void k_noalloc_total(const double* __restrict__ partial, int64_t chunks, double* __restrict__ out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double s = 0.0;
    for (int64_t c = 0; c < chunks; c++) s += partial[c];
    *out = s;
}

// The array's device address, looked up once per device with that device current. On
// the host, `g_noalloc_partials` names a host-side stand-in, not device memory, so it is
// never handed to a kernel.
constexpr int MAX_DEVICES = 64;
std::mutex g_lookup;
double* g_partials_of[MAX_DEVICES] = {};

sc_status partials_for_current_device(double** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) {
        cudaGetLastError();
        return SC_NO_DEVICE;
    }
    std::lock_guard<std::mutex> lock(g_lookup);
    if (!g_partials_of[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || !p) {
            cudaGetLastError();
            return SC_CUDA;
        }
        g_partials_of[dev] = static_cast<double*>(p);
    }
    *out = g_partials_of[dev];
    return SC_OK;
}

}  // namespace
}  // namespace sc

extern "C" sc_status sc_compliance_noalloc(const double* loads, const double* motions, int64_t n_values,
                                           double* compliance, void* stream) {
    using namespace sc;
    if (!loads || !motions || !compliance || n_values < 0) return SC_BAD_INPUT;
    if (n_values > SC_NOALLOC_MAX_VALUES) return SC_BAD_INPUT;
    double* partial = nullptr;
    sc_status s = partials_for_current_device(&partial);
    if (s != SC_OK) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int64_t chunks = (n_values + NOALLOC_CHUNK - 1) / NOALLOC_CHUNK;
    if (chunks > 0) {
        k_noalloc_chunks<<<(unsigned)chunks, NOALLOC_BLOCK, 0, st>>>(loads, motions, n_values, partial);
        g_launches.fetch_add(1, std::memory_order_relaxed);
    }
    k_noalloc_total<<<1, 1, 0, st>>>(partial, chunks, compliance);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (cudaGetLastError() != cudaSuccess) return SC_CUDA;
    return SC_OK;
}

static_assert(SC_NOALLOC_MAX_VALUES == sc::NOALLOC_CHUNK * sc::NOALLOC_PARTIALS,
              "the header's limit is the partial-sum array's capacity");
