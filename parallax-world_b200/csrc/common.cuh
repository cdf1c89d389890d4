// Shared plumbing of the statics solver: errors, stream-ordered device buffers that
// count their bytes, launch helpers and 6x6 block arithmetic.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cstdint>
#include <algorithm>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/statics_cuda.h"

namespace sc {

struct Error : std::runtime_error {
    sc_status status;
    Error(sc_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

#define SC_CK(call)                                                                                   \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            throw ::sc::Error(SC_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_) + " (" +    \
                                           __FILE__ + ":" + std::to_string(__LINE__) + ")");         \
    } while (0)

extern std::atomic<int64_t> g_launches;  // kernels launched by this library
#define SC_LAUNCH_CK()                                   \
    do {                                                 \
        ::sc::g_launches.fetch_add(1, std::memory_order_relaxed); \
        SC_CK(cudaGetLastError());                       \
    } while (0)

inline void require(bool ok, sc_status s, const std::string& msg) {
    if (!ok) throw Error(s, msg);
}

// Device memory of one context: what is held now and at most, the host time spent in
// the driver's allocate and free calls, and a cache of released blocks. Every buffer of a
// context lives on the context's one stream, so a released block can be handed to the
// next request on that stream at once (stream order keeps the old and new users apart),
// as cudaFreeAsync / cudaMallocAsync would, but without calling the driver, whose
// allocation calls were measured at milliseconds each: repeated solves of similar sizes
// then allocate nothing. Requests are rounded up to size classes (1/8 steps of their
// power of two, at least 512 bytes) and served by the smallest cached block of at least
// their class and at most twice it, so that similar sizes share blocks (a batch's groups
// differ in size, and a miss grows the driver's pool by mapping new memory, at tens of
// milliseconds a gigabyte; the slack counts as held). Like a caching
// allocator, the cache keeps what it is given up to `cap` bytes (half the device's memory
// by default); when the pool runs out, an allocation gives the cached blocks back and
// tries again.
struct MemStats {
    int64_t now = 0, peak = 0, top = 0;
    double alloc_ms = 0;
    int64_t allocs = 0;
    std::multimap<size_t, void*> cache;  // block bytes -> block
    size_t cached = 0;
    size_t cap = size_t(64) << 30;
    void add(int64_t b) {
        now += b;
        if (now > peak) peak = now;
        if (now > top) top = now;
    }
    static size_t size_class(size_t bytes) {
        if (bytes <= 512) return 512;
        size_t p2 = size_t(1) << (63 - __builtin_clzll((unsigned long long)(bytes - 1)));  // < bytes <= 2 p2
        size_t step = std::max<size_t>(p2 / 8, 512);
        return (bytes + step - 1) / step * step;
    }
    // the smallest cached block of at least `bytes` (a size class) and at most twice it,
    // or null; `bytes` becomes the block's size
    void* take(size_t& bytes) {
        auto it = cache.lower_bound(bytes);
        if (it == cache.end() || it->first > 2 * bytes) return nullptr;
        void* p = it->second;
        bytes = it->first;
        cached -= bytes;
        cache.erase(it);
        return p;
    }
    bool give(void* p, size_t bytes) {
        if (cached + bytes > cap) return false;
        cache.emplace(bytes, p);
        cached += bytes;
        return true;
    }
    // frees every cached block (stream-ordered on s)
    void trim(cudaStream_t s) {
        for (auto& kv : cache) cudaFreeAsync(kv.second, s);
        cache.clear();
        cached = 0;
    }
};

// A device array on a context's stream: from the context's block cache, else from the
// device's pool (cudaMallocAsync); released into the cache, else to the pool.
template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    size_t bytes = 0;  // the block's size (at least n * sizeof(T))
    cudaStream_t s = nullptr;
    MemStats* stats = nullptr;

    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept { *this = std::move(o); }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            n = o.n;
            bytes = o.bytes;
            s = o.s;
            stats = o.stats;
            o.p = nullptr;
            o.n = 0;
            o.bytes = 0;
        }
        return *this;
    }
    ~DBuf() { release(); }

    void release() {
        if (p) {
            if (stats) {
                stats->now -= (int64_t)bytes;
                if (!stats->give(p, bytes)) {
                    auto t0 = std::chrono::steady_clock::now();
                    cudaFreeAsync(p, s);
                    stats->alloc_ms +=
                        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
                }
            } else {
                cudaFreeAsync(p, s);
            }
        }
        p = nullptr;
        n = 0;
        bytes = 0;
    }
    void alloc(size_t count, cudaStream_t stream, MemStats* st) {
        release();
        s = stream;
        stats = st;
        n = count;
        if (!count) return;
        size_t want = count * sizeof(T);
        if (stats) {
            want = MemStats::size_class(want);
            if (void* q = stats->take(want)) {
                p = static_cast<T*>(q);
                bytes = want;
                stats->add((int64_t)bytes);
                return;
            }
        }
        auto t0 = std::chrono::steady_clock::now();
        cudaError_t e = cudaMallocAsync((void**)&p, want, stream);
        if (e == cudaErrorMemoryAllocation && stats && stats->cached) {
            cudaGetLastError();  // out of memory with blocks cached: give them back and retry
            stats->trim(stream);
            e = cudaMallocAsync((void**)&p, want, stream);
        }
        if (e != cudaSuccess) {
            p = nullptr;
            n = 0;
            SC_CK(e);
        }
        bytes = want;
        if (stats) {
            stats->add((int64_t)bytes);
            stats->alloc_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            stats->allocs++;
        }
    }
    void zero() {
        if (n) SC_CK(cudaMemsetAsync(p, 0, n * sizeof(T), s));
    }
    void upload(const T* host, size_t count) {
        if (count) SC_CK(cudaMemcpyAsync(p, host, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void download(T* host, size_t count) const {
        if (count) SC_CK(cudaMemcpyAsync(host, p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
    }
    std::vector<T> to_host() const {
        std::vector<T> h(n);
        download(h.data(), n);
        SC_CK(cudaStreamSynchronize(s));
        return h;
    }
    T* get() const { return p; }
    size_t size() const { return n; }
};

inline unsigned grid_for(int64_t n, int block) {
    int64_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > 0x7fffffffLL) g = 0x7fffffffLL;
    return (unsigned)g;
}

// ---------------------------------------------------------------- 6x6 block math
// Blocks are 36 values, row-major. Six-vectors are 6 consecutive values.

template <class T, class U>
__device__ __forceinline__ void mv6(const T* __restrict__ a, const U (&x)[6], U (&y)[6]) {
#pragma unroll
    for (int r = 0; r < 6; r++) {
        U acc = U(0);
#pragma unroll
        for (int c = 0; c < 6; c++) acc = fma(U(a[6 * r + c]), x[c], acc);
        y[r] = acc;
    }
}

template <class T, class U>
__device__ __forceinline__ void mv6t(const T* __restrict__ a, const U (&x)[6], U (&y)[6]) {
#pragma unroll
    for (int r = 0; r < 6; r++) {
        U acc = U(0);
#pragma unroll
        for (int c = 0; c < 6; c++) acc = fma(U(a[6 * c + r]), x[c], acc);
        y[r] = acc;
    }
}

// Gauss-Jordan inverse with partial pivoting, the last of equal maxima taken as the
// pivot (statics/src/bodies.rs:576-602). Returns false on a zero or non-finite pivot.
__host__ __device__ inline bool invert6(const double* m, double* out) {
    double a[6][6], inv[6][6];
    for (int r = 0; r < 6; r++)
        for (int c = 0; c < 6; c++) {
            a[r][c] = m[6 * r + c];
            inv[r][c] = r == c ? 1.0 : 0.0;
        }
    bool ok = true;
    for (int col = 0; col < 6; col++) {
        int piv = col;
        double best = fabs(a[col][col]);
        for (int x = col + 1; x < 6; x++) {
            double v = fabs(a[x][col]);
            if (v >= best) {
                best = v;
                piv = x;
            }
        }
        if (piv != col)
            for (int k = 0; k < 6; k++) {
                double t = a[col][k];
                a[col][k] = a[piv][k];
                a[piv][k] = t;
                t = inv[col][k];
                inv[col][k] = inv[piv][k];
                inv[piv][k] = t;
            }
        double d = a[col][col];
        if (!(d != 0.0) || !isfinite(d)) ok = false;
        for (int k = 0; k < 6; k++) {
            a[col][k] /= d;
            inv[col][k] /= d;
        }
        for (int r = 0; r < 6; r++) {
            double f = a[r][col];
            if (r != col && f != 0.0)
                for (int k = 0; k < 6; k++) {
                    a[r][k] -= f * a[col][k];
                    inv[r][k] -= f * inv[col][k];
                }
        }
    }
    for (int r = 0; r < 6; r++)
        for (int c = 0; c < 6; c++) out[6 * r + c] = inv[r][c];
    return ok;
}

}  // namespace sc
