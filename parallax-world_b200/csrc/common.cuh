// Shared plumbing of the statics solver: errors, stream-ordered device buffers that
// count their bytes, launch helpers and 6x6 block arithmetic.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
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

// Device memory accounting of one context: what is held now and at most.
struct MemStats {
    int64_t now = 0, peak = 0;
    void add(int64_t b) {
        now += b;
        if (now > peak) peak = now;
    }
};

// A stream-ordered device array (cudaMallocAsync from the device's pool).
template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
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
            s = o.s;
            stats = o.stats;
            o.p = nullptr;
            o.n = 0;
        }
        return *this;
    }
    ~DBuf() { release(); }

    void release() {
        if (p) {
            cudaFreeAsync(p, s);
            if (stats) stats->now -= (int64_t)(n * sizeof(T));
        }
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count, cudaStream_t stream, MemStats* st) {
        release();
        s = stream;
        stats = st;
        n = count;
        if (count) {
            SC_CK(cudaMallocAsync((void**)&p, count * sizeof(T), stream));
            if (stats) stats->add((int64_t)(count * sizeof(T)));
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
