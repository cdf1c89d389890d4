// Device kernels shared by the setup and the solve: block-sparse products, block
// Jacobi, transfers, chunked reductions. See solver.cuh for the data layout.
#pragma once
#include "solver.cuh"

namespace sc {

enum SpmvMode { SPMV_Y = 0, SPMV_ADD = 1, SPMV_RES = 2, SPMV_RES_SMOOTH = 3 };

__device__ __forceinline__ int64_t lower_bound_i32(const int32_t* __restrict__ a, int64_t lo, int64_t hi, int32_t v) {
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (a[mid] < v)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

template <class T>
__device__ __forceinline__ void ld6(const T* __restrict__ p, T (&o)[6]) {
    if constexpr (sizeof(T) == 8) {
        const double2* q = reinterpret_cast<const double2*>(p);
        double2 a = q[0], b = q[1], c = q[2];
        o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y; o[4] = c.x; o[5] = c.y;
    } else {
        const float2* q = reinterpret_cast<const float2*>(p);
        float2 a = q[0], b = q[1], c = q[2];
        o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y; o[4] = c.x; o[5] = c.y;
    }
}
template <class T>
__device__ __forceinline__ void st6(T* __restrict__ p, const T (&o)[6]) {
    if constexpr (sizeof(T) == 8) {
        double2* q = reinterpret_cast<double2*>(p);
        q[0] = make_double2(o[0], o[1]);
        q[1] = make_double2(o[2], o[3]);
        q[2] = make_double2(o[4], o[5]);
    } else {
        float2* q = reinterpret_cast<float2*>(p);
        q[0] = make_float2(o[0], o[1]);
        q[1] = make_float2(o[2], o[3]);
        q[2] = make_float2(o[4], o[5]);
    }
}

// Host launchers (kernels.cu).
// nnz (the stored blocks) picks the warps a row (one when 0); see warps_per_row.
template <class T>
void spmv(Context& ctx, int mode, int64_t nrows, const int64_t* rowptr, const int32_t* col, const T* val, const T* x,
          const T* r, T* y, const T* inv, const double* step, const int32_t* piece, const int32_t* skip_row,
          const int32_t* done, int64_t nnz = 0);
template <class T>
void jacobi(Context& ctx, int64_t n, const T* inv, const T* r, T* x, const double* step, const int32_t* piece,
            const int32_t* skip_row, const int32_t* done);
// z = x + step D^-1 left (the post-smoothing step, bodies.rs:396-401)
template <class T>
void jacobi_add(Context& ctx, int64_t n, const T* inv, const T* left, const T* x, T* z, const double* step,
                const int32_t* piece, const int32_t* skip_row, const int32_t* done);
template <class T>
void restrict_t(Context& ctx, int64_t ncoarse, const int64_t* tptr, const int64_t* tent, const int32_t* trow,
                const T* pval, const T* left, T* rc, const int32_t* piece_c, const int32_t* done);
template <class T>
void top_solve(Context& ctx, const Level& L, const T* r, T* z, const int32_t* done);
// out[p] = sum over piece p's parts of a.b (6 values a part), deterministic.
template <class T>
void seg_dot_t(Context& ctx, const Level& L, const T* a, const T* b, double* out);

}  // namespace sc
