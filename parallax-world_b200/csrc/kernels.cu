// Block-sparse products, block Jacobi, restriction, direct top solves and chunked
// reductions, in FP64 and FP32. All are HBM-bound streaming kernels.
#include "kernels.cuh"

namespace sc {

namespace {

// One warp per block row. Lane = 8*g + r: block slot g (4 blocks in flight per warp),
// block row r (lanes with r >= 6 idle). Each lane reads one 6-value row of a block
// (48 B FP64 / 24 B FP32, contiguous across the 6 lanes of a slot) and the 6 values of
// x at the block's column.
template <class T, int MODE>
__global__ void __launch_bounds__(256) k_spmv(int64_t nrows, const int64_t* __restrict__ rowptr,
                                              const int32_t* __restrict__ col, const T* __restrict__ val,
                                              const T* __restrict__ x, const T* __restrict__ r, T* __restrict__ y,
                                              const T* __restrict__ inv, const double* __restrict__ step,
                                              const int32_t* __restrict__ piece, const int32_t* __restrict__ skip_row,
                                              const int32_t* __restrict__ done) {
    int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (row >= nrows) return;
    int lane = threadIdx.x & 31;
    if (skip_row && skip_row[row]) return;
    int p = piece ? piece[row] : 0;
    if (done && done[p]) return;
    int g = lane >> 3, rr = lane & 7;
    T acc = T(0);
    int64_t e0 = rowptr[row], e1 = rowptr[row + 1];
    if (rr < 6) {
        // two of the slot's blocks (e, e + 4) loaded before either is used: 8 blocks in
        // flight per warp; the lane still adds its blocks in the order e0 + g, + 4, + 8, ...
        int64_t e = e0 + g;
        for (; e + 4 < e1; e += 8) {
            int32_t j0 = col[e], j1 = col[e + 4];
            T a0[6], x0[6], a1[6], x1[6];
            ld6<T>(val + 36 * e + 6 * rr, a0);
            ld6<T>(val + 36 * (e + 4) + 6 * rr, a1);
            ld6<T>(x + 6 * (int64_t)j0, x0);
            ld6<T>(x + 6 * (int64_t)j1, x1);
#pragma unroll
            for (int c = 0; c < 6; c++) acc = fma(a0[c], x0[c], acc);
#pragma unroll
            for (int c = 0; c < 6; c++) acc = fma(a1[c], x1[c], acc);
        }
        if (e < e1) {
            int32_t j = col[e];
            T a[6], xv[6];
            ld6<T>(val + 36 * e + 6 * rr, a);
            ld6<T>(x + 6 * (int64_t)j, xv);
#pragma unroll
            for (int c = 0; c < 6; c++) acc = fma(a[c], xv[c], acc);
        }
    }
    acc += __shfl_xor_sync(0xffffffffu, acc, 8);
    acc += __shfl_xor_sync(0xffffffffu, acc, 16);
    // lanes 0..5 hold row values
    if (MODE == SPMV_Y) {
        if (lane < 6) y[6 * row + lane] = acc;
    } else if (MODE == SPMV_ADD) {
        if (lane < 6) y[6 * row + lane] += acc;
    } else if (MODE == SPMV_RES) {
        if (lane < 6) y[6 * row + lane] = r[6 * row + lane] - acc;
    } else {
        T left = (lane < 6) ? r[6 * row + lane] - acc : T(0);
        T l6[6];
#pragma unroll
        for (int c = 0; c < 6; c++) l6[c] = __shfl_sync(0xffffffffu, left, c);
        if (lane < 6) {
            const T* d = inv + 36 * row + 6 * lane;
            T s = T(0);
#pragma unroll
            for (int c = 0; c < 6; c++) s = fma(d[c], l6[c], s);
            y[6 * row + lane] = x[6 * row + lane] + (T)step[p] * s;
        }
    }
}

// The same with each row split over WPR warps, for levels of few, long rows (coarse
// levels and their transfers), where one warp a row leaves the device idle. Warp w of a
// row takes its blocks e0 + 4 w + g, then every 4 WPR, two in flight; the warps' partial
// sums meet in shared memory and are added in warp order (a fixed order).
template <class T, int MODE, int WPR>
__global__ void __launch_bounds__(32 * (WPR > 8 ? WPR : 8)) k_spmv_split(
    int64_t nrows, const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col, const T* __restrict__ val,
    const T* __restrict__ x, const T* __restrict__ r, T* __restrict__ y, const T* __restrict__ inv,
    const double* __restrict__ step, const int32_t* __restrict__ piece, const int32_t* __restrict__ skip_row,
    const int32_t* __restrict__ done) {
    constexpr int RPC = WPR >= 8 ? 1 : 8 / WPR;  // rows per thread block
    constexpr int STRIDE = 4 * WPR;
    __shared__ T part[RPC * WPR][6];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wr = warp % WPR;
    const int64_t row = (int64_t)blockIdx.x * RPC + warp / WPR;
    bool active = row < nrows && !(skip_row && skip_row[row]);
    const int p = active && piece ? piece[row] : 0;
    if (active && done && done[p]) active = false;
    const int g = lane >> 3, rr = lane & 7;
    T acc = T(0);
    if (active && rr < 6) {
        const int64_t e1 = rowptr[row + 1];
        int64_t e = rowptr[row] + 4 * wr + g;
        for (; e + STRIDE < e1; e += 2 * STRIDE) {
            int32_t j0 = col[e], j1 = col[e + STRIDE];
            T a0[6], x0[6], a1[6], x1[6];
            ld6<T>(val + 36 * e + 6 * rr, a0);
            ld6<T>(val + 36 * (e + STRIDE) + 6 * rr, a1);
            ld6<T>(x + 6 * (int64_t)j0, x0);
            ld6<T>(x + 6 * (int64_t)j1, x1);
#pragma unroll
            for (int c = 0; c < 6; c++) acc = fma(a0[c], x0[c], acc);
#pragma unroll
            for (int c = 0; c < 6; c++) acc = fma(a1[c], x1[c], acc);
        }
        if (e < e1) {
            int32_t j = col[e];
            T a[6], xv[6];
            ld6<T>(val + 36 * e + 6 * rr, a);
            ld6<T>(x + 6 * (int64_t)j, xv);
#pragma unroll
            for (int c = 0; c < 6; c++) acc = fma(a[c], xv[c], acc);
        }
    }
    acc += __shfl_xor_sync(0xffffffffu, acc, 8);
    acc += __shfl_xor_sync(0xffffffffu, acc, 16);
    if (lane < 6) part[warp][lane] = acc;
    __syncthreads();
    if (!active || wr != 0) return;  // whole warps
    acc = T(0);
    if (lane < 6)
#pragma unroll
        for (int w = 0; w < WPR; w++) acc += part[warp + w][lane];
    if (MODE == SPMV_Y) {
        if (lane < 6) y[6 * row + lane] = acc;
    } else if (MODE == SPMV_ADD) {
        if (lane < 6) y[6 * row + lane] += acc;
    } else if (MODE == SPMV_RES) {
        if (lane < 6) y[6 * row + lane] = r[6 * row + lane] - acc;
    } else {
        T left = (lane < 6) ? r[6 * row + lane] - acc : T(0);
        T l6[6];
#pragma unroll
        for (int c = 0; c < 6; c++) l6[c] = __shfl_sync(0xffffffffu, left, c);
        if (lane < 6) {
            const T* d = inv + 36 * row + 6 * lane;
            T s = T(0);
#pragma unroll
            for (int c = 0; c < 6; c++) s = fma(d[c], l6[c], s);
            y[6 * row + lane] = x[6 * row + lane] + (T)step[p] * s;
        }
    }
}

// The same with half a warp a row (two rows a warp), for rows of a few blocks (the
// level-1 prolongation: P has about nine blocks a row): lanes 8 g + r of a half, g = 0, 1,
// take the row's blocks e0 + g, then every two, two in flight.
template <class T, int MODE>
__global__ void __launch_bounds__(256) k_spmv_half(int64_t nrows, const int64_t* __restrict__ rowptr,
                                                   const int32_t* __restrict__ col, const T* __restrict__ val,
                                                   const T* __restrict__ x, const T* __restrict__ r, T* __restrict__ y,
                                                   const T* __restrict__ inv, const double* __restrict__ step,
                                                   const int32_t* __restrict__ piece,
                                                   const int32_t* __restrict__ skip_row,
                                                   const int32_t* __restrict__ done) {
    const int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 4;
    const int lane = threadIdx.x & 31, h = lane & 16, hl = lane & 15;
    bool active = row < nrows && !(skip_row && skip_row[row]);
    const int p = active && piece ? piece[row] : 0;
    if (active && done && done[p]) active = false;
    const int g = hl >> 3, rr = hl & 7;
    T acc = T(0);
    if (active && rr < 6) {
        const int64_t e1 = rowptr[row + 1];
        int64_t e = rowptr[row] + g;
        for (; e + 2 < e1; e += 4) {
            int32_t j0 = col[e], j1 = col[e + 2];
            T a0[6], x0[6], a1[6], x1[6];
            ld6<T>(val + 36 * e + 6 * rr, a0);
            ld6<T>(val + 36 * (e + 2) + 6 * rr, a1);
            ld6<T>(x + 6 * (int64_t)j0, x0);
            ld6<T>(x + 6 * (int64_t)j1, x1);
#pragma unroll
            for (int c = 0; c < 6; c++) acc = fma(a0[c], x0[c], acc);
#pragma unroll
            for (int c = 0; c < 6; c++) acc = fma(a1[c], x1[c], acc);
        }
        if (e < e1) {
            int32_t j = col[e];
            T a[6], xv[6];
            ld6<T>(val + 36 * e + 6 * rr, a);
            ld6<T>(x + 6 * (int64_t)j, xv);
#pragma unroll
            for (int c = 0; c < 6; c++) acc = fma(a[c], xv[c], acc);
        }
    }
    acc += __shfl_xor_sync(0xffffffffu, acc, 8);
    // lanes h + 0..5 hold the half's row values
    if (MODE == SPMV_Y) {
        if (active && hl < 6) y[6 * row + hl] = acc;
    } else if (MODE == SPMV_ADD) {
        if (active && hl < 6) y[6 * row + hl] += acc;
    } else if (MODE == SPMV_RES) {
        if (active && hl < 6) y[6 * row + hl] = r[6 * row + hl] - acc;
    } else {
        T left = (active && hl < 6) ? r[6 * row + hl] - acc : T(0);
        T l6[6];
#pragma unroll
        for (int c = 0; c < 6; c++) l6[c] = __shfl_sync(0xffffffffu, left, h + c);
        if (active && hl < 6) {
            const T* d = inv + 36 * row + 6 * hl;
            T s = T(0);
#pragma unroll
            for (int c = 0; c < 6; c++) s = fma(d[c], l6[c], s);
            y[6 * row + hl] = x[6 * row + hl] + (T)step[p] * s;
        }
    }
}

template <class T>
__global__ void k_jacobi(int64_t n, const T* __restrict__ inv, const T* __restrict__ r, T* __restrict__ x,
                         const double* __restrict__ step, const int32_t* __restrict__ piece,
                         const int32_t* __restrict__ skip_row, const int32_t* __restrict__ done) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (skip_row && skip_row[k]) return;
    int p = piece ? piece[k] : 0;
    if (done && done[p]) return;
    T rv[6], o[6];
    ld6<T>(r + 6 * k, rv);
    T st = step ? (T)step[p] : T(1);
    const T* d = inv + 36 * k;
#pragma unroll
    for (int i = 0; i < 6; i++) {
        T s = T(0);
#pragma unroll
        for (int c = 0; c < 6; c++) s = fma(d[6 * i + c], rv[c], s);
        o[i] = s * st;
    }
    st6<T>(x + 6 * k, o);
}

template <class T>
__global__ void k_jacobi_add(int64_t n, const T* __restrict__ inv, const T* __restrict__ left, const T* __restrict__ x,
                             T* __restrict__ z, const double* __restrict__ step, const int32_t* __restrict__ piece,
                             const int32_t* __restrict__ skip_row, const int32_t* __restrict__ done) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (skip_row && skip_row[k]) return;
    int p = piece ? piece[k] : 0;
    if (done && done[p]) return;
    T lv[6], xv[6], o[6];
    ld6<T>(left + 6 * k, lv);
    ld6<T>(x + 6 * k, xv);
    T st = (T)step[p];
    const T* d = inv + 36 * k;
#pragma unroll
    for (int i = 0; i < 6; i++) {
        T s = T(0);
#pragma unroll
        for (int c = 0; c < 6; c++) s = fma(d[6 * i + c], lv[c], s);
        o[i] = xv[i] + st * s;
    }
    st6<T>(z + 6 * k, o);
}

// rc[c] = sum over P entries e in column c (fine row k) of P[e]' left[k].
template <class T>
__global__ void __launch_bounds__(256) k_restrict(int64_t nc, const int64_t* __restrict__ tptr,
                                                  const int64_t* __restrict__ tent, const int32_t* __restrict__ trow,
                                                  const T* __restrict__ pval, const T* __restrict__ left,
                                                  T* __restrict__ rc, const int32_t* __restrict__ piece_c,
                                                  const int32_t* __restrict__ done) {
    int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (c >= nc) return;
    int lane = threadIdx.x & 31;
    if (done && done[piece_c[c]]) return;
    int g = lane >> 3, rr = lane & 7;
    T acc = T(0);
    if (rr < 6) {
        for (int64_t t = tptr[c] + g; t < tptr[c + 1]; t += 4) {
            int64_t e = tent[t];
            int32_t k = trow[t];
            T lv[6];
            ld6<T>(left + 6 * (int64_t)k, lv);
            const T* b = pval + 36 * e + rr;
#pragma unroll
            for (int j = 0; j < 6; j++) acc = fma(b[6 * j], lv[j], acc);
        }
    }
    acc += __shfl_xor_sync(0xffffffffu, acc, 8);
    acc += __shfl_xor_sync(0xffffffffu, acc, 16);
    if (lane < 6) rc[6 * c + lane] = acc;
}

// z = Kinv r over each top piece's parts; one block per piece, FP64 arithmetic.
template <class T>
__global__ void __launch_bounds__(512) k_top_solve(const int32_t* __restrict__ top, const int64_t* __restrict__ pstart,
                                                   const int64_t* __restrict__ kinv_off, const double* __restrict__ kinv,
                                                   const T* __restrict__ r, T* __restrict__ z,
                                                   const int32_t* __restrict__ done) {
    extern __shared__ double rs[];
    int p = top[blockIdx.x];
    if (done && done[p]) return;
    int64_t k0 = pstart[p];
    int n = (int)(6 * (pstart[p + 1] - k0));
    const double* A = kinv + kinv_off[blockIdx.x];
    for (int i = threadIdx.x; i < n; i += blockDim.x) rs[i] = (double)r[6 * k0 + i];
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double s = 0.0;
        for (int j = 0; j < n; j++) s = fma(A[(int64_t)j * n + i], rs[j], s);
        z[6 * k0 + i] = (T)s;
    }
}

template <class T>
__global__ void __launch_bounds__(256) k_chunk_dot(const int64_t* __restrict__ chunk_lo, const T* __restrict__ a,
                                                   const T* __restrict__ b, double* __restrict__ partial) {
    int64_t lo = 6 * chunk_lo[blockIdx.x], hi = 6 * chunk_lo[blockIdx.x + 1];
    double s = 0.0;
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) s = fma((double)a[i], (double)b[i], s);
    __shared__ double red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// per piece: the sum of its chunks' partials, one warp per piece (strided lanes, then a
// shuffle tree: a fixed order)
__global__ void k_piece_sum(int np, const int64_t* __restrict__ piece_chunk, const double* __restrict__ partial,
                            double* __restrict__ out) {
    const int p = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (p >= np) return;
    double s = 0.0;
    for (int64_t c = piece_chunk[p] + lane; c < piece_chunk[p + 1]; c += 32) s += partial[c];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) out[p] = s;
}

}  // namespace

template <class T, int WPR>
void launch_split(Context& ctx, int mode, int64_t nrows, const int64_t* rowptr, const int32_t* col, const T* val,
                  const T* x, const T* r, T* y, const T* inv, const double* step, const int32_t* piece,
                  const int32_t* skip_row, const int32_t* done) {
    constexpr int RPC = WPR >= 8 ? 1 : 8 / WPR;
    constexpr int threads = 32 * (WPR > 8 ? WPR : 8);
    const unsigned g = grid_for(nrows, RPC);
    switch (mode) {
        case SPMV_Y:
            k_spmv_split<T, SPMV_Y, WPR><<<g, threads, 0, ctx.stream>>>(nrows, rowptr, col, val, x, r, y, inv, step,
                                                                         piece, skip_row, done);
            break;
        case SPMV_ADD:
            k_spmv_split<T, SPMV_ADD, WPR><<<g, threads, 0, ctx.stream>>>(nrows, rowptr, col, val, x, r, y, inv, step,
                                                                           piece, skip_row, done);
            break;
        case SPMV_RES:
            k_spmv_split<T, SPMV_RES, WPR><<<g, threads, 0, ctx.stream>>>(nrows, rowptr, col, val, x, r, y, inv, step,
                                                                           piece, skip_row, done);
            break;
        default:
            k_spmv_split<T, SPMV_RES_SMOOTH, WPR><<<g, threads, 0, ctx.stream>>>(nrows, rowptr, col, val, x, r, y, inv,
                                                                                  step, piece, skip_row, done);
    }
    SC_LAUNCH_CK();
}

// Warps a row: half a warp (0) where rows average under 12 blocks; one, unless the rows
// are too few to fill the device twice over and each warp would still stream 16 or more
// blocks (doubling up to 32).
static int warps_per_row(int64_t nrows, int64_t nnz) {
    static const int sms = [] {  // once (thread-safe)
        int dev = 0, v = 0;
        SC_CK(cudaGetDevice(&dev));
        SC_CK(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
        return v;
    }();
    const int64_t target = (int64_t)sms * 64;  // two waves of 32 warps an SM
    const int64_t avg = nnz / std::max<int64_t>(nrows, 1);
    if (avg < 12) return 0;
    int w = 1;
    while (w < 32 && nrows * w < target && avg >= 32 * w) w *= 2;
    return w;
}

template <class T>
void spmv(Context& ctx, int mode, int64_t nrows, const int64_t* rowptr, const int32_t* col, const T* val, const T* x,
          const T* r, T* y, const T* inv, const double* step, const int32_t* piece, const int32_t* skip_row,
          const int32_t* done, int64_t nnz) {
    if (nrows <= 0) return;
    const int wpr = nnz > 0 ? warps_per_row(nrows, nnz) : 1;
    if (wpr == 0) {
        const unsigned gh = grid_for(nrows * 16, 256);
        switch (mode) {
            case SPMV_Y:
                k_spmv_half<T, SPMV_Y><<<gh, 256, 0, ctx.stream>>>(nrows, rowptr, col, val, x, r, y, inv, step, piece,
                                                                   skip_row, done);
                break;
            case SPMV_ADD:
                k_spmv_half<T, SPMV_ADD><<<gh, 256, 0, ctx.stream>>>(nrows, rowptr, col, val, x, r, y, inv, step,
                                                                     piece, skip_row, done);
                break;
            case SPMV_RES:
                k_spmv_half<T, SPMV_RES><<<gh, 256, 0, ctx.stream>>>(nrows, rowptr, col, val, x, r, y, inv, step,
                                                                     piece, skip_row, done);
                break;
            default:
                k_spmv_half<T, SPMV_RES_SMOOTH><<<gh, 256, 0, ctx.stream>>>(nrows, rowptr, col, val, x, r, y, inv,
                                                                            step, piece, skip_row, done);
        }
        SC_LAUNCH_CK();
        return;
    }
    switch (wpr) {
        case 2: return launch_split<T, 2>(ctx, mode, nrows, rowptr, col, val, x, r, y, inv, step, piece, skip_row, done);
        case 4: return launch_split<T, 4>(ctx, mode, nrows, rowptr, col, val, x, r, y, inv, step, piece, skip_row, done);
        case 8: return launch_split<T, 8>(ctx, mode, nrows, rowptr, col, val, x, r, y, inv, step, piece, skip_row, done);
        case 16: return launch_split<T, 16>(ctx, mode, nrows, rowptr, col, val, x, r, y, inv, step, piece, skip_row, done);
        case 32: return launch_split<T, 32>(ctx, mode, nrows, rowptr, col, val, x, r, y, inv, step, piece, skip_row, done);
        default: break;
    }
    unsigned g = grid_for(nrows * 32, 256);
    switch (mode) {
        case SPMV_Y:
            k_spmv<T, SPMV_Y><<<g, 256, 0, ctx.stream>>>(nrows, rowptr, col, val, x, r, y, inv, step, piece, skip_row, done);
            break;
        case SPMV_ADD:
            k_spmv<T, SPMV_ADD><<<g, 256, 0, ctx.stream>>>(nrows, rowptr, col, val, x, r, y, inv, step, piece, skip_row, done);
            break;
        case SPMV_RES:
            k_spmv<T, SPMV_RES><<<g, 256, 0, ctx.stream>>>(nrows, rowptr, col, val, x, r, y, inv, step, piece, skip_row, done);
            break;
        default:
            k_spmv<T, SPMV_RES_SMOOTH><<<g, 256, 0, ctx.stream>>>(nrows, rowptr, col, val, x, r, y, inv, step, piece,
                                                                  skip_row, done);
    }
    SC_LAUNCH_CK();
}

template <class T>
void jacobi(Context& ctx, int64_t n, const T* inv, const T* r, T* x, const double* step, const int32_t* piece,
            const int32_t* skip_row, const int32_t* done) {
    if (n <= 0) return;
    k_jacobi<T><<<grid_for(n, 256), 256, 0, ctx.stream>>>(n, inv, r, x, step, piece, skip_row, done);
    SC_LAUNCH_CK();
}

template <class T>
void jacobi_add(Context& ctx, int64_t n, const T* inv, const T* left, const T* x, T* z, const double* step,
                const int32_t* piece, const int32_t* skip_row, const int32_t* done) {
    if (n <= 0) return;
    k_jacobi_add<T><<<grid_for(n, 256), 256, 0, ctx.stream>>>(n, inv, left, x, z, step, piece, skip_row, done);
    SC_LAUNCH_CK();
}

template <class T>
void restrict_t(Context& ctx, int64_t nc, const int64_t* tptr, const int64_t* tent, const int32_t* trow,
                const T* pval, const T* left, T* rc, const int32_t* piece_c, const int32_t* done) {
    if (nc <= 0) return;
    k_restrict<T><<<grid_for(nc * 32, 256), 256, 0, ctx.stream>>>(nc, tptr, tent, trow, pval, left, rc, piece_c, done);
    SC_LAUNCH_CK();
}

template <class T>
void top_solve(Context& ctx, const Level& L, const T* r, T* z, const int32_t* done) {
    if (L.top_h.empty()) return;
    int64_t maxn = 0;
    for (int p : L.top_h) maxn = std::max<int64_t>(maxn, 6 * (L.pstart[p + 1] - L.pstart[p]));
    size_t sm = (size_t)std::max<int64_t>(maxn, 1) * sizeof(double);
    if (sm > 48 * 1024)
        SC_CK(cudaFuncSetAttribute(k_top_solve<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_top_solve<T><<<(unsigned)L.top_h.size(), 512, sm, ctx.stream>>>(L.top.get(), L.pstart_d.get(), L.kinv_off.get(),
                                                                       L.kinv.get(), r, z, done);
    SC_LAUNCH_CK();
}

template <class T>
void seg_dot_t(Context& ctx, const Level& L, const T* a, const T* b, double* out) {
    int np = (int)L.pstart.size() - 1;
    if (ctx.partial.size() < (size_t)std::max<int64_t>(L.nchunks, 1)) ctx.partial.alloc(L.nchunks + 1024, ctx.stream, &ctx.mem);
    if (L.nchunks > 0) {
        k_chunk_dot<T><<<(unsigned)L.nchunks, 256, 0, ctx.stream>>>(L.chunk_lo.get(), a, b, ctx.partial.get());
        SC_LAUNCH_CK();
    }
    k_piece_sum<<<grid_for((int64_t)np * 32, 128), 128, 0, ctx.stream>>>(np, L.piece_chunk.get(), ctx.partial.get(),
                                                                        out);
    SC_LAUNCH_CK();
}

void seg_dot(Context& ctx, const Level& L, const double* a, const double* b, double* out) {
    seg_dot_t<double>(ctx, L, a, b, out);
}

#define SC_INST(T)                                                                                                 \
    template void spmv<T>(Context&, int, int64_t, const int64_t*, const int32_t*, const T*, const T*, const T*, T*, \
                          const T*, const double*, const int32_t*, const int32_t*, const int32_t*, int64_t);       \
    template void jacobi<T>(Context&, int64_t, const T*, const T*, T*, const double*, const int32_t*,              \
                            const int32_t*, const int32_t*);                                                       \
    template void jacobi_add<T>(Context&, int64_t, const T*, const T*, const T*, T*, const double*, const int32_t*, \
                                const int32_t*, const int32_t*);                                                   \
    template void restrict_t<T>(Context&, int64_t, const int64_t*, const int64_t*, const int32_t*, const T*,       \
                                const T*, T*, const int32_t*, const int32_t*);                                     \
    template void top_solve<T>(Context&, const Level&, const T*, T*, const int32_t*);                             \
    template void seg_dot_t<T>(Context&, const Level&, const T*, const T*, double*);
SC_INST(double)
SC_INST(float)

}  // namespace sc
