// Row-by-row products of the Galerkin triple product; see rowprod.cuh. Thread blocks of
// 192 threads, one per output row (and tile of its slots):
//   1. (k_rows_count) the row's A entries are staged in shared memory, a thread each:
//      the first entry of its B row inside the window (a binary search, kept for step 2)
//      and the count from there; then all candidates, split evenly over the threads,
//      set their column's bit in a shared bitmap of the window. The row's count is the
//      bitmap's.
//   2. (k_rows_fill) the bitmap again, a scan of its words' counts (a column's slot is
//      the count of the bits below it), the sorted columns written, then the values:
//      A's entries in order, 32 groups of six threads taking B row j's entries (thread
//      c of a group owns column c of the output block, as the sorted-candidate sums do),
//      the blocks summed in shared memory and written once. A barrier after each A entry
//      keeps the additions to one block in A's entry order, so every load is issued
//      ahead of the barrier it would otherwise wait at: A's next-but-one block and the
//      first round of the next entry's B blocks are in flight while this entry is added.
//      Rows with more slots than one block holds go in tiles of slots, a block each.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdlib>

#include "kernels.cuh"
#include "rowprod.cuh"

namespace sc {

namespace {

constexpr int RP_THREADS = 192;  // the count kernel's threads; the fill kernel's for long B rows
constexpr int RP_SMALL = 64;     // the fill kernel's threads where B rows are short
constexpr int RP_META = 256;  // A entries staged at a time (SC_ROWS_META lowers it)

// The staged A entries of a segment: the first B entry inside the window, the count
// from there to the end of the B row, its exclusive prefix (pos[nm] = the total), and
// for TRANSPOSED the block of aval.
struct Meta {
    int64_t* f0;
    int* len;
    int* pos;
    int64_t* ent;
};
template <int TH>
using MetaScan = cub::BlockScan<int, TH>;

// Stages A entries [s0, s0 + nm) (nm <= 2 * TH) in M -- thread t takes entries
// 2t and 2t + 1, reading their first B entry from `first`, or, SEARCH, finding it by a
// binary search and storing it in `found` -- then sets the window bits of every B entry
// from there on, the candidates split evenly over the threads with four loads in flight.
// Returns the segment's candidates (block-uniform).
template <bool SEARCH, int MODE, int TH>
__device__ int stage_and_mark(const RowArgs& a, int64_t s0, int nm, int32_t l, int32_t h,
                              const int64_t* __restrict__ first, int64_t* __restrict__ found, const Meta& M,
                              uint32_t* bm, typename MetaScan<TH>::TempStorage& tmp) {
    int len[2] = {0, 0};
#pragma unroll
    for (int u = 0; u < 2; u++) {
        const int m = 2 * (int)threadIdx.x + u;
        if (m < nm) {
            const int64_t e = s0 + m;
            const int32_t j = a.acol[e];
            const int64_t b1 = a.brow[j + 1];
            int64_t f0;
            if (SEARCH) {
                f0 = lower_bound_i32(a.bcol, a.brow[j], b1, l);
                found[e] = f0;
            } else {
                f0 = first[e];
            }
            M.f0[m] = f0;
            len[u] = (int)(b1 - f0);
            M.len[m] = len[u];
            if (MODE == ROWS_TRANSPOSED) M.ent[m] = a.aent[e];
        }
    }
    int pos[2], total;
    MetaScan<TH>(tmp).ExclusiveSum(len, pos, total);
#pragma unroll
    for (int u = 0; u < 2; u++)
        if (2 * (int)threadIdx.x + u < nm) M.pos[2 * threadIdx.x + u] = pos[u];
    if (threadIdx.x == 0) M.pos[nm] = total;
    __syncthreads();
    const int per = (total + TH - 1) / TH;
    int idx = min(total, (int)threadIdx.x * per);
    const int iend = min(total, idx + per);
    if (idx < iend) {
        int lo_m = 0, hi_m = nm;  // the entry holding candidate idx: pos[m] <= idx < pos[m + 1]
        while (hi_m - lo_m > 1) {
            const int mid = (lo_m + hi_m) >> 1;
            if (M.pos[mid] <= idx)
                lo_m = mid;
            else
                hi_m = mid;
        }
        int m = lo_m;
        int64_t f = M.f0[m] + (idx - M.pos[m]);
        int left = M.pos[m + 1] - idx;
        while (idx < iend) {
            int32_t cv[4];
            int k = 0;
#pragma unroll
            for (int u = 0; u < 4; u++) {
                if (idx < iend) {
                    while (left == 0) {
                        m++;
                        f = M.f0[m];
                        left = M.len[m];
                    }
                    cv[u] = a.bcol[f];
                    f++;
                    left--;
                    idx++;
                    k++;
                }
            }
#pragma unroll
            for (int u = 0; u < 4; u++)
                if (u < k) {
                    const uint32_t c = (uint32_t)(cv[u] - l);
                    if (c < (uint32_t)(h - l)) atomicOr(&bm[c >> 5], 1u << (c & 31));
                }
        }
    }
    __syncthreads();
    return total;
}

__global__ void __launch_bounds__(RP_THREADS) k_rows_count(int64_t nrows, RowArgs a, int64_t* __restrict__ first,
                                                         int64_t* __restrict__ cnt,
                                                         unsigned long long* __restrict__ cands) {
    extern __shared__ int64_t cmeta[];
    using Reduce = cub::BlockReduce<int64_t, RP_THREADS>;
    __shared__ union {
        typename Reduce::TempStorage red;
        typename MetaScan<RP_THREADS>::TempStorage scan;
    } tmp;
    const Meta M{cmeta, reinterpret_cast<int*>(cmeta + RP_META), reinterpret_cast<int*>(cmeta + RP_META) + RP_META,
                 nullptr};
    uint32_t* bm = reinterpret_cast<uint32_t*>(M.pos + RP_META + 2);
    const int64_t i = blockIdx.x;
    const int32_t l = a.lo[i], h = a.hi[i];
    const int nw = h > l ? (h - l + 31) >> 5 : 0;
    for (int w = threadIdx.x; w < nw; w += RP_THREADS) bm[w] = 0u;
    __syncthreads();
    int64_t mine = 0;
    if (nw > 0) {
        const int64_t e0 = a.arow[i], e1 = a.arow[i + 1];
        for (int64_t s0 = e0; s0 < e1; s0 += RP_META)
            mine += stage_and_mark<true, ROWS_PLAIN, RP_THREADS>(a, s0, (int)min((int64_t)RP_META, e1 - s0), l, h, nullptr,
                                                     first, M, bm, tmp.scan);
    }
    int64_t n = 0;
    for (int w = threadIdx.x; w < nw; w += RP_THREADS) n += __popc(bm[w]);
    n = Reduce(tmp.red).Sum(n);
    if (threadIdx.x == 0) {
        cnt[i] = n;
        if (mine) atomicAdd(cands, (unsigned long long)mine);
    }
}

// What entry x = 6 r + j of op(A) for A entry e is made from: the value (PLAIN, and
// TRANSPOSED from block ent), or K0's block descriptor; a_make turns it into the value.
template <int MODE>
__device__ __forceinline__ double a_fetch(const RowArgs& a, int64_t e, int64_t ent, int x) {
    if constexpr (MODE == ROWS_K0)
        return (double)a.k0.desc[e];
    else if constexpr (MODE == ROWS_TRANSPOSED)
        return a.aval[36 * ent + 6 * (x % 6) + x / 6];
    else
        return a.aval[36 * e + x];
}
template <int MODE>
__device__ __forceinline__ double a_make(double raw, const double* __restrict__ T, const K0Row& row, int x) {
    if constexpr (MODE == ROWS_K0)
        return k0_entry(T, row, (uint8_t)(int)raw, x / 6, x % 6);
    else
        return raw;
}

// one B entry's column and the thread's column c of its block
struct BEntry {
    int32_t col;
    double b[6];
};

// AREG: each step's A block is copied into registers and held for all the step's rounds
// (else read from shared memory, where it is read again after every accumulator store)
template <int MODE, int TH, bool AREG>
__global__ void __launch_bounds__(TH, TH == RP_THREADS ? 2 : 6) k_rows_fill(int64_t nrows, RowArgs a, const int64_t* __restrict__ first,
                                                           const int64_t* __restrict__ crow,
                                                           int32_t* __restrict__ ccol, double* __restrict__ cval,
                                                           int S, int nwmax, int meta) {
    extern __shared__ double smem[];
    constexpr int NG = TH / 6;  // groups of six threads
    __shared__ typename MetaScan<TH>::TempStorage scan;
    double* acc = smem;                                             // S blocks
    double* T = acc + (size_t)S * 36;                               // K0: the scaled template
    double* Ast = T + (MODE == ROWS_K0 ? 36 * 36 : 0);              // two staged A blocks
    int64_t* mf0 = reinterpret_cast<int64_t*>(Ast + 72);            // the staged A entries
    int64_t* ment = mf0 + meta;
    int* mlen = reinterpret_cast<int*>(ment + meta);
    const Meta M{mf0, mlen, mlen + meta, ment};
    uint32_t* bm = reinterpret_cast<uint32_t*>(M.pos + meta + 2);   // window bitmap
    int* pre = reinterpret_cast<int*>(bm + nwmax);                  // bits below each word

    const int64_t i = blockIdx.x;
    const int32_t l = a.lo[i], h = a.hi[i];
    const int64_t c0 = crow[i];
    const int nslots = (int)(crow[i + 1] - c0);
    const int t0 = (int)blockIdx.y * S;
    if (h <= l || t0 >= nslots) return;
    const int t1 = min(nslots, t0 + S);
    const int nw = (h - l + 31) >> 5;
    if constexpr (MODE == ROWS_K0)
        for (int t = threadIdx.x; t < 36 * 36; t += TH) T[t] = a.k0.tpl_s[t];
    for (int w = threadIdx.x; w < nw; w += TH) bm[w] = 0u;
    for (int x = threadIdx.x; x < S * 36; x += TH) acc[x] = 0.0;
    __syncthreads();
    const int64_t e0 = a.arow[i], e1 = a.arow[i + 1];
    for (int64_t s0 = e0; s0 < e1; s0 += meta)
        stage_and_mark<false, MODE, TH>(a, s0, (int)min((int64_t)meta, e1 - s0), l, h, first, nullptr, M, bm, scan);
    {
        const int per = (nw + TH - 1) / TH;
        const int w0 = min(nw, (int)threadIdx.x * per), w1 = min(nw, w0 + per);
        int s = 0;
        for (int w = w0; w < w1; w++) s += __popc(bm[w]);
        int ex = 0;
        MetaScan<TH>(scan).ExclusiveSum(s, ex);
        for (int w = w0; w < w1; w++) {
            pre[w] = ex;
            ex += __popc(bm[w]);
        }
    }
    __syncthreads();
    if (blockIdx.y == 0)
        for (int w = threadIdx.x; w < nw; w += TH) {
            uint32_t m = bm[w];
            int64_t o = c0 + pre[w];
            while (m) {
                const int b = __ffs(m) - 1;
                ccol[o++] = l + 32 * w + b;
                m &= m - 1u;
            }
        }

    K0Row row{};
    if constexpr (MODE == ROWS_K0) row = k0_row(a.k0, i);
    const int g = threadIdx.x / 6, c = threadIdx.x % 6;
    const bool grp = g < NG;  // the last threads of a 64-thread block make no group
    const int x36 = threadIdx.x;  // the A entry this thread stages, when < 36
    auto fetch = [&](int64_t f, BEntry& x) {
        x.col = a.bcol[f];
        const double* bb = a.bval + 36 * f;
#pragma unroll
        for (int j = 0; j < 6; j++) x.b[j] = bb[6 * j + c];
    };
    // acc(slot) column c += A B_f column c, for a B entry in this tile
    auto add = [&](const double* A, const BEntry& x) {
        const uint32_t col = (uint32_t)(x.col - l);
        if (col >= (uint32_t)(h - l)) return;
        const int w = (int)(col >> 5);
        const int slot = pre[w] + __popc(bm[w] & ((1u << (col & 31)) - 1u)) - t0;
        if ((unsigned)slot >= (unsigned)(t1 - t0)) return;
        double* o = acc + 36 * slot;
#pragma unroll
        for (int r = 0; r < 6; r++) {
            double s = 0.0;
#pragma unroll
            for (int j = 0; j < 6; j++) s = fma(A[6 * r + j], x.b[j], s);
            o[6 * r + c] += s;
        }
    };
    const bool restage = e1 - e0 > meta;  // else the one segment's entries are still staged
    for (int64_t s0 = e0; s0 < e1; s0 += meta) {
        const int nm = (int)min((int64_t)meta, e1 - s0);
        __syncthreads();  // the last segment's users of the staged entries are done
        if (restage) {
            for (int m = threadIdx.x; m < nm; m += TH) {
                const int64_t e = s0 + m;
                mf0[m] = first[e];
                mlen[m] = (int)(a.brow[a.acol[e] + 1] - mf0[m]);
                if constexpr (MODE == ROWS_TRANSPOSED) ment[m] = a.aent[e];
            }
            __syncthreads();
        }
        double araw = 0.0;  // A(m + 1) while entry m is added
        if (x36 < 36) {
            Ast[x36] = a_make<MODE>(a_fetch<MODE>(a, s0, ment[0], x36), T, row, x36);
            if (nm > 1) araw = a_fetch<MODE>(a, s0 + 1, ment[1], x36);
        }
        BEntry nx;
        bool hn = grp && g < mlen[0];
        if (hn) fetch(mf0[0] + g, nx);
        __syncthreads();
        for (int m = 0; m < nm; m++) {
            if (x36 < 36 && m + 1 < nm) {
                Ast[36 * ((m + 1) & 1) + x36] = a_make<MODE>(araw, T, row, x36);
                if (m + 2 < nm) araw = a_fetch<MODE>(a, s0 + m + 2, ment[m + 2], x36);
            }
            double Ar[AREG ? 36 : 1];
            const double* A = Ast + 36 * (m & 1);
            if (AREG) {
#pragma unroll
                for (int x = 0; x < 36; x++) Ar[x] = A[x];
                A = Ar;
            }
            const BEntry cur = nx;
            const bool hc = hn;
            const int64_t fs = mf0[m] + g, fe = mf0[m] + mlen[m];
            hn = false;
            if (m + 1 < nm) {
                hn = grp && g < mlen[m + 1];
                if (hn) fetch(mf0[m + 1] + g, nx);
            }
            if (hc) add(A, cur);
            for (int64_t f = fs + NG; grp && f < fe; f += 2 * NG) {
                BEntry x0, x1;
                fetch(f, x0);
                const bool h1 = f + NG < fe;
                if (h1) fetch(f + NG, x1);
                add(A, x0);
                if (h1) add(A, x1);
            }
            __syncthreads();
        }
    }
    for (int x = threadIdx.x; x < (t1 - t0) * 36; x += TH) cval[36 * (c0 + t0) + x] = acc[x];
}

__global__ void k_kp_windows(int64_t n, const int32_t* __restrict__ up, const int64_t* __restrict__ prow,
                             const int32_t* __restrict__ pcol, const int32_t* __restrict__ piece,
                             const int64_t* __restrict__ cpstart, int32_t* __restrict__ lo, int32_t* __restrict__ hi) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (up[k] < 0 || prow[k + 1] == prow[k]) {
        lo[k] = 0;
        hi[k] = 0;
    } else {
        lo[k] = pcol[prow[k]];
        hi[k] = (int32_t)cpstart[piece[k] + 1];
    }
}

__global__ void k_upper_windows(int64_t nc, const int32_t* __restrict__ cpiece, const int64_t* __restrict__ cpstart,
                                int32_t* __restrict__ lo, int32_t* __restrict__ hi) {
    int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= nc) return;
    lo[c] = (int32_t)c;
    hi[c] = (int32_t)cpstart[cpiece[c] + 1];
}

// staged A entries: first B entry and value block (8 bytes each), count and prefix
size_t meta_bytes(int meta) { return (size_t)meta * 2 * sizeof(int64_t) + (size_t)(2 * meta + 2) * sizeof(int); }

template <int MODE, int TH, bool AREG>
void launch_fill_th(Context& ctx, int64_t nrows, const RowArgs& a, const int64_t* first, const int64_t* crow,
                    int32_t* ccol, double* cval, int S, int ntiles, int nwmax, int meta) {
    meta = std::min(meta, 2 * TH);
    size_t smem = (size_t)S * 36 * sizeof(double) + (MODE == ROWS_K0 ? 36 * 36 * sizeof(double) : 0) +
                  72 * sizeof(double) + meta_bytes(meta) + 2 * (size_t)nwmax * sizeof(uint32_t);
    SC_CK(cudaFuncSetAttribute(k_rows_fill<MODE, TH, AREG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_rows_fill<MODE, TH, AREG><<<dim3((unsigned)nrows, (unsigned)ntiles), TH, smem, ctx.stream>>>(
        nrows, a, first, crow, ccol, cval, S, nwmax, meta);
    SC_LAUNCH_CK();
}

// By the B blocks a step adds on average: under 16, 64-thread blocks (ten groups), so
// more rows run at once and a barrier holds two warps; from 40 (three rounds of the 32
// groups or more), 192 threads holding each A block in registers (fewer shared-memory
// reads, fewer blocks an SM); 192 threads otherwise.
template <int MODE>
void launch_fill(Context& ctx, int64_t nrows, const RowArgs& a, const int64_t* first, const int64_t* crow,
                 int32_t* ccol, double* cval, int S, int ntiles, int nwmax, int meta, int variant) {
    if (variant == 0)
        launch_fill_th<MODE, RP_SMALL, false>(ctx, nrows, a, first, crow, ccol, cval, S, ntiles, nwmax, meta);
    else if (variant == 1)
        launch_fill_th<MODE, RP_THREADS, false>(ctx, nrows, a, first, crow, ccol, cval, S, ntiles, nwmax, meta);
    else
        launch_fill_th<MODE, RP_THREADS, true>(ctx, nrows, a, first, crow, ccol, cval, S, ntiles, nwmax, meta);
}

}  // namespace

void kp_windows(Context& ctx, int64_t n, const int32_t* up, const int64_t* prow, const int32_t* pcol,
                const int32_t* piece, const int64_t* cpstart, int32_t* lo, int32_t* hi) {
    k_kp_windows<<<grid_for(n, 256), 256, 0, ctx.stream>>>(n, up, prow, pcol, piece, cpstart, lo, hi);
    SC_LAUNCH_CK();
}

void upper_windows(Context& ctx, int64_t nc, const int32_t* cpiece, const int64_t* cpstart, int32_t* lo, int32_t* hi) {
    k_upper_windows<<<grid_for(nc, 256), 256, 0, ctx.stream>>>(nc, cpiece, cpstart, lo, hi);
    SC_LAUNCH_CK();
}

void row_products(Context& ctx, int mode, const RowArgs& a, int64_t nrows, int64_t max_width, DBuf<int64_t>& crow,
                  DBuf<int32_t>& ccol, DBuf<double>& cval, int64_t& cnnz, int64_t& cands) {
    require(max_width <= ROWS_MAX_WIDTH, SC_BAD_INPUT, "row products: window wider than the bitmap");
    cudaStream_t st = ctx.stream;
    MemStats* ms = &ctx.mem;
    const int nwmax = (int)std::max<int64_t>((max_width + 31) / 32, 1);
    DBuf<int64_t> first, cnt;
    DBuf<unsigned long long> nc;
    first.alloc(std::max<int64_t>(a.annz, 1), st, ms);
    cnt.alloc(nrows + 1, st, ms);
    nc.alloc(1, st, ms);
    nc.zero();
    SC_CK(cudaMemsetAsync(cnt.get() + nrows, 0, sizeof(int64_t), st));
    if (nrows > 0) {
        const size_t smem = RP_META * sizeof(int64_t) + (2 * RP_META + 2) * sizeof(int) + nwmax * sizeof(uint32_t);
        k_rows_count<<<(unsigned)nrows, RP_THREADS, smem, st>>>(nrows, a, first.get(), cnt.get(), nc.get());
        SC_LAUNCH_CK();
    }
    crow.alloc(nrows + 1, st, ms);
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.get(), crow.get(), nrows + 1, st);
    cub::DeviceScan::ExclusiveSum(ctx.cub_scratch(tb), tb, cnt.get(), crow.get(), nrows + 1, st);
    DBuf<int64_t> most;
    most.alloc(1, st, ms);
    cub::DeviceReduce::Max(nullptr, tb, cnt.get(), most.get(), nrows + 1, st);
    cub::DeviceReduce::Max(ctx.cub_scratch(tb), tb, cnt.get(), most.get(), nrows + 1, st);
    int64_t h[3] = {0, 0, 0};
    SC_CK(cudaMemcpyAsync(&h[0], crow.get() + nrows, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    SC_CK(cudaMemcpyAsync(&h[1], most.get(), sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    SC_CK(cudaMemcpyAsync(&h[2], nc.get(), sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    SC_CK(cudaStreamSynchronize(st));
    cnnz = h[0];
    cands = h[2];
    cnt.release();
    ccol.alloc(std::max<int64_t>(cnnz, 1), st, ms);
    cval.alloc(36 * std::max<int64_t>(cnnz, 1), st, ms);
    if (cnnz == 0) return;
    // slots summed by one block: the widest row, at most 256 blocks (72 KB); wider rows
    // go in several tiles, one block each. SC_ROWS_SLOTS and SC_ROWS_META shrink the
    // tiles and the staged entries (to test the tiling).
    int cap = 256, meta = RP_META;
    if (const char* v = std::getenv("SC_ROWS_SLOTS")) cap = std::max(1, std::min(cap, std::atoi(v)));
    if (const char* v = std::getenv("SC_ROWS_META")) meta = std::max(1, std::min(meta, std::atoi(v)));
    const int S = (int)std::min<int64_t>(cap, (h[1] + 7) / 8 * 8);
    const int ntiles = (int)((h[1] + S - 1) / S);
    require(ntiles <= 65535, SC_BAD_INPUT, "row products: too many slot tiles");
    // the form by the B blocks a step adds on average (see launch_fill); SC_ROWS_VARIANT
    // = 0, 1 or 2 forces one (to test each)
    const int64_t per = cands / std::max<int64_t>(a.annz, 1);
    int variant = per < 16 ? 0 : per < 40 ? 1 : 2;
    if (const char* v = std::getenv("SC_ROWS_VARIANT")) variant = std::max(0, std::min(2, std::atoi(v)));
    if (mode == ROWS_K0)
        launch_fill<ROWS_K0>(ctx, nrows, a, first.get(), crow.get(), ccol.get(), cval.get(), S, ntiles, nwmax, meta,
                             variant);
    else if (mode == ROWS_TRANSPOSED)
        launch_fill<ROWS_TRANSPOSED>(ctx, nrows, a, first.get(), crow.get(), ccol.get(), cval.get(), S, ntiles, nwmax,
                                     meta, variant);
    else
        launch_fill<ROWS_PLAIN>(ctx, nrows, a, first.get(), crow.get(), ccol.get(), cval.get(), S, ntiles, nwmax,
                                meta, variant);
}

}  // namespace sc
