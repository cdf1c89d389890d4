// The solve: conjugate gradients on level 0 (statics/src/bodies.rs:338-373),
// preconditioned by one V-cycle (bodies.rs:377-403), for every piece of a batch at
// once with per-piece scalars; and the mixed-precision variant, FP32 operators inside
// FP64 iterative refinement.
#include <chrono>

#include <cstdlib>
#include <type_traits>

#include "kernels.cuh"

namespace sc {

template <class T>
static const T* VAL(const Level& L);
template <>
const double* VAL<double>(const Level& L) { return L.val.get(); }
template <>
const float* VAL<float>(const Level& L) { return L.val32.get(); }
template <class T>
static const T* INV(const Level& L);
template <>
const double* INV<double>(const Level& L) { return L.inv.get(); }
template <>
const float* INV<float>(const Level& L) { return L.inv32.get(); }
template <class T>
static const T* PVAL(const Level& L);
template <>
const double* PVAL<double>(const Level& L) { return L.pval.get(); }
template <>
const float* PVAL<float>(const Level& L) { return L.pval32.get(); }
template <class T>
static const T* PTVAL(const Level& L);
template <>
const double* PTVAL<double>(const Level& L) { return L.ptval.get(); }
template <>
const float* PTVAL<float>(const Level& L) { return L.ptval32.get(); }
template <class T>
static DBuf<T>& VR(Level& L);
template <>
DBuf<double>& VR<double>(Level& L) { return L.r; }
template <>
DBuf<float>& VR<float>(Level& L) { return L.r32; }
template <class T>
static DBuf<T>& VX(Level& L);
template <>
DBuf<double>& VX<double>(Level& L) { return L.x; }
template <>
DBuf<float>& VX<float>(Level& L) { return L.x32; }
template <class T>
static DBuf<T>& VL(Level& L);
template <>
DBuf<double>& VL<double>(Level& L) { return L.left; }
template <>
DBuf<float>& VL<float>(Level& L) { return L.left32; }
template <class T>
static DBuf<T>& VZ(Level& L);
template <>
DBuf<double>& VZ<double>(Level& L) { return L.z; }
template <>
DBuf<float>& VZ<float>(Level& L) { return L.z32; }
template <class T>
static DBuf<T>& VT(Level& L);
template <>
DBuf<double>& VT<double>(Level& L) { return L.t; }
template <>
DBuf<float>& VT<float>(Level& L) { return L.t32; }
template <class T>
static DBuf<T>& VU(Level& L);
template <>
DBuf<double>& VU<double>(Level& L) { return L.u; }
template <>
DBuf<float>& VU<float>(Level& L) { return L.u32; }

template <class T>
void level_apply(Context& ctx, const Batch& b, int l, const T* x, T* y) {
    const Level& L = b.levels[l];
    if (l == 0 && L.matrix_free)
        stencil_apply<T>(ctx, b, x, y, nullptr, nullptr);
    else
        spmv<T>(ctx, SPMV_Y, L.n, L.rowptr.get(), L.col.get(), VAL<T>(L), x, nullptr, y, nullptr, nullptr,
                L.piece.get(), nullptr, nullptr, L.nnzb);
}
template void level_apply<double>(Context&, const Batch&, int, const double*, double*);
template void level_apply<float>(Context&, const Batch&, int, const float*, float*);

template <class T>
static void ensure(Context& ctx, DBuf<T>& v, int64_t n) {
    if ((int64_t)v.size() < n) v.alloc(std::max<int64_t>(n, 1), ctx.stream, &ctx.mem);
}

template <class T>
static void alloc_cycle(Context& ctx, Batch& b) {
    for (size_t l = 0; l < b.levels.size(); l++) {
        Level& L = b.levels[l];
        int64_t n6 = 6 * L.n;
        ensure(ctx, VX<T>(L), n6);
        ensure(ctx, VL<T>(L), n6);
        if (l > 0) {
            ensure(ctx, VR<T>(L), n6);
            ensure(ctx, VZ<T>(L), n6);
        } else if (L.matrix_free && b.levels.size() > 1) {
            ensure(ctx, VT<T>(L), n6);
            ensure(ctx, VU<T>(L), n6);
        }
    }
}

template <class T>
constexpr int fam_of(int f64) {
    return sizeof(T) == 8 ? f64 : f64 + 1;
}
// algorithmic bytes of a block-sparse product: blocks, x once, y (and r) once
template <class T>
static double spmv_bytes(const Level& L, int vec_passes) {
    return (double)sizeof(T) * (36.0 * (double)L.nnzb + 6.0 * (double)L.n * vec_passes);
}
template <class T>
static double transfer_bytes(const Level& L, const Level& C) {
    return (double)sizeof(T) * (36.0 * (double)L.pnnz + 6.0 * (double)L.n + 6.0 * (double)C.n);
}

// One V-cycle from level l: z = M r (bodies.rs:377-403). Pieces whose top is level l are
// solved directly there; the others smooth, hand the residual up, take the correction
// back and smooth again.
template <class T>
static void cycle(Context& ctx, Batch& b, int l, const T* r, T* z, const int32_t* done) {
    Level& L = b.levels[l];
    bool deepest = l + 1 == (int)b.levels.size();
    if (!deepest && l == 0 && L.matrix_free) {
        // level 0 of voxel pieces: smoother and both transfers matrix-free
        Level& C = b.levels[1];
        T* x = VX<T>(L).get();
        level0_down<T>(ctx, b, r, x, VL<T>(L).get(), VT<T>(L).get(), VU<T>(L).get(), VR<T>(C).get(), done);
        cycle<T>(ctx, b, 1, VR<T>(C).get(), VZ<T>(C).get(), done);
        level0_up<T>(ctx, b, r, x, VT<T>(L).get(), VZ<T>(C).get(), z, done);
    } else if (!deepest) {
        const int32_t* skip = L.top_of_part.get();
        T* x = VX<T>(L).get();
        T* left = VL<T>(L).get();
        bool mf = l == 0 && L.matrix_free;
        double vb = (double)sizeof(T) * 6.0 * (double)L.n;
        // x = step D^-1 r (bodies.rs:386), and any further sweeps
        {
            ProfScope ps(ctx, fam_of<T>(SC_FAM_SMOOTH64), 2 * vb + 36.0 * sizeof(T) * L.n);
            jacobi<T>(ctx, L.n, INV<T>(L), r, x, L.step.get(), L.piece.get(), skip, done);
        }
        for (int sweep = 1; sweep < b.sweeps; sweep++) {
            if (mf) {
                level0_smooth<T>(ctx, b, r, x, left, done);
            } else {
                ProfScope ps(ctx, fam_of<T>(SC_FAM_SPMV64), spmv_bytes<T>(L, 3) + vb + 36.0 * sizeof(T) * L.n);
                spmv<T>(ctx, SPMV_RES_SMOOTH, L.n, L.rowptr.get(), L.col.get(), VAL<T>(L), x, r, left, INV<T>(L),
                        L.step.get(), L.piece.get(), skip, done, L.nnzb);
            }
            SC_CK(cudaMemcpyAsync(x, left, 6 * L.n * sizeof(T), cudaMemcpyDeviceToDevice, ctx.stream));
        }
        // left = r - K x (bodies.rs:387)
        if (mf) {
            stencil_residual<T>(ctx, b, x, r, left, skip, done);
        } else {
            ProfScope ps(ctx, fam_of<T>(SC_FAM_SPMV64), spmv_bytes<T>(L, 3));
            spmv<T>(ctx, SPMV_RES, L.n, L.rowptr.get(), L.col.get(), VAL<T>(L), x, r, left, nullptr, nullptr,
                    L.piece.get(), skip, done, L.nnzb);
        }
        Level& C = b.levels[l + 1];
        // coarse = P' left (bodies.rs:388-390)
        {
            ProfScope ps(ctx, fam_of<T>(SC_FAM_TRANSFER64), transfer_bytes<T>(L, C));
            spmv<T>(ctx, SPMV_Y, C.n, L.tptr.get(), L.trow.get(), PTVAL<T>(L), left, nullptr, VR<T>(C).get(),
                    nullptr, nullptr, C.piece.get(), nullptr, done, L.pnnz);
        }
        cycle<T>(ctx, b, l + 1, VR<T>(C).get(), VZ<T>(C).get(), done);
        // x += P y (bodies.rs:392-395)
        {
            ProfScope ps(ctx, fam_of<T>(SC_FAM_TRANSFER64), transfer_bytes<T>(L, C) + vb);
            spmv<T>(ctx, SPMV_ADD, L.n, L.prow.get(), L.pcol.get(), PVAL<T>(L), VZ<T>(C).get(), nullptr, x, nullptr,
                    nullptr, L.piece.get(), skip, done, L.pnnz);
        }
        // z = x + step D^-1 (r - K x) (bodies.rs:396-401), after any further sweeps
        for (int sweep = 1; sweep < b.sweeps; sweep++) {
            if (mf) {
                level0_smooth<T>(ctx, b, r, x, left, done);
            } else {
                ProfScope ps(ctx, fam_of<T>(SC_FAM_SPMV64), spmv_bytes<T>(L, 3) + vb + 36.0 * sizeof(T) * L.n);
                spmv<T>(ctx, SPMV_RES_SMOOTH, L.n, L.rowptr.get(), L.col.get(), VAL<T>(L), x, r, left, INV<T>(L),
                        L.step.get(), L.piece.get(), skip, done, L.nnzb);
            }
            SC_CK(cudaMemcpyAsync(x, left, 6 * L.n * sizeof(T), cudaMemcpyDeviceToDevice, ctx.stream));
        }
        if (mf) {
            stencil_residual<T>(ctx, b, x, r, left, skip, done);
            ProfScope ps(ctx, fam_of<T>(SC_FAM_SMOOTH64), 3 * vb + 36.0 * sizeof(T) * L.n);
            jacobi_add<T>(ctx, L.n, INV<T>(L), left, x, z, L.step.get(), L.piece.get(), skip, done);
        } else {
            ProfScope ps(ctx, fam_of<T>(SC_FAM_SPMV64), spmv_bytes<T>(L, 3) + vb + 36.0 * sizeof(T) * L.n);
            spmv<T>(ctx, SPMV_RES_SMOOTH, L.n, L.rowptr.get(), L.col.get(), VAL<T>(L), x, r, z, INV<T>(L),
                    L.step.get(), L.piece.get(), skip, done, L.nnzb);
        }
    }
    if (!L.top_h.empty()) {
        ProfScope ps(ctx, SC_FAM_TOP, 0.0);
        top_solve<T>(ctx, L, r, z, done);
    }
}

// ---- per-piece CG scalars and chunked vector updates ---------------------------------
namespace {

struct CgScalars {
    double* bb;     // |b|^2
    double* goal;   // tol |b|
    double* rz;
    double* rr;
    double* pap;
    double* next;
    double* alpha;
    int32_t* done;
    int64_t* iters;
    int32_t* status;
    int64_t* replaced;  // per piece: residual replacements (k_cg_verify)
};

__global__ void k_cg_init(int np, double tol, CgScalars s, const int32_t* __restrict__ start_done) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    s.goal[p] = tol * sqrt(s.bb[p]);
    s.done[p] = start_done ? start_done[p] : 0;
    s.iters[p] = 0;
}

// top of an iteration (bodies.rs:352): stop when |r| <= goal; NaN stops with BREAKDOWN
__global__ void k_cg_check(int np, int64_t max_iter, CgScalars s, int32_t* ndone) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    if (!s.done[p]) {
        double nr = sqrt(s.rr[p]);
        if (nr <= s.goal[p]) {
            s.done[p] = 1;
        } else if (!(nr == nr) || !(s.rz[p] == s.rz[p])) {
            s.done[p] = 1;
            atomicMax(s.status + p, (int)SC_BREAKDOWN);
        } else if (s.iters[p] >= max_iter) {
            s.done[p] = 1;
            atomicMax(s.status + p, (int)SC_MAXITER);
        }
    }
    if (s.done[p]) atomicAdd(ndone, 1);
}

__global__ void k_cg_alpha(int np, CgScalars s) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np || s.done[p]) return;
    double pap = s.pap[p];
    if (!(pap > 0.0)) {
        s.done[p] = 1;
        atomicMax(s.status + p, (int)SC_BREAKDOWN);
        return;
    }
    s.alpha[p] = s.rz[p] / pap;  // bodies.rs:356
}

// beta = next / rz; rz = next (bodies.rs:366-370); counts the iteration
__global__ void k_cg_beta(int np, CgScalars s, double* beta) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np || s.done[p]) return;
    beta[p] = s.next[p] / s.rz[p];
    s.rz[p] = s.next[p];
    s.iters[p] += 1;
}

// beta for a preconditioner applied in lower precision (not exactly symmetric): the
// Polak-Ribiere form (z', r' - r) / (z, r) = -alpha (z', Ap) / (z, r), which equals
// next / rz when the preconditioner is symmetric; rz = next; counts the iteration
__global__ void k_cg_beta_flex(int np, CgScalars s, const double* __restrict__ zap, double* beta) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np || s.done[p]) return;
    beta[p] = -s.alpha[p] * zap[p] / s.rz[p];
    s.rz[p] = s.next[p];
    s.iters[p] += 1;
}

// A piece whose recursive residual said converged is held to its true residual
// rr_true = |b - K x|^2, recomputed in FP64: where that misses the goal the piece goes on
// (the recursion drifted from b - K x by more than the tolerance) and is counted, so its
// residual can be replaced by the true one. Pieces stopped by a breakdown or the cap keep
// their status.
__global__ void k_cg_verify(int np, CgScalars s, const double* __restrict__ rr_true, const double* __restrict__ ff,
                            int32_t* __restrict__ count) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    if (!s.done[p] || s.status[p] != (int)SC_OK) return;
    // a piece at its FP64 floor (no FP64 x does better: see k_floor_delta) has met it too
    if (!(sqrt(rr_true[p]) <= fmax(s.goal[p], sqrt(ff[p])))) {
        s.done[p] = 0;
        s.replaced[p] += 1;
        atomicAdd(count, 1);
    }
}

// delta = eps |x| sigma, sigma = +-1 from a hash of the index: x moved by one unit in the
// last place of each value, in random directions. |K delta| is the residual that rounding
// x to FP64 alone leaves, the floor no FP64 vector of motions gets under: on slender
// pieces with large motions it is above 1e-8 |b| (the reference's own FP64 solve stops
// there too), and the solve takes a piece that reached it as converged.
__global__ void k_floor_delta(int64_t n, const double* __restrict__ x, double* __restrict__ delta) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t h = (uint64_t)i * 0x9E3779B97F4A7C15ull;
    h ^= h >> 31;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 29;
    const double sgn = (h >> 63) ? -1.0 : 1.0;
    delta[i] = sgn * 0x1.0p-52 * fabs(x[i]);
}

// The condition of the device-side iteration loop: go on while a piece is not done and
// fewer than `chunk` iterations ran since the launch (count is zeroed before each launch;
// any value it holds ends the loop within chunk + 1 iterations).
__global__ void k_loop_more(cudaGraphConditionalHandle h, const int32_t* __restrict__ ndone, int np,
                            uint32_t* __restrict__ count, uint32_t chunk) {
    uint32_t c = *count + 1u;
    *count = c;
    cudaGraphSetConditional(h, (*ndone < np && c < chunk) ? 1u : 0u);
}

// b = a in another precision for the pieces not done, one block per chunk
template <class A, class B>
__global__ void __launch_bounds__(256) k_cast_chunks(const int64_t* __restrict__ chunk_lo,
                                                     const int32_t* __restrict__ cpiece, const int32_t* __restrict__ done,
                                                     const A* __restrict__ a, B* __restrict__ b) {
    int c = blockIdx.x;
    if (done && done[cpiece[c]]) return;
    int64_t lo = 6 * chunk_lo[c], hi = 6 * chunk_lo[c + 1];
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) b[i] = (B)a[i];
}

// x += alpha p; r -= alpha Ap (bodies.rs:357-362), one block per chunk
template <class V, class S>
__global__ void __launch_bounds__(256) k_axpy2(const int64_t* __restrict__ chunk_lo, const int32_t* __restrict__ cpiece,
                                               const int32_t* __restrict__ done, const double* __restrict__ alpha,
                                               S* __restrict__ x, const V* __restrict__ p, V* __restrict__ r,
                                               const V* __restrict__ ap, float* __restrict__ r32) {
    int c = blockIdx.x;
    int pc = cpiece[c];
    if (done[pc]) return;
    double a = alpha[pc];
    int64_t lo = 6 * chunk_lo[c], hi = 6 * chunk_lo[c + 1];
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        x[i] += (S)(a * (double)p[i]);
        const V rn = (V)((double)r[i] - a * (double)ap[i]);
        r[i] = rn;
        if (r32) r32[i] = (float)rn;  // the FP32 V-cycle's input, written in the same pass
    }
}

// p = z + beta p (bodies.rs:365-369)
template <class V, class Z = V>
__global__ void __launch_bounds__(256) k_pupdate(const int64_t* __restrict__ chunk_lo, const int32_t* __restrict__ cpiece,
                                                 const int32_t* __restrict__ done, const double* __restrict__ beta,
                                                 V* __restrict__ p, const Z* __restrict__ z) {
    int c = blockIdx.x;
    int pc = cpiece[c];
    if (done[pc]) return;
    double bt = beta[pc];
    int64_t lo = 6 * chunk_lo[c], hi = 6 * chunk_lo[c + 1];
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) p[i] = (V)((double)z[i] + bt * (double)p[i]);
}

// two dots in one pass: out_a = a.b, out_c = a.a
template <class T, class U = T>
__global__ void __launch_bounds__(256) k_chunk_dot2(const int64_t* __restrict__ chunk_lo, const int32_t* __restrict__ cpiece,
                                                    const int32_t* __restrict__ done, const T* __restrict__ a,
                                                    const U* __restrict__ b, double* __restrict__ pa,
                                                    double* __restrict__ pb) {
    int c = blockIdx.x;
    __shared__ double r1[256], r2[256];
    double s1 = 0.0, s2 = 0.0;
    if (!done || !done[cpiece[c]]) {
        int64_t lo = 6 * chunk_lo[c], hi = 6 * chunk_lo[c + 1];
        for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
            double av = (double)a[i];
            s1 = fma(av, (double)b[i], s1);
            s2 = fma(av, av, s2);
        }
    }
    r1[threadIdx.x] = s1;
    r2[threadIdx.x] = s2;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            r1[threadIdx.x] += r1[threadIdx.x + w];
            r2[threadIdx.x] += r2[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        pa[c] = r1[0];
        pb[c] = r2[0];
    }
}

// per piece: the sums of its chunks' two partials, one warp per piece (each lane a
// strided run of chunks, then a shuffle tree: a fixed order, so the same value every run)
__global__ void k_piece_sum2(int np, const int64_t* __restrict__ piece_chunk, const double* __restrict__ pa,
                             const double* __restrict__ pb, const int32_t* __restrict__ done, double* __restrict__ oa,
                             double* __restrict__ ob) {
    const int p = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (p >= np) return;
    if (done && done[p]) return;
    double s1 = 0.0, s2 = 0.0;
    for (int64_t c = piece_chunk[p] + lane; c < piece_chunk[p + 1]; c += 32) {
        s1 += pa[c];
        if (ob) s2 += pb[c];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        s1 += __shfl_xor_sync(0xffffffffu, s1, off);
        s2 += __shfl_xor_sync(0xffffffffu, s2, off);
    }
    if (lane == 0) {
        oa[p] = s1;
        if (ob) ob[p] = s2;
    }
}

template <class T>
__global__ void k_copy_cast(int64_t n, const double* __restrict__ a, T* __restrict__ b) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) b[i] = (T)a[i];
}




}  // namespace

struct CgState {
    DBuf<double> scal;  // 9 arrays of np
    DBuf<int32_t> flags;
    DBuf<int64_t> iters;
    DBuf<int64_t> replaced;
    DBuf<int32_t> ndone;
    DBuf<uint32_t> loop_count;  // iterations since the device-side loop's launch
    CgScalars s{};
    double* beta = nullptr;
    double* zap = nullptr;  // (z, Ap) for the Polak-Ribiere beta
    int np = 0;
    void init(Context& ctx, int npieces, int32_t* status) {
        np = npieces;
        scal.alloc(9 * (size_t)np, ctx.stream, &ctx.mem);
        scal.zero();
        flags.alloc(np, ctx.stream, &ctx.mem);
        flags.zero();
        iters.alloc(np, ctx.stream, &ctx.mem);
        iters.zero();
        replaced.alloc(np, ctx.stream, &ctx.mem);
        replaced.zero();
        ndone.alloc(1, ctx.stream, &ctx.mem);
        loop_count.alloc(1, ctx.stream, &ctx.mem);
        double* q = scal.get();
        s.bb = q;
        s.goal = q + np;
        s.rz = q + 2 * np;
        s.rr = q + 3 * np;
        s.pap = q + 4 * np;
        s.next = q + 5 * np;
        s.alpha = q + 6 * np;
        beta = q + 7 * np;
        zap = q + 8 * np;
        s.done = flags.get();
        s.iters = iters.get();
        s.status = status;
        s.replaced = replaced.get();
    }
};

static bool timeout_hit(int64_t timeout_ms, std::chrono::steady_clock::time_point t0) {
    return timeout_ms > 0 &&
           std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() > timeout_ms;
}

// reduction scratch sized before a capture (a capture may not allocate)
static void ensure_partial(Context& ctx, const Level& L) {
    if ((int64_t)ctx.partial.size() < 2 * std::max<int64_t>(L.nchunks, 1) + 2048)
        ctx.partial.alloc(2 * (L.nchunks + 1024) + 2048, ctx.stream, &ctx.mem);
}
static void prepare_top(const Level&) {}

// two chunked dots (a.b and a.a) per piece
template <class T, class U = T>
static void dot2(Context& ctx, const Level& L, const int32_t* done, const T* a, const U* b, double* oab, double* oaa) {
    int np = (int)L.pstart.size() - 1;
    if ((int64_t)ctx.partial.size() < 2 * std::max<int64_t>(L.nchunks, 1))
        ctx.partial.alloc(2 * (L.nchunks + 1024), ctx.stream, &ctx.mem);
    double* pa = ctx.partial.get();
    double* pb = pa + std::max<int64_t>(L.nchunks, 1);
    if (L.nchunks > 0) {
        k_chunk_dot2<T, U><<<(unsigned)L.nchunks, 256, 0, ctx.stream>>>(L.chunk_lo.get(), L.chunk_piece.get(), done, a,
                                                                       b, pa, pb);
        SC_LAUNCH_CK();
    }
    k_piece_sum2<<<grid_for((int64_t)np * 32, 128), 128, 0, ctx.stream>>>(np, L.piece_chunk.get(), pa, pb, done, oab,
                                                                         oaa);
    SC_LAUNCH_CK();
}

// CUDA graphs replay the CG iterations unless the environment sets SC_NO_GRAPHS=1 (for
// kernel profilers, which then see every launch on its own) or kernels are being timed.
static bool graphs_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("SC_NO_GRAPHS");
        return !(e && e[0] == '1');
    }();
    return on;
}

// A graph of one conditional WHILE node whose body is what `fill` launches on `st`
// (captured), instantiated; null where the driver offers no conditional nodes (the
// caller then replays a plain graph from the host). The body must end by setting the
// condition through ctx.loop_handle, which this creates.
template <class F>
static cudaGraphExec_t capture_loop(cudaStream_t st, F&& fill, Context& ctx) {
    cudaGraph_t g = nullptr;
    if (cudaGraphCreate(&g, 0) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    cudaGraphExec_t exec = nullptr;
    cudaGraphNodeParams prm = {};
    prm.type = cudaGraphNodeTypeConditional;
    prm.conditional.type = cudaGraphCondTypeWhile;
    prm.conditional.size = 1;
    cudaGraphNode_t node;
    if (cudaGraphConditionalHandleCreate(&ctx.loop_handle, g, 1, cudaGraphCondAssignDefault) == cudaSuccess &&
        (prm.conditional.handle = ctx.loop_handle, cudaGraphAddNode(&node, g, nullptr, 0, &prm) == cudaSuccess) &&
        cudaStreamBeginCaptureToGraph(st, prm.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        cudaGraph_t body = nullptr;
        try {
            fill();
        } catch (...) {
            cudaStreamEndCapture(st, &body);
            cudaGraphDestroy(g);
            throw;
        }
        if (cudaStreamEndCapture(st, &body) == cudaSuccess && cudaGraphInstantiate(&exec, g, 0) != cudaSuccess)
            exec = nullptr;
    }
    cudaGetLastError();
    cudaGraphDestroy(g);
    return exec;
}

// Per piece |K delta|^2 with delta = eps |x| sigma (k_floor_delta): the squared residual
// that rounding x to FP64 leaves.
static void residual_floor(Context& ctx, Batch& b, const double* x, double* ff) {
    Level& L = b.levels[0];
    const int64_t n6 = 6 * L.n;
    DBuf<double> delta, kd;
    delta.alloc(n6, ctx.stream, &ctx.mem);
    kd.alloc(n6, ctx.stream, &ctx.mem);
    k_floor_delta<<<grid_for(n6, 256), 256, 0, ctx.stream>>>(n6, x, delta.get());
    SC_LAUNCH_CK();
    if (L.matrix_free)
        stencil_apply<double>(ctx, b, delta.get(), kd.get(), nullptr, nullptr);
    else
        spmv<double>(ctx, SPMV_Y, L.n, L.rowptr.get(), L.col.get(), L.val.get(), delta.get(), nullptr, kd.get(),
                     nullptr, nullptr, L.piece.get(), nullptr, nullptr, L.nnzb);
    dot2<double>(ctx, L, nullptr, kd.get(), kd.get(), ff, nullptr);
}

// Times a solve may replace the residuals of pieces whose true residual missed the goal.
constexpr int MAX_REPLACEMENTS = 8;

// PCG with per-piece scalars on level 0. V is the vector type of p, r, z, Ap; S the
// type of x; P the precision of the V-cycle preconditioner (with rp, zp its vectors when
// it differs from V). On return x holds the solution of K x = rhs for each piece. Returns
// the kernels one iteration of the device-side loop launches (0 when the loop ran from
// the host), for the launch count.
template <class V, class S, class P = V>
static int64_t pcg(Context& ctx, Batch& b, const V* rhs, S* x, V* r, V* z, V* p, V* ap, double tol, int64_t max_iter,
                CgState& cg, int64_t timeout_ms, std::chrono::steady_clock::time_point t_start,
                const int32_t* start_done = nullptr, P* rp = nullptr, P* zp = nullptr) {
    Level& L = b.levels[0];
    cudaStream_t st = ctx.stream;
    int np = b.npieces;
    int64_t n6 = 6 * L.n;
    constexpr bool same = std::is_same<V, P>::value;
    static_assert(same || std::is_same<P, float>::value, "the preconditioner runs in V or in FP32");
    // The preconditioned residual: z itself, or (FP32 cycle) zp, which the dots and the
    // direction update read directly (no FP64 copy of z is made); rp, the cycle's input,
    // is written by the residual update itself.
    const P* zs = same ? reinterpret_cast<const P*>(z) : zp;
    auto precondition = [&]() {
        if constexpr (same)
            cycle<V>(ctx, b, 0, r, z, cg.s.done);
        else
            cycle<P>(ctx, b, 0, rp, zp, cg.s.done);
    };
    SC_CK(cudaMemsetAsync(x, 0, n6 * sizeof(S), st));
    SC_CK(cudaMemcpyAsync(r, rhs, n6 * sizeof(V), cudaMemcpyDeviceToDevice, st));
    dot2<V>(ctx, L, nullptr, rhs, rhs, cg.s.bb, nullptr);
    k_cg_init<<<grid_for(np, 128), 128, 0, st>>>(np, tol, cg.s, start_done);
    SC_LAUNCH_CK();
    if constexpr (!same) {
        if (L.nchunks > 0) {
            k_cast_chunks<V, P><<<(unsigned)L.nchunks, 256, 0, st>>>(L.chunk_lo.get(), L.chunk_piece.get(),
                                                                      cg.s.done, r, rp);
            SC_LAUNCH_CK();
        }
    }
    precondition();
    if constexpr (same) {
        SC_CK(cudaMemcpyAsync(p, z, n6 * sizeof(V), cudaMemcpyDeviceToDevice, st));
    } else if (L.nchunks > 0) {
        k_cast_chunks<P, V><<<(unsigned)L.nchunks, 256, 0, st>>>(L.chunk_lo.get(), L.chunk_piece.get(), cg.s.done,
                                                                  zp, p);
        SC_LAUNCH_CK();
    }
    dot2<V, P>(ctx, L, cg.s.done, r, zs, cg.s.rz, cg.s.rr);
    // one iteration (bodies.rs:351-371), ending with the next iteration's check
    auto body = [&]() {
        if (L.matrix_free) {
            stencil_apply<V>(ctx, b, p, ap, nullptr, cg.s.done);
        } else {
            ProfScope ps(ctx, fam_of<V>(SC_FAM_SPMV64), spmv_bytes<V>(L, 2));
            spmv<V>(ctx, SPMV_Y, L.n, L.rowptr.get(), L.col.get(), VAL<V>(L), p, nullptr, ap, nullptr, nullptr,
                    L.piece.get(), nullptr, cg.s.done, L.nnzb);
        }
        dot2<V>(ctx, L, cg.s.done, p, ap, cg.s.pap, nullptr);
        k_cg_alpha<<<grid_for(np, 128), 128, 0, st>>>(np, cg.s);
        SC_LAUNCH_CK();
        if (L.nchunks > 0) {
            k_axpy2<V, S><<<(unsigned)L.nchunks, 256, 0, st>>>(L.chunk_lo.get(), L.chunk_piece.get(), cg.s.done,
                                                              cg.s.alpha, x, p, r, ap,
                                                              same ? nullptr : reinterpret_cast<float*>(rp));
            SC_LAUNCH_CK();
        }
        precondition();
        dot2<V, P>(ctx, L, cg.s.done, r, zs, cg.s.next, cg.s.rr);
        if constexpr (same) {
            k_cg_beta<<<grid_for(np, 128), 128, 0, st>>>(np, cg.s, cg.beta);
        } else {
            dot2<V, P>(ctx, L, cg.s.done, ap, zs, cg.zap, nullptr);
            k_cg_beta_flex<<<grid_for(np, 128), 128, 0, st>>>(np, cg.s, cg.zap, cg.beta);
        }
        SC_LAUNCH_CK();
        if (L.nchunks > 0) {
            k_pupdate<V, P><<<(unsigned)L.nchunks, 256, 0, st>>>(L.chunk_lo.get(), L.chunk_piece.get(), cg.s.done,
                                                                cg.beta, p, zs);
            SC_LAUNCH_CK();
        }
        SC_CK(cudaMemsetAsync(cg.ndone.get(), 0, sizeof(int32_t), st));
        k_cg_check<<<grid_for(np, 128), 128, 0, st>>>(np, max_iter, cg.s, cg.ndone.get());
        SC_LAUNCH_CK();
    };
    // Residual replacement: r = b - K x in FP64 for the pieces whose true residual misses
    // the goal (k_cg_verify sets them going again), then z = M r, p = z (a restart from
    // the current x), and the dots of the next check. Returns whether any piece goes on.
    static_assert(std::is_same<V, double>::value && std::is_same<S, double>::value,
                  "the conjugate gradients' vectors and x are FP64");
    const double* rhs64 = rhs;
    int32_t* ndone_h = ctx.pinned_i32();
    DBuf<double> res, rr_true, ff;
    DBuf<int32_t> nrep;
    res.alloc(n6, st, &ctx.mem);
    rr_true.alloc(np, st, &ctx.mem);
    ff.alloc(np, st, &ctx.mem);
    nrep.alloc(1, st, &ctx.mem);
    auto replace_residuals = [&]() -> bool {
        if (L.matrix_free)
            stencil_residual<double>(ctx, b, x, rhs64, res.get(), nullptr, nullptr);
        else
            spmv<double>(ctx, SPMV_RES, L.n, L.rowptr.get(), L.col.get(), L.val.get(), x, rhs64, res.get(), nullptr,
                         nullptr, L.piece.get(), nullptr, nullptr, L.nnzb);
        dot2<double>(ctx, L, nullptr, res.get(), res.get(), rr_true.get(), nullptr);
        residual_floor(ctx, b, x, ff.get());
        SC_CK(cudaMemsetAsync(nrep.get(), 0, sizeof(int32_t), st));
        k_cg_verify<<<grid_for(np, 128), 128, 0, st>>>(np, cg.s, rr_true.get(), ff.get(), nrep.get());
        SC_LAUNCH_CK();
        SC_CK(cudaMemcpyAsync(ndone_h, nrep.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        SC_CK(cudaStreamSynchronize(st));
        if (*ndone_h == 0) return false;
        if (L.nchunks > 0) {
            k_cast_chunks<double, V><<<(unsigned)L.nchunks, 256, 0, st>>>(L.chunk_lo.get(), L.chunk_piece.get(),
                                                                          cg.s.done, res.get(), r);
            SC_LAUNCH_CK();
            if constexpr (!same) {
                k_cast_chunks<V, P><<<(unsigned)L.nchunks, 256, 0, st>>>(L.chunk_lo.get(), L.chunk_piece.get(),
                                                                          cg.s.done, r, rp);
                SC_LAUNCH_CK();
            }
        }
        precondition();
        if (L.nchunks > 0) {
            k_cast_chunks<P, V><<<(unsigned)L.nchunks, 256, 0, st>>>(L.chunk_lo.get(), L.chunk_piece.get(), cg.s.done,
                                                                      zs, p);
            SC_LAUNCH_CK();
        }
        dot2<V, P>(ctx, L, cg.s.done, r, zs, cg.s.rz, cg.s.rr);
        SC_CK(cudaMemsetAsync(cg.ndone.get(), 0, sizeof(int32_t), st));
        k_cg_check<<<grid_for(np, 128), 128, 0, st>>>(np, max_iter, cg.s, cg.ndone.get());
        SC_LAUNCH_CK();
        return true;
    };
    cudaGraphExec_t exec = nullptr, loop = nullptr;
    int64_t per_iteration = 0, graph_kernels = 0;
    // iterations one launch of the device-side loop runs at most between looks at the
    // done count (and at the time limit)
    const uint32_t chunk = 32;
    try {
        // Replaying a captured iteration saves ~50 launches an iteration; timing
        // individual kernels (profiling) launches them one by one instead.
        bool use_graph = ctx.prof.mask == 0 && graphs_enabled();
        if (use_graph) {
            ensure_partial(ctx, L);
            for (auto& lv : b.levels) prepare_top(lv);
            // first choice: the iterations loop on the device, a graph whose conditional
            // WHILE node replays the iteration until every piece is done (or `chunk` ran)
            const int64_t l0 = g_launches.load();
            loop = capture_loop(st, [&] {
                body();
                k_loop_more<<<1, 1, 0, st>>>(ctx.loop_handle, cg.ndone.get(), np, cg.loop_count.get(), chunk);
                SC_LAUNCH_CK();
            }, ctx);
            per_iteration = g_launches.load() - l0;
            g_launches.fetch_sub(per_iteration);  // counted per iteration run, below
            if (!loop) {
                per_iteration = 0;
                cudaGraph_t graph = nullptr;
                SC_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                try {
                    body();
                } catch (...) {
                    cudaStreamEndCapture(st, &graph);
                    if (graph) cudaGraphDestroy(graph);
                    throw;
                }
                SC_CK(cudaStreamEndCapture(st, &graph));
                cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
                cudaGraphDestroy(graph);
                SC_CK(e);
                graph_kernels = g_launches.load() - l0;
            }
        }
        SC_CK(cudaMemsetAsync(cg.ndone.get(), 0, sizeof(int32_t), st));
        k_cg_check<<<grid_for(np, 128), 128, 0, st>>>(np, max_iter, cg.s, cg.ndone.get());
        SC_LAUNCH_CK();
        // iterations run between looks at the done count (finished pieces' kernels return at once)
        const int per_look = 4;
        int replacements = 0;
        for (;;) {
            SC_CK(cudaMemcpyAsync(ndone_h, cg.ndone.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            SC_CK(cudaStreamSynchronize(st));
            if (*ndone_h >= np) {
                // every piece stopped: those whose true residual misses the goal take it as
                // their residual and go on (residual replacement), a bounded number of times
                if (replacements++ >= MAX_REPLACEMENTS || !replace_residuals()) break;
                continue;
            }
            if (timeout_ms > 0 &&
                std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count() >
                    timeout_ms)
                throw Error(SC_TIMEOUT, "solve ran past its time limit");
            if (loop) {
                SC_CK(cudaMemsetAsync(cg.loop_count.get(), 0, sizeof(uint32_t), st));
                SC_CK(cudaGraphLaunch(loop, st));
                continue;
            }
            for (int g = 0; g < per_look; g++) {
                if (exec) {
                    SC_CK(cudaGraphLaunch(exec, st));
                    g_launches.fetch_add(graph_kernels);
                } else {
                    body();
                }
            }
        }
    } catch (...) {
        if (exec) cudaGraphExecDestroy(exec);
        if (loop) cudaGraphExecDestroy(loop);
        throw;
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (loop) cudaGraphExecDestroy(loop);
    return per_iteration;
}

// the device-side loop ran one iteration per iteration of its slowest piece (and one
// more whose kernels returned at once after the last piece finished)
static void count_loop_launches(int64_t per_iteration, const std::vector<int64_t>& iters) {
    if (per_iteration <= 0) return;
    int64_t most = 0;
    for (int64_t i : iters) most = std::max(most, i);
    g_launches.fetch_add(per_iteration * (most + 1));
}

// |b - K x| / |b| per piece, in FP64, and the floor of that ratio rounding x to FP64
// leaves (residual_floor)
static void true_residual(Context& ctx, Batch& b, const double* x, SolveStats& st) {
    Level& L = b.levels[0];
    int np = b.npieces;
    DBuf<double> res, nr;
    res.alloc(6 * L.n, ctx.stream, &ctx.mem);
    nr.alloc(3 * np, ctx.stream, &ctx.mem);
    if (L.matrix_free)
        stencil_residual<double>(ctx, b, x, b.loads.get(), res.get(), nullptr, nullptr);
    else
        spmv<double>(ctx, SPMV_RES, L.n, L.rowptr.get(), L.col.get(), L.val.get(), x, b.loads.get(), res.get(),
                     nullptr, nullptr, L.piece.get(), nullptr, nullptr, L.nnzb);
    dot2<double>(ctx, L, nullptr, res.get(), res.get(), nr.get(), nullptr);
    dot2<double>(ctx, L, nullptr, b.loads.get(), b.loads.get(), nr.get() + np, nullptr);
    residual_floor(ctx, b, x, nr.get() + 2 * np);
    std::vector<double> h = nr.to_host();
    st.residual.resize(np);
    st.floor.resize(np);
    for (int p = 0; p < np; p++) {
        st.residual[p] = h[np + p] > 0 ? std::sqrt(h[p] / h[np + p]) : 0.0;
        st.floor[p] = h[np + p] > 0 ? std::sqrt(h[2 * np + p] / h[np + p]) : 0.0;
    }
}

void pcg_fp64(Context& ctx, Batch& b, const sc_options& opt, DBuf<double>& x, SolveStats& stats) {
    auto t0 = std::chrono::steady_clock::now();
    Level& L = b.levels[0];
    int64_t n6 = 6 * L.n;
    alloc_cycle<double>(ctx, b);
    x.alloc(n6, ctx.stream, &ctx.mem);
    DBuf<double> r, z, p, ap;
    r.alloc(n6, ctx.stream, &ctx.mem);
    z.alloc(n6, ctx.stream, &ctx.mem);
    p.alloc(n6, ctx.stream, &ctx.mem);
    ap.alloc(n6, ctx.stream, &ctx.mem);
    CgState cg;
    cg.init(ctx, b.npieces, b.status_d.get());
    int64_t per_it = pcg<double, double>(ctx, b, b.loads.get(), x.get(), r.get(), z.get(), p.get(), ap.get(), opt.tol,
                                         opt.max_iter, cg, opt.timeout_ms, t0);
    std::vector<int64_t> it(b.npieces);
    cg.iters.download(it.data(), b.npieces);
    SC_CK(cudaStreamSynchronize(ctx.stream));
    count_loop_launches(per_it, it);
    stats.iterations = it;
    stats.refinements = cg.replaced.to_host();
    true_residual(ctx, b, x.get(), stats);
}

// ---- mixed precision --------------------------------------------------------------
namespace {

// end of an FP32 iteration: a piece whose iterated residual says converged (or that hit
// the cap) stops as a candidate until the next FP64 check
__global__ void k_mixed_check(int np, int64_t max_iter, CgScalars s, int32_t* __restrict__ cand,
                              int32_t* __restrict__ ndone) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    if (!s.done[p]) {
        double nr = sqrt(s.rr[p]);
        if (nr <= s.goal[p] || s.iters[p] >= max_iter) {
            s.done[p] = 1;
            cand[p] = 1;
        } else if (!(nr == nr) || !(s.rz[p] == s.rz[p])) {
            s.done[p] = 1;
            atomicMax(s.status + p, (int)SC_BREAKDOWN);
        }
    }
    if (s.done[p]) atomicAdd(ndone, 1);
}

// which pieces take the FP64 update: all but those finished for good
__global__ void k_mixed_mask(int np, const int32_t* __restrict__ done, const int32_t* __restrict__ cand,
                             int32_t* __restrict__ skip) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < np) skip[p] = (done[p] && !cand[p]) ? 1 : 0;
}

// x64 += x32; x32 = 0 (one block per chunk)
__global__ void __launch_bounds__(256) k_fold_x(const int64_t* __restrict__ chunk_lo, const int32_t* __restrict__ cpiece,
                                                const int32_t* __restrict__ skip, double* __restrict__ x64,
                                                float* __restrict__ x32) {
    int c = blockIdx.x;
    if (skip && skip[cpiece[c]]) return;
    int64_t lo = 6 * chunk_lo[c], hi = 6 * chunk_lo[c + 1];
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        x64[i] += (double)x32[i];
        x32[i] = 0.0f;
    }
}

__global__ void __launch_bounds__(256) k_to32(const int64_t* __restrict__ chunk_lo, const int32_t* __restrict__ cpiece,
                                              const int32_t* __restrict__ skip, const double* __restrict__ a,
                                              float* __restrict__ b) {
    int c = blockIdx.x;
    if (skip && skip[cpiece[c]]) return;
    int64_t lo = 6 * chunk_lo[c], hi = 6 * chunk_lo[c + 1];
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) b[i] = (float)a[i];
}

// the FP64 verdict on the true residual b - K x64
__global__ void k_mixed_true(int np, int64_t max_iter, CgScalars s, const int32_t* __restrict__ skip,
                             const double* __restrict__ rr64, int32_t* __restrict__ cand, int32_t* __restrict__ nfinal,
                             int64_t* __restrict__ updates) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    if (!skip[p]) {
        updates[p] += 1;
        double nr = sqrt(rr64[p]);
        cand[p] = 0;
        if (nr <= s.goal[p]) {
            s.done[p] = 1;
        } else if (s.iters[p] >= max_iter) {
            s.done[p] = 1;
            atomicMax(s.status + p, (int)SC_MAXITER);
        } else if (!(nr == nr)) {
            s.done[p] = 1;
            atomicMax(s.status + p, (int)SC_BREAKDOWN);
        } else {
            s.done[p] = 0;
        }
    }
    if (s.done[p] && !cand[p]) atomicAdd(nfinal, 1);
}

}  // namespace

// Mixed precision: one preconditioned CG whose vectors, operator (the stencil), smoother,
// transfers and coarse operators are FP32 with FP32 accumulation, and whose dot products
// and scalars (alpha, beta) are FP64; the solution is folded into an FP64 x every
// `period` iterations and whenever the FP32 residual claims convergence, and there the
// true residual b - K x is recomputed by the FP64 stencil and replaces the FP32 one
// (reliable updates): the FP64 iterative refinement. The dense top solve is FP64.
static void float_operators(Context& ctx, Batch& b) {
    for (size_t l = 0; l < b.levels.size(); l++) {
        Level& L = b.levels[l];
        if (L.val.size()) to_float(ctx, L.val, L.val32);
        if (L.inv.size()) to_float(ctx, L.inv, L.inv32);
        if (L.pval.size()) to_float(ctx, L.pval, L.pval32);
        if (L.ptval.size()) to_float(ctx, L.ptval, L.ptval32);
        if (L.mf_r.size()) to_float(ctx, L.mf_r, L.mf_r32);
    }
}

// FP64 conjugate gradients (vectors, operator, dots and scalars in FP64) preconditioned
// by the V-cycle in FP32 (stencil, smoother, transfers and coarse operators with FP32
// accumulation; the dense top solve FP64). The FP32 cycle is not exactly symmetric, so
// beta takes the Polak-Ribiere form.
void pcg_fp32_cycle(Context& ctx, Batch& b, const sc_options& opt, DBuf<double>& x, SolveStats& stats) {
    auto t0 = std::chrono::steady_clock::now();
    float_operators(ctx, b);
    alloc_cycle<float>(ctx, b);
    Level& L = b.levels[0];
    int64_t n6 = 6 * L.n;
    x.alloc(n6, ctx.stream, &ctx.mem);
    DBuf<double> r, p, ap;  // the preconditioned residual stays FP32 (z32)
    for (auto* v : {&r, &p, &ap}) v->alloc(n6, ctx.stream, &ctx.mem);
    DBuf<float> r32, z32;
    r32.alloc(n6, ctx.stream, &ctx.mem);
    z32.alloc(n6, ctx.stream, &ctx.mem);
    CgState cg;
    cg.init(ctx, b.npieces, b.status_d.get());
    int64_t per_it = pcg<double, double, float>(ctx, b, b.loads.get(), x.get(), r.get(), nullptr, p.get(), ap.get(),
                                                opt.tol, opt.max_iter, cg, opt.timeout_ms, t0, nullptr, r32.get(),
                                                z32.get());
    std::vector<int64_t> it(b.npieces);
    cg.iters.download(it.data(), b.npieces);
    SC_CK(cudaStreamSynchronize(ctx.stream));
    count_loop_launches(per_it, it);
    stats.iterations = it;
    stats.refinements = cg.replaced.to_host();
    true_residual(ctx, b, x.get(), stats);
}

void pcg_mixed(Context& ctx, Batch& b, const sc_options& opt, DBuf<double>& x, SolveStats& stats) {
    auto t0 = std::chrono::steady_clock::now();
    cudaStream_t st = ctx.stream;
    int np = b.npieces;
    float_operators(ctx, b);
    alloc_cycle<float>(ctx, b);
    Level& L = b.levels[0];
    int64_t n6 = 6 * L.n;
    x.alloc(n6, st, &ctx.mem);
    x.zero();
    DBuf<double> r64;
    r64.alloc(n6, st, &ctx.mem);
    DBuf<float> x32, r, z, p, ap;
    for (auto* v : {&x32, &r, &z, &p, &ap}) v->alloc(n6, st, &ctx.mem);
    x32.zero();
    DBuf<int32_t> cand, skip, counts;
    cand.alloc(np, st, &ctx.mem);
    cand.zero();
    skip.alloc(np, st, &ctx.mem);
    skip.zero();
    counts.alloc(2, st, &ctx.mem);
    DBuf<double> rr64;
    rr64.alloc(np, st, &ctx.mem);
    DBuf<int64_t> updates;
    updates.alloc(np, st, &ctx.mem);
    updates.zero();
    CgState cg;
    cg.init(ctx, np, b.status_d.get());
    const int64_t max_iter = opt.max_iter;
    auto chunks = [&](auto kernel, auto... args) {
        if (L.nchunks > 0) {
            kernel<<<(unsigned)L.nchunks, 256, 0, st>>>(L.chunk_lo.get(), L.chunk_piece.get(), args...);
            SC_LAUNCH_CK();
        }
    };
    // start: r = b in FP32, z = M r, p = z
    dot2<double>(ctx, L, nullptr, b.loads.get(), b.loads.get(), cg.s.bb, nullptr);
    k_cg_init<<<grid_for(np, 128), 128, 0, st>>>(np, opt.tol, cg.s, nullptr);
    SC_LAUNCH_CK();
    chunks(k_to32, (const int32_t*)nullptr, (const double*)b.loads.get(), r.get());
    cycle<float>(ctx, b, 0, r.get(), z.get(), cg.s.done);
    SC_CK(cudaMemcpyAsync(p.get(), z.get(), n6 * sizeof(float), cudaMemcpyDeviceToDevice, st));
    dot2<float>(ctx, L, cg.s.done, r.get(), z.get(), cg.s.rz, cg.s.rr);
    // the first half of an iteration: Ap, alpha, x32 and r32
    auto first = [&]() {
        if (L.matrix_free)
            stencil_apply<float>(ctx, b, p.get(), ap.get(), nullptr, cg.s.done);
        else
            spmv<float>(ctx, SPMV_Y, L.n, L.rowptr.get(), L.col.get(), L.val32.get(), p.get(), nullptr, ap.get(),
                        nullptr, nullptr, L.piece.get(), nullptr, cg.s.done, L.nnzb);
        dot2<float>(ctx, L, cg.s.done, p.get(), ap.get(), cg.s.pap, nullptr);
        k_cg_alpha<<<grid_for(np, 128), 128, 0, st>>>(np, cg.s);
        SC_LAUNCH_CK();
        chunks(k_axpy2<float, float>, (const int32_t*)cg.s.done, (const double*)cg.s.alpha, x32.get(),
               (const float*)p.get(), r.get(), (const float*)ap.get(), (float*)nullptr);
    };
    // the FP64 update: fold x32 into x, r = b - K x in FP64, its verdict
    auto update = [&]() {
        k_mixed_mask<<<grid_for(np, 128), 128, 0, st>>>(np, cg.s.done, cand.get(), skip.get());
        SC_LAUNCH_CK();
        chunks(k_fold_x, (const int32_t*)skip.get(), x.get(), x32.get());
        if (L.matrix_free)
            stencil_residual<double>(ctx, b, x.get(), b.loads.get(), r64.get(), nullptr, skip.get());
        else
            spmv<double>(ctx, SPMV_RES, L.n, L.rowptr.get(), L.col.get(), L.val.get(), x.get(), b.loads.get(),
                         r64.get(), nullptr, nullptr, L.piece.get(), nullptr, skip.get(), L.nnzb);
        dot2<double>(ctx, L, skip.get(), r64.get(), r64.get(), rr64.get(), nullptr);
        chunks(k_to32, (const int32_t*)skip.get(), (const double*)r64.get(), r.get());
        SC_CK(cudaMemsetAsync(counts.get(), 0, 2 * sizeof(int32_t), st));
        k_mixed_true<<<grid_for(np, 128), 128, 0, st>>>(np, max_iter, cg.s, skip.get(), rr64.get(), cand.get(),
                                                        counts.get() + 1, updates.get());
        SC_LAUNCH_CK();
    };
    // the second half: z = M r, beta, p; then the FP32 verdict
    auto second = [&]() {
        cycle<float>(ctx, b, 0, r.get(), z.get(), cg.s.done);
        dot2<float>(ctx, L, cg.s.done, r.get(), z.get(), cg.s.next, cg.s.rr);
        k_cg_beta<<<grid_for(np, 128), 128, 0, st>>>(np, cg.s, cg.beta);
        SC_LAUNCH_CK();
        chunks(k_pupdate<float>, (const int32_t*)cg.s.done, (const double*)cg.beta, p.get(), (const float*)z.get());
        SC_CK(cudaMemsetAsync(counts.get(), 0, sizeof(int32_t), st));
        k_mixed_check<<<grid_for(np, 128), 128, 0, st>>>(np, max_iter, cg.s, cand.get(), counts.get());
        SC_LAUNCH_CK();
    };
    int32_t* counts_h = ctx.pinned_i32();
    cudaGraphExec_t plain = nullptr, upd = nullptr;
    int64_t plain_kernels = 0, upd_kernels = 0;
    auto capture = [&](auto fn, int64_t& kernels) {
        const int64_t l0 = g_launches.load();
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        SC_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        try {
            fn();
        } catch (...) {
            cudaStreamEndCapture(st, &graph);
            if (graph) cudaGraphDestroy(graph);
            throw;
        }
        SC_CK(cudaStreamEndCapture(st, &graph));
        cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        SC_CK(e);
        kernels = g_launches.load() - l0;
        g_launches.fetch_sub(kernels);  // counted per replay
        return exec;
    };
    try {
        bool use_graph = ctx.prof.mask == 0 && graphs_enabled();
        auto it_plain = [&]() { first(); second(); };
        auto it_upd = [&]() { first(); update(); second(); };
        if (use_graph) {
            ensure_partial(ctx, L);
            plain = capture(it_plain, plain_kernels);
            upd = capture(it_upd, upd_kernels);
        }
        // the starting verdict: b = 0 finishes at once
        SC_CK(cudaMemsetAsync(counts.get(), 0, 2 * sizeof(int32_t), st));
        k_mixed_check<<<grid_for(np, 128), 128, 0, st>>>(np, max_iter, cg.s, cand.get(), counts.get());
        SC_LAUNCH_CK();
        const int period = 8;
        int since = 0;
        bool all_stopped = false;
        for (;;) {
            if (timeout_hit(opt.timeout_ms, t0)) throw Error(SC_TIMEOUT, "solve ran past its time limit");
            bool do_update = all_stopped || since >= period - 1;
            if (do_update) {
                if (all_stopped) {
                    update();  // every piece stopped: only the FP64 verdict is left
                    second();
                } else if (upd) {
                    SC_CK(cudaGraphLaunch(upd, st));
                    g_launches.fetch_add(upd_kernels);
                } else {
                    it_upd();
                }
                since = 0;
            } else {
                if (plain) {
                    SC_CK(cudaGraphLaunch(plain, st));
                    g_launches.fetch_add(plain_kernels);
                } else {
                    it_plain();
                }
                since++;
            }
            SC_CK(cudaMemcpyAsync(counts_h, counts.get(), 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            SC_CK(cudaStreamSynchronize(st));
            if (do_update && counts_h[1] >= np) break;
            all_stopped = counts_h[0] >= np;
        }
        // pieces stopped by a breakdown keep what they reached
        chunks(k_fold_x, (const int32_t*)nullptr, x.get(), x32.get());
    } catch (...) {
        if (plain) cudaGraphExecDestroy(plain);
        if (upd) cudaGraphExecDestroy(upd);
        throw;
    }
    if (plain) cudaGraphExecDestroy(plain);
    if (upd) cudaGraphExecDestroy(upd);
    std::vector<int64_t> it(np), up(np);
    cg.iters.download(it.data(), np);
    updates.download(up.data(), np);
    SC_CK(cudaStreamSynchronize(st));
    stats.iterations = it;
    stats.refinements = up;
    true_residual(ctx, b, x.get(), stats);
}

}  // namespace sc
