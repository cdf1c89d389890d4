// Solver::new of the engine's solver (mechanics/src/solve.rs:241-296, 320-347, 361-386) on
// the device: the nodes' block inverses and smoother step, then level after level the
// rigid aggregates of the parts joined within each octree cell a level up, their centres,
// offsets and Galerkin blocks T(r)' M T(s), block inverses by Cholesky with dropped pivots
// after the turn regularisation, the smoother step by ten power steps, and the direct top.
//
// The levels are the reference's bit for bit (the same parts, blocks and steps). This file
// is compiled without fused multiply-adds (-fmad=false), so every product and sum is
// rounded apart as the Rust code rounds it, and every sum runs in the reference's order:
//   - the union-find's roots (solve.rs:245-250: the greater root hangs under the lesser)
//     are each component's least part, which min-label propagation finds; ids by first
//     appearance are then the roots' ranks;
//   - an aggregate's centre sums its members in order, one thread an aggregate;
//   - its diagonal block adds its members' lifted blocks in member order, then its inner
//     pairs' (m + m') in pair order; each pair across two aggregates (a < c) adds into
//     block (a, c) in pair order (a stable sort of the pairs by (a, c), one thread a
//     group), blocks in (a, c) order -- the order mech.cu's host copy adds them in;
//   - a power step's product adds, row by row, the diagonal block's terms, then each pair
//     touching the row in pair order (a stable sort of the pairs' ends by part); the
//     norms, sums over every value in order, are taken on the host from a copy.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>

#include "mech.cuh"

namespace sc {

namespace {

constexpr int LT = 128;

int end_bit_for(int64_t v) {
    int b = 1;
    while (b < 63 && (int64_t(1) << b) <= v) b++;
    return b;
}

template <class T>
void scan_exclusive(Context& ctx, const T* in, T* out, int64_t n) {
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, n, ctx.stream);
    cub::DeviceScan::ExclusiveSum(ctx.cub_scratch(tb), tb, in, out, n, ctx.stream);
}

// a stable sort of (key, value) pairs by key's low end_bit bits
template <class K, class V>
void sort_pairs(Context& ctx, const K* kin, K* kout, const V* vin, V* vout, int64_t n, int end_bit) {
    if (n <= 0) return;
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, kin, kout, vin, vout, n, 0, end_bit, ctx.stream);
    cub::DeviceRadixSort::SortPairs(ctx.cub_scratch(tb), tb, kin, kout, vin, vout, n, 0, end_bit, ctx.stream);
}

template <class T>
T read_one(Context& ctx, const T* p) {
    T v{};
    SC_CK(cudaMemcpyAsync(&v, p, sizeof(T), cudaMemcpyDeviceToHost, ctx.stream));
    SC_CK(cudaStreamSynchronize(ctx.stream));
    return v;
}

// ---- dense blocks, each operation as the host's copy orders it -------------------------
// The inverse operator of an N x N block by Cholesky, pivots below 1e-12 of the largest
// dropped (solve.rs:123-186): a is destroyed; out[c * N + r] = (A^-1 e_c)[r].
template <int N>
__device__ void chol_inverse_d(double* a, double* out) {
    double largest = 0.0;
    for (int i = 0; i < N; i++) largest = fmax(largest, a[i * N + i]);
    bool dropped[N];
    for (int j = 0; j < N; j++) {
        double d = a[j * N + j];
        for (int k = 0; k < j; k++) d -= a[j * N + k] * a[j * N + k];
        if (d <= largest * 1e-12) {
            dropped[j] = true;
            for (int i = j; i < N; i++) a[i * N + j] = 0.0;
            continue;
        }
        dropped[j] = false;
        d = sqrt(d);
        a[j * N + j] = d;
        for (int i = j + 1; i < N; i++) {
            double s = a[i * N + j];
            for (int k = 0; k < j; k++) s -= a[i * N + k] * a[j * N + k];
            a[i * N + j] = s / d;
        }
    }
    for (int c = 0; c < N; c++) {
        double b[N];
        for (int i = 0; i < N; i++) b[i] = i == c ? 1.0 : 0.0;
        for (int i = 0; i < N; i++) {
            if (dropped[i]) {
                b[i] = 0.0;
                continue;
            }
            double s = 0.0;
            for (int k = 0; k < i; k++) s += a[i * N + k] * b[k];
            b[i] = (b[i] - s) / a[i * N + i];
        }
        for (int i = N - 1; i >= 0; i--) {
            if (dropped[i]) {
                b[i] = 0.0;
                continue;
            }
            double s = 0.0;
            for (int k = i + 1; k < N; k++) s += a[k * N + i] * b[k];
            b[i] = (b[i] - s) / a[i * N + i];
        }
        for (int r = 0; r < N; r++) out[c * N + r] = b[r];
    }
}

// a B x B block (row-major) embedded as the 6 x 6 block of a part (solve.rs:97-103)
template <int B>
__device__ void embed6(const double* m, double* out) {
    for (int i = 0; i < 36; i++) out[i] = 0.0;
    for (int r = 0; r < B; r++)
        for (int c = 0; c < B; c++) out[6 * r + c] = m[B * r + c];
}

// T(r)' M T(s) (solve.rs:77-94), M 6 x 6
__device__ void lift6_d(const double* m, const double* r, const double* s, double* out) {
    const double xr[9] = {0.0, r[2], -r[1], -r[2], 0.0, r[0], r[1], -r[0], 0.0};
    const double xs[9] = {0.0, s[2], -s[1], -s[2], 0.0, s[0], s[1], -s[0], 0.0};
    double t[36];
    for (int i = 0; i < 36; i++) t[i] = m[i];
    for (int row = 0; row < 6; row++)
        for (int c = 0; c < 3; c++) {
            double acc = 0.0;
            for (int k = 0; k < 3; k++) acc += m[6 * row + k] * xs[3 * k + c];
            t[6 * row + 3 + c] += acc;
        }
    for (int i = 0; i < 36; i++) out[i] = t[i];
    for (int r3 = 0; r3 < 3; r3++)
        for (int col = 0; col < 6; col++) {
            double acc = 0.0;
            for (int k = 0; k < 3; k++) acc += xr[3 * k + r3] * t[6 * k + col];
            out[6 * (3 + r3) + col] += acc;
        }
}

// ---- kernels ----------------------------------------------------------------------------
// each part's block inverse; REG: the turn regularisation first (solve.rs:264-269)
template <int N, bool REG>
__global__ void k_block_inverses(int64_t n, const double* __restrict__ blocks, double size, double* __restrict__ inv) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= n) return;
    double a[N * N];
    for (int i = 0; i < N * N; i++) a[i] = blocks[(int64_t)N * N * p + i];
    if (REG) {
        const double t = (a[0] + a[N + 1] + a[2 * N + 2]) / 3.0;
        for (int k = 3; k < 6; k++) a[k * N + k] += 1e-6 * t * size * size;
    }
    chol_inverse_d<N>(a, inv + (int64_t)N * N * p);
}

// the pairs' ends as (part, 2 q + side), for a stable sort by part
__global__ void k_pair_ends(int64_t np, const uint32_t* __restrict__ pi, const uint32_t* __restrict__ pj,
                            uint32_t* __restrict__ key, uint64_t* __restrict__ val, int64_t* __restrict__ deg) {
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= np) return;
    key[2 * q] = pi[q];
    key[2 * q + 1] = pj[q];
    val[2 * q] = 2 * (uint64_t)q;
    val[2 * q + 1] = 2 * (uint64_t)q + 1;
    atomicAdd(reinterpret_cast<unsigned long long*>(deg + pi[q]), 1ull);
    atomicAdd(reinterpret_cast<unsigned long long*>(deg + pj[q]), 1ull);
}

// y = S x over B-vectors (solve.rs:63-73, 306-317): the diagonal block's terms, then each
// pair touching the row in pair order
template <int B>
__global__ void k_incidence_apply(int64_t n, const int64_t* __restrict__ ptr, const uint64_t* __restrict__ ent,
                                  const double* __restrict__ diag, const double* __restrict__ pm,
                                  const uint32_t* __restrict__ pi, const uint32_t* __restrict__ pj,
                                  const double* __restrict__ x, double* __restrict__ y) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double yv[B];
    for (int r = 0; r < B; r++) {
        double acc = 0.0;
        for (int c = 0; c < B; c++) acc += diag[(int64_t)B * B * i + B * r + c] * x[(int64_t)B * i + c];
        yv[r] = acc;
    }
    for (int64_t t = ptr[i]; t < ptr[i + 1]; t++) {
        const uint64_t e = ent[t];
        const int64_t q = (int64_t)(e >> 1);
        const double* m = pm + (int64_t)B * B * q;
        if ((e & 1) == 0) {
            const double* xj = x + (int64_t)B * pj[q];
            for (int r = 0; r < B; r++) {
                double a = 0.0;
                for (int c = 0; c < B; c++) a += m[B * r + c] * xj[c];
                yv[r] += a;
            }
        } else {
            const double* xj = x + (int64_t)B * pi[q];
            for (int r = 0; r < B; r++) {
                double a = 0.0;
                for (int c = 0; c < B; c++) a += m[B * c + r] * xj[c];
                yv[r] += a;
            }
        }
    }
    for (int r = 0; r < B; r++) y[(int64_t)B * i + r] = yv[r];
}

// y = inv x, part by part
template <int B>
__global__ void k_block_over(int64_t n, const double* __restrict__ inv, const double* __restrict__ x,
                             double* __restrict__ y) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= n) return;
    for (int r = 0; r < B; r++) {
        double acc = 0.0;
        for (int c = 0; c < B; c++) acc += inv[(int64_t)B * B * p + B * r + c] * x[(int64_t)B * p + c];
        y[(int64_t)B * p + r] = acc;
    }
}

__device__ __forceinline__ int64_t half_key(int64_t v) { return v >= 0 ? v / 2 : -((-v + 1) / 2); }  // div_euclid(2)

__global__ void k_parent_keys(int64_t n, const int64_t* __restrict__ keys, int64_t* __restrict__ pk) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= 3 * n) return;
    pk[i] = half_key(keys[i]);
}

__global__ void k_iota(int64_t n, int32_t* __restrict__ v) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) v[i] = (int32_t)i;
}

// the pairs joined (both ends in one octree cell a level up) hang the greater label's
// root under the lesser
__global__ void k_hook(int64_t np, const uint32_t* __restrict__ pi, const uint32_t* __restrict__ pj,
                       const int64_t* __restrict__ pk, int32_t* lab, int32_t* __restrict__ changed) {
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= np) return;
    const int64_t a = pi[q], b = pj[q];
    if (pk[3 * a] != pk[3 * b] || pk[3 * a + 1] != pk[3 * b + 1] || pk[3 * a + 2] != pk[3 * b + 2]) return;
    const int32_t ra = lab[a], rb = lab[b];
    if (ra == rb) return;
    atomicMin(lab + max(ra, rb), min(ra, rb));
    *changed = 1;
}

// every label to its root (labels only ever fall, so the chase ends)
__global__ void k_compress(int64_t n, int32_t* lab) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int32_t l = lab[i];
    while (true) {
        const int32_t u = *((volatile int32_t*)lab + l);
        if (u == l) break;
        l = u;
    }
    lab[i] = l;
}

__global__ void k_root_flags(int64_t n, const int32_t* __restrict__ lab, int32_t* __restrict__ flag) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) flag[i] = lab[i] == (int32_t)i ? 1 : 0;
}

__global__ void k_part_of(int64_t n, const int32_t* __restrict__ lab, const int32_t* __restrict__ id,
                          int32_t* __restrict__ of, int64_t* __restrict__ cnt) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t a = id[lab[i]];
    of[i] = a;
    atomicAdd(reinterpret_cast<unsigned long long*>(cnt + a), 1ull);
}

// an aggregate's centre: its members' positions summed in order, times 1 / count
// (solve.rs:251-253), and its octree key a level up
__global__ void k_centres(int64_t nc, const int64_t* __restrict__ mptr, const int32_t* __restrict__ mem,
                          const double* __restrict__ at, const int64_t* __restrict__ pk, double* __restrict__ cat,
                          int64_t* __restrict__ ckeys) {
    const int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (a >= nc) return;
    double s[3] = {0.0, 0.0, 0.0}, count = 0.0;
    int64_t last = 0;
    for (int64_t t = mptr[a]; t < mptr[a + 1]; t++) {
        const int64_t i = mem[t];
        for (int k = 0; k < 3; k++) s[k] = s[k] + at[3 * i + k];
        count += 1.0;
        last = i;
    }
    for (int k = 0; k < 3; k++) {
        cat[3 * a + k] = s[k] * (1.0 / count);
        ckeys[3 * a + k] = pk[3 * last + k];
    }
}

// each finer part's offset from its aggregate's centre
__global__ void k_offsets(int64_t nf, const int32_t* __restrict__ of, const double* __restrict__ at,
                          const double* __restrict__ cat, double* __restrict__ r) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nf) return;
    for (int k = 0; k < 3; k++) r[3 * i + k] = at[3 * i + k] - cat[3 * (int64_t)of[i] + k];
}

// each pair's (lesser, greater) aggregate pair as the key of a stable sort
__global__ void k_pair_groups(int64_t np, const uint32_t* __restrict__ pi, const uint32_t* __restrict__ pj,
                              const int32_t* __restrict__ of, uint64_t* __restrict__ key, uint32_t* __restrict__ q) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= np) return;
    const uint32_t a = (uint32_t)of[pi[e]], b = (uint32_t)of[pj[e]];
    key[e] = ((uint64_t)min(a, b) << 32) | max(a, b);
    q[e] = (uint32_t)e;
}

__global__ void k_group_flags(int64_t np, const uint64_t* __restrict__ skey, int64_t* __restrict__ flag) {
    const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= np) return;
    flag[g] = (g == 0 || skey[g] != skey[g - 1]) ? 1 : 0;
}

__global__ void k_group_starts(int64_t np, const int64_t* __restrict__ flag, const int64_t* __restrict__ gid,
                               const uint64_t* __restrict__ skey, int64_t* __restrict__ gstart,
                               int64_t* __restrict__ cross) {
    const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= np || !flag[g]) return;
    gstart[gid[g]] = g;
    cross[gid[g]] = (skey[g] >> 32) != (skey[g] & 0xffffffffull) ? 1 : 0;
}

// each aggregate's diagonal block: its members' lifted blocks, in member order
template <int B>
__global__ void k_member_blocks(int64_t nc, const int64_t* __restrict__ mptr, const int32_t* __restrict__ mem,
                                const double* __restrict__ fdiag, const double* __restrict__ r,
                                double* __restrict__ cdiag) {
    const int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (a >= nc) return;
    double d[36];
    for (int k = 0; k < 36; k++) d[k] = 0.0;
    for (int64_t t = mptr[a]; t < mptr[a + 1]; t++) {
        const int64_t i = mem[t];
        double m[36], l[36];
        embed6<B>(fdiag + (int64_t)B * B * i, m);
        lift6_d(m, r + 3 * i, r + 3 * i, l);
        for (int k = 0; k < 36; k++) d[k] += l[k];
    }
    for (int k = 0; k < 36; k++) cdiag[36 * a + k] = d[k];
}

// A group of pairs with one (a, c) key: inside an aggregate (a = c) each pair's m and m'
// added to its diagonal block in pair order; across two, their sum (each as from a to c)
// is coarse pair number cross[group]
template <int B>
__global__ void k_group_blocks(int64_t ng, const int64_t* __restrict__ gstart, const uint64_t* __restrict__ skey,
                               const uint32_t* __restrict__ sq, const uint32_t* __restrict__ pi,
                               const uint32_t* __restrict__ pj, const double* __restrict__ pm,
                               const int32_t* __restrict__ of, const double* __restrict__ r,
                               const int64_t* __restrict__ cross, double* __restrict__ cdiag,
                               uint32_t* __restrict__ cpi, uint32_t* __restrict__ cpj, double* __restrict__ cpm) {
    const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= ng) return;
    const uint64_t key = skey[gstart[g]];
    const uint32_t a = (uint32_t)(key >> 32), c = (uint32_t)key;
    double acc[36];
    if (a == c) {
        for (int k = 0; k < 36; k++) acc[k] = cdiag[36 * (int64_t)a + k];
    } else {
        for (int k = 0; k < 36; k++) acc[k] = 0.0;
    }
    for (int64_t t = gstart[g]; t < gstart[g + 1]; t++) {
        const int64_t q = sq[t];
        const int64_t i = pi[q], j = pj[q];
        double m[36], l[36];
        embed6<B>(pm + (int64_t)B * B * q, m);
        lift6_d(m, r + 3 * i, r + 3 * j, l);
        if (a == c) {
            for (int k = 0; k < 36; k++) acc[k] += l[k];
            for (int x = 0; x < 6; x++)
                for (int y = 0; y < 6; y++) acc[6 * x + y] += l[6 * y + x];
        } else if (of[i] < of[j]) {
            for (int k = 0; k < 36; k++) acc[k] += l[k];
        } else {
            for (int x = 0; x < 6; x++)
                for (int y = 0; y < 6; y++) acc[6 * x + y] += l[6 * y + x];
        }
    }
    if (a == c) {
        for (int k = 0; k < 36; k++) cdiag[36 * (int64_t)a + k] = acc[k];
    } else {
        const int64_t o = cross[g];
        cpi[o] = a;
        cpj[o] = c;
        for (int k = 0; k < 36; k++) cpm[36 * o + k] = acc[k];
    }
}

// full block rows: every part's diagonal block and both triangles of every pair, as
// (row << 32 | column, source) for a stable sort: source -1 - p a diagonal block, 2 e pair
// e, 2 e + 1 pair e transposed
__global__ void k_row_entries(int64_t n, int64_t np, const uint32_t* __restrict__ pi, const uint32_t* __restrict__ pj,
                              uint64_t* __restrict__ key, int64_t* __restrict__ src) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) {
        key[t] = ((uint64_t)t << 32) | (uint64_t)t;
        src[t] = -1 - t;
    } else if (t < n + 2 * np) {
        const int64_t e = (t - n) >> 1;
        const bool tr = (t - n) & 1;
        const uint64_t i = pi[e], j = pj[e];
        key[t] = tr ? ((j << 32) | i) : ((i << 32) | j);
        src[t] = 2 * e + (tr ? 1 : 0);
    }
}

template <int B>
__global__ void k_row_fill(int64_t n, int64_t m, const uint64_t* __restrict__ skey, const int64_t* __restrict__ ssrc,
                           const double* __restrict__ diag, const double* __restrict__ pm,
                           int64_t* __restrict__ rowptr, int32_t* __restrict__ col, double* __restrict__ val) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= m) return;
    const int64_t row = (int64_t)(skey[t] >> 32);
    if (t == 0 || (int64_t)(skey[t - 1] >> 32) != row) rowptr[row] = t;
    if (t == m - 1) rowptr[n] = m;
    col[t] = (int32_t)(skey[t] & 0xffffffffull);
    const int64_t s = ssrc[t];
    double* out = val + (int64_t)B * B * t;
    if (s < 0) {
        const double* d = diag + (int64_t)B * B * (-1 - s);
        for (int k = 0; k < B * B; k++) out[k] = d[k];
    } else {
        const double* p = pm + (int64_t)B * B * (s >> 1);
        if (s & 1) {
            for (int x = 0; x < B; x++)
                for (int y = 0; y < B; y++) out[B * x + y] = p[B * y + x];
        } else {
            for (int k = 0; k < B * B; k++) out[k] = p[k];
        }
    }
}

// ---- host drivers -----------------------------------------------------------------------
// A system on the device: parts (keys, positions, B x B diagonal blocks) and pairs.
struct DevSys {
    int64_t n = 0, np = 0;
    DBuf<int64_t> keys;
    DBuf<double> at, diag;
    DBuf<uint32_t> pi, pj;
    DBuf<double> pm;
};

// each part's pairs in pair order (entry 2 q + side), for the power steps' products
struct DevIncidence {
    DBuf<int64_t> ptr;
    DBuf<uint64_t> ent;
};

DevIncidence incidence(Context& ctx, const DevSys& s) {
    cudaStream_t st = ctx.stream;
    MemStats* ms = &ctx.mem;
    DevIncidence I;
    DBuf<int64_t> deg;
    deg.alloc(s.n + 1, st, ms);
    deg.zero();
    I.ptr.alloc(s.n + 1, st, ms);
    I.ent.alloc(std::max<int64_t>(2 * s.np, 1), st, ms);
    if (s.np > 0) {
        DBuf<uint32_t> key, key_s;
        DBuf<uint64_t> val;
        key.alloc(2 * s.np, st, ms);
        key_s.alloc(2 * s.np, st, ms);
        val.alloc(2 * s.np, st, ms);
        k_pair_ends<<<grid_for(s.np, LT), LT, 0, st>>>(s.np, s.pi.get(), s.pj.get(), key.get(), val.get(), deg.get());
        SC_LAUNCH_CK();
        sort_pairs(ctx, key.get(), key_s.get(), val.get(), I.ent.get(), 2 * s.np, end_bit_for(s.n));
    }
    scan_exclusive(ctx, deg.get(), I.ptr.get(), s.n + 1);
    return I;
}

double host_norm(const std::vector<double>& v) {
    double s = 0.0;
    for (double x : v) s += x * x;
    return std::sqrt(s);
}

// 4/3 over the largest eigenvalue of inv S, ten power steps from the reference's start
// (solve.rs:274-296): the products on the device, the norms on the host in order
template <int B>
double power_step(Context& ctx, const DevSys& s, const DevIncidence& I, const double* inv) {
    cudaStream_t st = ctx.stream;
    MemStats* ms = &ctx.mem;
    const int64_t n = s.n;
    std::vector<double> v((size_t)(B * n)), w((size_t)(B * n));
    for (int64_t k = 0; k < n; k++)
        for (int q = 0; q < B; q++) v[(size_t)(B * k + q)] = 1.0 + (double)((7 * k + 3 * q) % 11) / 11.0;
    DBuf<double> dv, da, dw;
    dv.alloc(B * n, st, ms);
    da.alloc(B * n, st, ms);
    dw.alloc(B * n, st, ms);
    double most = 1.0;
    for (int it = 0; it < 10; it++) {
        dv.upload(v.data(), v.size());
        k_incidence_apply<B><<<grid_for(n, LT), LT, 0, st>>>(n, I.ptr.get(), I.ent.get(), s.diag.get(), s.pm.get(),
                                                            s.pi.get(), s.pj.get(), dv.get(), da.get());
        SC_LAUNCH_CK();
        k_block_over<B><<<grid_for(n, LT), LT, 0, st>>>(n, inv, da.get(), dw.get());
        SC_LAUNCH_CK();
        dw.download(w.data(), w.size());
        SC_CK(cudaStreamSynchronize(st));
        const double nw = host_norm(w), nv = host_norm(v);
        if (nw == 0.0) break;
        most = nw / nv;
        for (size_t k = 0; k < v.size(); k++) v[k] = w[k] / nw;
    }
    return 4.0 / 3.0 / most;
}

// full B x B block rows of a system (columns in order)
template <int B>
void block_rows(Context& ctx, const DevSys& s, DBuf<int64_t>& rowptr, DBuf<int32_t>& col, DBuf<double>& val,
                int64_t& nnzb) {
    cudaStream_t st = ctx.stream;
    MemStats* ms = &ctx.mem;
    const int64_t m = s.n + 2 * s.np;
    DBuf<uint64_t> key, key_s;
    DBuf<int64_t> src, src_s;
    key.alloc(m, st, ms);
    key_s.alloc(m, st, ms);
    src.alloc(m, st, ms);
    src_s.alloc(m, st, ms);
    k_row_entries<<<grid_for(m, LT), LT, 0, st>>>(s.n, s.np, s.pi.get(), s.pj.get(), key.get(), src.get());
    SC_LAUNCH_CK();
    sort_pairs(ctx, key.get(), key_s.get(), src.get(), src_s.get(), m, 32 + end_bit_for(s.n));
    rowptr.alloc(s.n + 1, st, ms);
    col.alloc(m, st, ms);
    val.alloc((size_t)B * B * m, st, ms);
    k_row_fill<B><<<grid_for(m, LT), LT, 0, st>>>(s.n, m, key_s.get(), src_s.get(), s.diag.get(), s.pm.get(),
                                                  rowptr.get(), col.get(), val.get());
    SC_LAUNCH_CK();
    nnzb = m;
}

// One level up from system f (B x B blocks): the level's maps and blocks into L, the
// coarse system into c (solve.rs:241-271).
template <int B>
void coarsen(Context& ctx, const DevSys& f, double size, MechLevel& L, DevSys& c) {
    cudaStream_t st = ctx.stream;
    MemStats* ms = &ctx.mem;
    const int64_t nf = f.n, np = f.np;
    DBuf<int64_t> pk;
    pk.alloc(3 * nf, st, ms);
    k_parent_keys<<<grid_for(3 * nf, LT), LT, 0, st>>>(nf, f.keys.get(), pk.get());
    SC_LAUNCH_CK();
    // the union-find's roots: each component's least part
    DBuf<int32_t> lab, changed;
    lab.alloc(nf, st, ms);
    changed.alloc(1, st, ms);
    k_iota<<<grid_for(nf, LT), LT, 0, st>>>(nf, lab.get());
    SC_LAUNCH_CK();
    for (int round = 0; np > 0; round++) {
        if (round > 64 + 2 * end_bit_for(nf)) throw std::runtime_error("mech levels: labels did not settle");
        changed.zero();
        k_hook<<<grid_for(np, LT), LT, 0, st>>>(np, f.pi.get(), f.pj.get(), pk.get(), lab.get(), changed.get());
        SC_LAUNCH_CK();
        k_compress<<<grid_for(nf, LT), LT, 0, st>>>(nf, lab.get());
        SC_LAUNCH_CK();
        if (read_one(ctx, changed.get()) == 0) break;
    }
    // ids by first appearance: the roots' ranks
    DBuf<int32_t> flag, id;
    flag.alloc(nf + 1, st, ms);
    id.alloc(nf + 1, st, ms);
    k_root_flags<<<grid_for(nf, LT), LT, 0, st>>>(nf, lab.get(), flag.get());
    SC_LAUNCH_CK();
    SC_CK(cudaMemsetAsync(flag.get() + nf, 0, sizeof(int32_t), st));
    scan_exclusive(ctx, flag.get(), id.get(), nf + 1);
    const int64_t nc = read_one(ctx, id.get() + nf);
    L.n = nc;
    L.of.alloc(nf, st, ms);
    DBuf<int64_t> cnt;
    cnt.alloc(nc + 1, st, ms);
    cnt.zero();
    k_part_of<<<grid_for(nf, LT), LT, 0, st>>>(nf, lab.get(), id.get(), L.of.get(), cnt.get());
    SC_LAUNCH_CK();
    L.mptr.alloc(nc + 1, st, ms);
    scan_exclusive(ctx, cnt.get(), L.mptr.get(), nc + 1);
    // members in order: a stable sort of the parts by aggregate
    {
        DBuf<int32_t> of_s, iota;
        of_s.alloc(nf, st, ms);
        iota.alloc(nf, st, ms);
        L.mem.alloc(nf, st, ms);
        k_iota<<<grid_for(nf, LT), LT, 0, st>>>(nf, iota.get());
        SC_LAUNCH_CK();
        sort_pairs(ctx, L.of.get(), of_s.get(), iota.get(), L.mem.get(), nf, end_bit_for(nc));
    }
    c.n = nc;
    c.keys.alloc(3 * nc, st, ms);
    c.at.alloc(3 * nc, st, ms);
    k_centres<<<grid_for(nc, LT), LT, 0, st>>>(nc, L.mptr.get(), L.mem.get(), f.at.get(), pk.get(), c.at.get(),
                                               c.keys.get());
    SC_LAUNCH_CK();
    L.r.alloc(3 * nf, st, ms);
    k_offsets<<<grid_for(nf, LT), LT, 0, st>>>(nf, L.of.get(), f.at.get(), c.at.get(), L.r.get());
    SC_LAUNCH_CK();
    // the blocks
    c.diag.alloc(36 * nc, st, ms);
    k_member_blocks<B><<<grid_for(nc, LT), LT, 0, st>>>(nc, L.mptr.get(), L.mem.get(), f.diag.get(), L.r.get(),
                                                        c.diag.get());
    SC_LAUNCH_CK();
    c.np = 0;
    if (np > 0) {
        DBuf<uint64_t> key, skey;
        DBuf<uint32_t> q, sq;
        key.alloc(np, st, ms);
        skey.alloc(np, st, ms);
        q.alloc(np, st, ms);
        sq.alloc(np, st, ms);
        k_pair_groups<<<grid_for(np, LT), LT, 0, st>>>(np, f.pi.get(), f.pj.get(), L.of.get(), key.get(), q.get());
        SC_LAUNCH_CK();
        sort_pairs(ctx, key.get(), skey.get(), q.get(), sq.get(), np, 32 + end_bit_for(nc));
        DBuf<int64_t> gflag, gid;
        gflag.alloc(np + 1, st, ms);
        gid.alloc(np + 1, st, ms);
        k_group_flags<<<grid_for(np, LT), LT, 0, st>>>(np, skey.get(), gflag.get());
        SC_LAUNCH_CK();
        SC_CK(cudaMemsetAsync(gflag.get() + np, 0, sizeof(int64_t), st));
        scan_exclusive(ctx, gflag.get(), gid.get(), np + 1);
        const int64_t ng = read_one(ctx, gid.get() + np);
        DBuf<int64_t> gstart, cross, cidx;
        gstart.alloc(ng + 1, st, ms);
        cross.alloc(ng + 1, st, ms);
        cidx.alloc(ng + 1, st, ms);
        k_group_starts<<<grid_for(np, LT), LT, 0, st>>>(np, gflag.get(), gid.get(), skey.get(), gstart.get(),
                                                        cross.get());
        SC_LAUNCH_CK();
        SC_CK(cudaMemcpyAsync(gstart.get() + ng, &np, sizeof(int64_t), cudaMemcpyHostToDevice, st));
        SC_CK(cudaMemsetAsync(cross.get() + ng, 0, sizeof(int64_t), st));
        scan_exclusive(ctx, cross.get(), cidx.get(), ng + 1);
        c.np = read_one(ctx, cidx.get() + ng);
        c.pi.alloc(std::max<int64_t>(c.np, 1), st, ms);
        c.pj.alloc(std::max<int64_t>(c.np, 1), st, ms);
        c.pm.alloc(36 * std::max<int64_t>(c.np, 1), st, ms);
        k_group_blocks<B><<<grid_for(ng, LT), LT, 0, st>>>(ng, gstart.get(), skey.get(), sq.get(), f.pi.get(),
                                                           f.pj.get(), f.pm.get(), L.of.get(), L.r.get(),
                                                           cidx.get(), c.diag.get(), c.pi.get(), c.pj.get(),
                                                           c.pm.get());
        SC_LAUNCH_CK();
    }
}

}  // namespace

void mech_device_levels(Context& ctx, int64_t n, const int64_t* sites, const double* at, const double* diag,
                        int64_t npairs, const uint32_t* pi, const uint32_t* pj, const double* pb, double size,
                        MechLevels& out) {
    cudaStream_t st = ctx.stream;
    MemStats* ms = &ctx.mem;
    // the nodes: 3 x 3 blocks
    DevSys f;
    f.n = n;
    f.np = npairs;
    f.keys.alloc(3 * n, st, ms);
    f.keys.upload(sites, 3 * n);
    f.at.alloc(3 * n, st, ms);
    f.at.upload(at, 3 * n);
    f.diag.alloc(9 * n, st, ms);
    f.diag.upload(diag, 9 * n);
    f.pi.alloc(std::max<int64_t>(npairs, 1), st, ms);
    f.pj.alloc(std::max<int64_t>(npairs, 1), st, ms);
    f.pm.alloc(9 * std::max<int64_t>(npairs, 1), st, ms);
    f.pi.upload(pi, npairs);
    f.pj.upload(pj, npairs);
    f.pm.upload(pb, 9 * npairs);
    out.n0 = n;
    out.inv0.alloc(9 * n, st, ms);
    k_block_inverses<3, false><<<grid_for(n, LT), LT, 0, st>>>(n, f.diag.get(), 0.0, out.inv0.get());
    SC_LAUNCH_CK();
    {
        const DevIncidence I = incidence(ctx, f);
        out.step0 = power_step<3>(ctx, f, I, out.inv0.get());
    }
    int64_t nnz0 = 0;
    block_rows<3>(ctx, f, out.rowptr0, out.col0, out.val0, nnz0);
    // the coarse levels (solve.rs:365-385)
    out.lv.clear();
    double sz = size;
    DevSys cur;
    bool first = true;
    for (;;) {
        MechLevel L;
        DevSys c;
        if (first)
            coarsen<3>(ctx, f, sz * 2.0, L, c);
        else
            coarsen<6>(ctx, cur, sz * 2.0, L, c);
        const int64_t before = first ? n : out.lv.back().n;
        first = false;
        const double lsize = sz * 2.0;
        sz *= 2.0;
        L.b.alloc(6 * L.n, st, ms);
        L.x.alloc(6 * L.n, st, ms);
        L.res.alloc(6 * L.n, st, ms);
        L.t.alloc(6 * L.n, st, ms);
        L.inv.alloc(36 * L.n, st, ms);
        k_block_inverses<6, true><<<grid_for(L.n, LT), LT, 0, st>>>(L.n, c.diag.get(), lsize, L.inv.get());
        SC_LAUNCH_CK();
        if ((size_t)L.n <= MECH_DIRECT || L.n == before) {
            // the direct top, on the host (small: at most MECH_DIRECT parts, or a level
            // that no longer shrinks)
            std::vector<double> hd(36 * L.n), hm(36 * c.np);
            std::vector<uint32_t> hi(c.np), hj(c.np);
            c.diag.download(hd.data(), hd.size());
            if (c.np > 0) {
                c.pi.download(hi.data(), c.np);
                c.pj.download(hj.data(), c.np);
                c.pm.download(hm.data(), hm.size());
            }
            SC_CK(cudaStreamSynchronize(st));
            const std::vector<double> top =
                mech_top_inverse(L.n, hd.data(), c.np, hi.data(), hj.data(), hm.data(), lsize);
            L.top_inv.alloc(top.size(), st, ms);
            L.top_inv.upload(top.data(), top.size());
            SC_CK(cudaStreamSynchronize(st));
            L.direct = true;
            L.step_h = 0.0;
            out.lv.push_back(std::move(L));
            break;
        }
        {
            const DevIncidence I = incidence(ctx, c);
            L.step_h = power_step<6>(ctx, c, I, L.inv.get());
        }
        L.step.alloc(1, st, ms);
        L.step.upload(&L.step_h, 1);
        block_rows<6>(ctx, c, L.rowptr, L.col, L.val, L.nnzb);
        SC_CK(cudaStreamSynchronize(st));  // the step's host copy goes out of scope after the upload
        out.lv.push_back(std::move(L));
        cur = std::move(c);
    }
}

}  // namespace sc
