// The hierarchy of bodies within bodies (statics/src/bodies.rs:123-282, 444-461), built
// on the device for every piece of a batch at once:
//   * block inverses of each part's own block (Gauss-Jordan, bodies.rs:576-602);
//   * the smoother step 4/3 / lambda_max(D^-1 K) by 12 power steps from the reference's
//     start vector (bodies.rs:180-190);
//   * bodies: connected pieces of equal octree key over the level's stored pairs, ids by
//     first appearance (bodies.rs:472-496) -- bit-exact: component minima by label
//     propagation, ids by an exclusive scan over the roots in part order;
//   * the smoothed prolongator P = (I - step D^-1 K) P0 and the Galerkin product P'KP
//     (bodies.rs:228-282), symbolic patterns by expand / sort / unique (the pattern is
//     the reference's merge pattern, structural zeros included), values by one warp
//     per output row;
//   * each piece's top level as a dense factor (bodies.rs:286-315), kept as its inverse.
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <cstdlib>

#include "kernels.cuh"
#include "level0_blocks.cuh"
#include "rowprod.cuh"

namespace sc {


namespace {

__global__ void k_find_diag_invert(int64_t n, const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                                   const double* __restrict__ val, double* __restrict__ inv,
                                   const int32_t* __restrict__ piece, int32_t* __restrict__ status) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    int64_t e = lower_bound_i32(col, rowptr[k], rowptr[k + 1], (int32_t)k);
    bool ok = e < rowptr[k + 1] && col[e] == (int32_t)k;
    double tmp[36];
    if (ok) ok = invert6(val + 36 * e, tmp);
    if (!ok) {
        for (int i = 0; i < 36; i++) tmp[i] = 0.0;
        if (status) atomicMax(status + piece[k], (int)SC_BREAKDOWN);
    }
    for (int i = 0; i < 36; i++) inv[36 * k + i] = tmp[i];
}

// the same for a matrix-free level 0: each part's own block from the cell template
__global__ void k_diag_invert_k0(int64_t n, K0View v, double* __restrict__ inv, const int32_t* __restrict__ piece,
                                 int32_t* __restrict__ status) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    K0Row row = k0_row(v, k);
    double blk[36], tmp[36];
    for (int t = 0; t < 36; t++) blk[t] = k0_entry(v.tpl_s, row, K0_DIAG, t / 6, t % 6);
    bool ok = invert6(blk, tmp);
    if (!ok) {
        for (int i = 0; i < 36; i++) tmp[i] = 0.0;
        if (status) atomicMax(status + piece[k], (int)SC_BREAKDOWN);
    }
    for (int i = 0; i < 36; i++) inv[36 * k + i] = tmp[i];
}

__global__ void k_to_float(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}

// v[k][s] = 1 + ((7k + 3s) mod 11) / 11, k counted within the piece (bodies.rs:181)
__global__ void k_power_start(int64_t n, const int64_t* __restrict__ pstart, const int32_t* __restrict__ piece,
                              double* __restrict__ v) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    int64_t kl = k - pstart[piece[k]];
    for (int s = 0; s < 6; s++) v[6 * k + s] = 1.0 + (double)((7 * kl + 3 * s) % 11) / 11.0;
}

// most = |w| / |v|; v = w / |w| (bodies.rs:184-187)
__global__ void k_power_scale(int64_t n, const int32_t* __restrict__ piece, const double* __restrict__ ww,
                              const double* __restrict__ w, double* __restrict__ v) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= 6 * n) return;
    double scale = 1.0 / sqrt(ww[piece[i / 6]]);
    v[i] = w[i] * scale;
}

__global__ void k_power_most(int np, const double* __restrict__ ww, const double* __restrict__ vv,
                             double* __restrict__ most) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    most[p] = sqrt(ww[p]) / sqrt(vv[p]);
}

__global__ void k_step(int np, const double* __restrict__ most, double* __restrict__ step) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    step[p] = 4.0 / 3.0 / most[p];
}

// ---- bodies ---------------------------------------------------------------------
__device__ __forceinline__ bool same_key(const int64_t* __restrict__ site, int64_t i, int64_t j, int64_t mask) {
    return (site[3 * i] & mask) == (site[3 * j] & mask) && (site[3 * i + 1] & mask) == (site[3 * j + 1] & mask) &&
           (site[3 * i + 2] & mask) == (site[3 * j + 2] & mask);
}

__global__ void k_label_init(int64_t n, int32_t* __restrict__ label) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k < n) label[k] = (int32_t)k;
}

// One sweep of minimum-label propagation over pairs of equal key, then pointer jumping.
__global__ void k_label_sweep(int64_t n, const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                              const int64_t* __restrict__ site, int64_t mask, const int32_t* __restrict__ active,
                              const int32_t* __restrict__ piece, int32_t* __restrict__ label,
                              int32_t* __restrict__ changed) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (!active[piece[k]]) return;
    int32_t m = label[k];
    for (int64_t e = rowptr[k]; e < rowptr[k + 1]; e++) {
        int32_t j = col[e];
        if (j == (int32_t)k) continue;
        if (same_key(site, k, j, mask)) {
            int32_t lj = label[j];
            if (lj < m) m = lj;
        }
    }
    int32_t old = label[k];
    if (m < old) {
        atomicMin(label + k, m);
        atomicMin(label + old, m);
        *changed = 1;
    }
}

__global__ void k_label_jump(int64_t n, int32_t* __restrict__ label) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    int32_t l = label[k];
    int32_t ll = label[l];
    while (ll != l) {
        l = ll;
        ll = label[l];
    }
    label[k] = l;
}

__global__ void k_roots(int64_t n, const int32_t* __restrict__ label, const int32_t* __restrict__ piece,
                        int64_t* __restrict__ root, int32_t* __restrict__ bodies_per_piece) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    int r = label[k] == (int32_t)k;
    root[k] = r;
    if (r) atomicAdd(bodies_per_piece + piece[k], 1);
}

__global__ void k_mask_roots(int64_t n, const int32_t* __restrict__ piece, const int32_t* __restrict__ active,
                             int64_t* __restrict__ root) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (!active[piece[k]]) root[k] = 0;
}

__global__ void k_up(int64_t n, const int32_t* __restrict__ label, const int64_t* __restrict__ id,
                     const int32_t* __restrict__ piece, const int32_t* __restrict__ active, int32_t* __restrict__ up,
                     int32_t* __restrict__ top_of_part) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    bool a = active[piece[k]];
    up[k] = a ? (int32_t)id[label[k]] : -1;
    top_of_part[k] = a ? 0 : 1;
}

// members of each body in part order: body c's parts are mem[moff[c] .. moff[c+1])
__global__ void k_centroid(int64_t nc, const int64_t* __restrict__ moff, const int32_t* __restrict__ mem,
                           const double* __restrict__ centre, const int64_t* __restrict__ site,
                           const int32_t* __restrict__ piece, double* __restrict__ centre_c,
                           int64_t* __restrict__ site_c, int32_t* __restrict__ piece_c) {
    int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= nc) return;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, cnt = 0.0;
    for (int64_t t = moff[c]; t < moff[c + 1]; t++) {
        int32_t k = mem[t];
        s0 += centre[3 * (int64_t)k];
        s1 += centre[3 * (int64_t)k + 1];
        s2 += centre[3 * (int64_t)k + 2];
        cnt += 1.0;
    }
    double inv = 1.0 / cnt;
    centre_c[3 * c] = s0 * inv;
    centre_c[3 * c + 1] = s1 * inv;
    centre_c[3 * c + 2] = s2 * inv;
    int32_t k0 = mem[moff[c]];
    for (int q = 0; q < 3; q++) site_c[3 * c + q] = site[3 * (int64_t)k0 + q];
    piece_c[c] = piece[k0];
}

__global__ void k_offsets_from_sorted(int64_t m, const int32_t* __restrict__ keys, int64_t nkeys,
                                      int64_t* __restrict__ off) {
    // off[c] = first index with keys >= c, for c in [0, nkeys]; keys sorted
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i > m) return;
    int32_t prev = i == 0 ? -1 : keys[i - 1];
    int32_t cur = i == m ? (int32_t)nkeys : keys[i];
    for (int32_t c = prev + 1; c <= cur; c++) off[c] = i;
}

// ---- patterns by expand / sort / unique --------------------------------------------
__global__ void k_count_P(int64_t n, const int64_t* __restrict__ rowptr, const int32_t* __restrict__ up,
                          int64_t* __restrict__ cnt) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    cnt[k] = up[k] >= 0 ? rowptr[k + 1] - rowptr[k] : 0;
}
__global__ void k_fill_P(int64_t n, const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                         const int32_t* __restrict__ up, const int64_t* __restrict__ off, uint64_t* __restrict__ keys,
                         int cb) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (up[k] < 0) return;
    int64_t o = off[k];
    for (int64_t e = rowptr[k]; e < rowptr[k + 1]; e++) keys[o++] = ((uint64_t)k << cb) | (uint32_t)up[col[e]];
}
// candidates of K P, per block K_kq (entry e of K, row krow[e]): one per block P_qf,
// (k, col of P_qf) with contribution (e << 32 | f). Entries are laid out in entry order,
// so the list is row by row, K's columns in order, then P's.
// Only the blocks of K P that P' (K P) reads are made: an entry (k, c) of P meets the
// blocks (k, d >= c) of K P row k, so columns below P row k's first column are never
// read (about a third of K P) and are left out.
__device__ __forceinline__ int64_t kp_first(const int64_t* __restrict__ prow, const int32_t* __restrict__ pcol,
                                            int32_t k, int32_t q) {
    return lower_bound_i32(pcol, prow[q], prow[q + 1], pcol[prow[k]]);
}
__global__ void k_count_KP(int64_t nnz, const int32_t* __restrict__ krow, const int32_t* __restrict__ col,
                           const int64_t* __restrict__ prow, const int32_t* __restrict__ pcol,
                           const int32_t* __restrict__ up, int64_t* __restrict__ cnt) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    const int32_t k = krow[e], q = col[e];
    cnt[e] = up[k] >= 0 ? prow[q + 1] - kp_first(prow, pcol, k, q) : 0;
}
__global__ void k_fill_KP(int64_t nnz, const int32_t* __restrict__ krow, const int32_t* __restrict__ col,
                          const int64_t* __restrict__ prow, const int32_t* __restrict__ pcol,
                          const int32_t* __restrict__ up, const int64_t* __restrict__ off, uint64_t* __restrict__ keys,
                          uint64_t* __restrict__ vals, int cb) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    int32_t k = krow[e];
    if (up[k] < 0) return;
    int32_t q = col[e];
    int64_t o = off[e];
    for (int64_t f = kp_first(prow, pcol, k, q); f < prow[q + 1]; f++, o++) {
        keys[o] = ((uint64_t)(uint32_t)k << cb) | (uint32_t)pcol[f];
        vals[o] = ((uint64_t)e << 32) | (uint64_t)f;
    }
}
// per P entry e = (k, c), k = prow_of[e]: the columns d >= c of KP row k
__global__ void k_count_C(int64_t pnnz, const int32_t* __restrict__ prow_of, const int32_t* __restrict__ pcol,
                          const int64_t* __restrict__ kprow, const int32_t* __restrict__ kpcol, int64_t* __restrict__ cnt) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= pnnz) return;
    int32_t k = prow_of[e];
    int64_t lb = lower_bound_i32(kpcol, kprow[k], kprow[k + 1], pcol[e]);
    cnt[e] = kprow[k + 1] - lb;
}
// candidates of the upper P'KP: (c, d) for each entry (k, c) of P with c0 <= c < c1 and
// each block (k, d >= c) of K P, contribution (entry of P << 32 | entry of KP)
__global__ void k_fill_C(int64_t pnnz, const int32_t* __restrict__ prow_of, const int32_t* __restrict__ pcol,
                         const int64_t* __restrict__ kprow, const int32_t* __restrict__ kpcol,
                         const int64_t* __restrict__ off, uint64_t* __restrict__ keys, uint64_t* __restrict__ vals,
                         int cb, int32_t c0, int32_t c1) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= pnnz) return;
    int32_t k = prow_of[e];
    int32_t c = pcol[e];
    if (c < c0 || c >= c1) return;
    int64_t lb = lower_bound_i32(kpcol, kprow[k], kprow[k + 1], c);
    int64_t o = off[e];
    for (int64_t f = lb; f < kprow[k + 1]; f++, o++) {
        keys[o] = ((uint64_t)(uint32_t)c << cb) | (uint32_t)kpcol[f];
        vals[o] = ((uint64_t)e << 32) | (uint64_t)f;
    }
}
// the upper P'KP's candidates per coarse row (cnt zeroed beforehand)
__global__ void k_row_cands(int64_t pnnz, const int32_t* __restrict__ pcol, const int64_t* __restrict__ ecnt,
                            int64_t* __restrict__ cnt) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e < pnnz && ecnt[e]) atomicAdd(reinterpret_cast<unsigned long long*>(cnt + pcol[e]), (unsigned long long)ecnt[e]);
}
// the counts of the P entries whose coarse row is in [c0, c1), others 0
__global__ void k_slice_counts(int64_t pnnz, const int32_t* __restrict__ pcol, const int64_t* __restrict__ ecnt,
                               int32_t c0, int32_t c1, int64_t* __restrict__ out) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e < pnnz) out[e] = (pcol[e] >= c0 && pcol[e] < c1) ? ecnt[e] : 0;
}
// a += b
__global__ void k_add_i64(int64_t n, int64_t* __restrict__ a, const int64_t* __restrict__ b) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) a[i] += b[i];
}
// keys are (row << cb | col)
__global__ void k_unpack_pattern(int64_t m, const uint64_t* __restrict__ keys, int32_t* __restrict__ col,
                                 int32_t* __restrict__ row, int cb) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= m) return;
    col[i] = (int32_t)(keys[i] & ((uint64_t(1) << cb) - 1));
    row[i] = (int32_t)(keys[i] >> cb);
}

// ---- numeric products, one warp per output row ----------------------------------------
// acc(r, c) += sum_j A(r, j) B(j, c) for the lane's entries (e = lane, lane + 32 < 36).
// A transposed when TA. B is a rigid shift [I M; 0 I] with M w = w x r when RB (rv = r).
template <bool TA, bool RB>
__device__ __forceinline__ void warp_block_mac(int lane, const double* __restrict__ A, const double* __restrict__ B,
                                               const double* rv, double* __restrict__ C) {
#pragma unroll
    for (int rep = 0; rep < 2; rep++) {
        int e = lane + 32 * rep;
        if (e >= 36) break;
        int r = e / 6, c = e % 6;
        double s = 0.0;
        if (RB) {
            // column c of R: c < 3 -> e_c; c >= 3 -> (M[:, c-3], e_c)
            double a0 = TA ? A[0 * 6 + r] : A[r * 6 + 0];
            double a1 = TA ? A[1 * 6 + r] : A[r * 6 + 1];
            double a2 = TA ? A[2 * 6 + r] : A[r * 6 + 2];
            if (c < 3) {
                s = c == 0 ? a0 : (c == 1 ? a1 : a2);
            } else {
                double ac = TA ? A[c * 6 + r] : A[r * 6 + c];
                // M = [[0, r2, -r1], [-r2, 0, r0], [r1, -r0, 0]]
                double m0, m1, m2;
                if (c == 3) { m0 = 0.0; m1 = -rv[2]; m2 = rv[1]; }
                else if (c == 4) { m0 = rv[2]; m1 = 0.0; m2 = -rv[0]; }
                else { m0 = -rv[1]; m1 = rv[0]; m2 = 0.0; }
                s = fma(a0, m0, fma(a1, m1, fma(a2, m2, ac)));
            }
        } else {
#pragma unroll
            for (int j = 0; j < 6; j++) {
                double a = TA ? A[j * 6 + r] : A[r * 6 + j];
                s = fma(a, B[j * 6 + c], s);
            }
        }
        C[e] += s;
    }
}

// S[k][pos(up[o])] += K_ko R_o over the row; then P_k = delta R_k - step D_k^-1 S.
// K0: level 0 of voxel pieces, blocks made from the cell template (val unused).
template <bool K0>
__global__ void __launch_bounds__(256) k_num_P(int64_t n, const int64_t* __restrict__ rowptr,
                                               const int32_t* __restrict__ col, const double* __restrict__ val,
                                               K0View k0, const int32_t* __restrict__ up,
                                               const double* __restrict__ rvec, const double* __restrict__ inv,
                                               const double* __restrict__ step, const int32_t* __restrict__ piece,
                                               const int64_t* __restrict__ prow, const int32_t* __restrict__ pcol,
                                               double* __restrict__ pval) {
    // S's blocks of the warp's row are summed in shared memory when the P row has at most
    // NUM_P_SMEM blocks (else in pval, zeroed beforehand): the same additions, in order
    constexpr int NUM_P_SMEM = 12;
    __shared__ double blk_s[8][36];                 // K0: the warp's current block
    __shared__ double s_s[8][NUM_P_SMEM * 36];
    int64_t k = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (k >= n) return;
    int lane = threadIdx.x & 31;
    if (up[k] < 0) return;
    const int w = (threadIdx.x >> 5) & 7;
    double* blk = blk_s[w];
    K0Row row{};
    if (K0) row = k0_row(k0, k);
    const int64_t p0 = prow[k], p1 = prow[k + 1];
    const bool local = p1 - p0 <= NUM_P_SMEM;
    double* S = local ? s_s[w] : pval + 36 * p0;
    if (local)
        for (int t = lane; t < 36 * (int)(p1 - p0); t += 32) S[t] = 0.0;
    __syncwarp();
    const int64_t e1 = rowptr[k + 1];
    for (int64_t eb = rowptr[k]; eb < e1; eb += 32) {
        // lane t finds its entry's block of P row k (independent searches), then the
        // warp adds the entries one by one
        int32_t mo = 0;
        int mpos = 0;
        if (eb + lane < e1) {
            mo = col[eb + lane];
            mpos = (int)(lower_bound_i32(pcol, p0, p1, up[mo]) - p0);
        }
        const int nb = (int)min((int64_t)32, e1 - eb);
        for (int t = 0; t < nb; t++) {
            const int64_t e = eb + t;
            const int32_t o = __shfl_sync(0xffffffffu, mo, t);
            const int pos = __shfl_sync(0xffffffffu, mpos, t);
            double rv[3] = {rvec[3 * (int64_t)o], rvec[3 * (int64_t)o + 1], rvec[3 * (int64_t)o + 2]};
            const double* A = val + 36 * e;
            if (K0) {
                uint8_t d = k0.desc[e];
                for (int q = lane; q < 36; q += 32) blk[q] = k0_entry(k0.tpl_s, row, d, q / 6, q % 6);
                __syncwarp();
                A = blk;
            }
            warp_block_mac<false, true>(lane, A, nullptr, rv, S + 36 * pos);
            __syncwarp();
        }
    }
    double st = step[piece[k]];
    const double* D = inv + 36 * k;
    double rk[3] = {rvec[3 * k], rvec[3 * k + 1], rvec[3 * k + 2]};
    for (int64_t pos = p0; pos < p1; pos++) {
        const double* Sp = S + 36 * (pos - p0);
        double out[2];
#pragma unroll
        for (int rep = 0; rep < 2; rep++) {
            int e = lane + 32 * rep;
            out[rep] = 0.0;
            if (e < 36) {
                int r = e / 6, c = e % 6;
                double s = 0.0;
                for (int j = 0; j < 6; j++) s = fma(D[r * 6 + j], Sp[j * 6 + c], s);
                double rig = 0.0;
                if (pcol[pos] == up[k]) {
                    if (r == c) rig = 1.0;
                    else if (r < 3 && c >= 3) {
                        // M[r][c-3]
                        int cc = c - 3;
                        if (r == 0) rig = cc == 1 ? rk[2] : (cc == 2 ? -rk[1] : 0.0);
                        if (r == 1) rig = cc == 0 ? -rk[2] : (cc == 2 ? rk[0] : 0.0);
                        if (r == 2) rig = cc == 0 ? rk[1] : (cc == 1 ? -rk[0] : 0.0);
                    }
                }
                out[rep] = rig + (-st) * s;
            }
        }
        __syncwarp();
        double* P = pval + 36 * pos;
        if (lane < 36) P[lane] = out[0];
        if (lane + 32 < 36) P[lane + 32] = out[1];
        __syncwarp();
    }
}



// Every output block of a product as the ordered sum of its contributions: after the
// symbolic sort, output block q's contributions are vals[seg[q] .. seg[q+1]), each the
// pair (a << 32 | b) of a left block and a right block, in the order the candidates were
// generated (a stable sort), so the sum is deterministic. Every entry (r, c) is summed
// over the contributions in list order, each contribution's six products first, as a
// one-thread-per-entry sum would.
constexpr int SUM_GROUPS = 32;  // output blocks per thread block, 6 threads each
constexpr int SUM_THREADS = 6 * SUM_GROUPS;
// out[q] = sum over q's contributions (a << 32 | b) of op(A_a) B_b, op = transpose when TA.
// Six threads per output block, thread c owning its column c: each reads the whole left
// block (the same addresses across the six, one transaction) and its column of the
// right one, so a contribution costs 42 loads a thread instead of 12 for each of 36
// threads.
template <bool TA, class TAV, class TB>
__global__ void __launch_bounds__(SUM_THREADS) k_sum_products(int64_t nout, const int64_t* __restrict__ seg,
                                                             const uint64_t* __restrict__ vals,
                                                             const TAV* __restrict__ A,
                                                             const TB* __restrict__ B, double* __restrict__ out) {
    const int g = threadIdx.x / 6, c = threadIdx.x % 6;
    const int64_t q = (int64_t)blockIdx.x * SUM_GROUPS + g;
    if (q >= nout) return;
    int64_t i = seg[q];
    const int64_t end = seg[q + 1];
    double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    // one contribution's operands: column c of its right block and its left block
    struct Ops {
        double bc[6];
        double av[36];
    };
    auto load = [&](uint64_t v, Ops& o) {
        const TB* bb = B + 36 * (int64_t)(v & 0xffffffffu);
#pragma unroll
        for (int j = 0; j < 6; j++) o.bc[j] = (double)bb[j * 6 + c];
        if constexpr (sizeof(TAV) == 8) {
            const double2* a2 = reinterpret_cast<const double2*>(A + 36 * (int64_t)(v >> 32));
#pragma unroll
            for (int t = 0; t < 18; t++) {
                double2 w = a2[t];
                o.av[2 * t] = w.x;
                o.av[2 * t + 1] = w.y;
            }
        } else {
            const float4* a4 = reinterpret_cast<const float4*>(A + 36 * (int64_t)(v >> 32));
#pragma unroll
            for (int t = 0; t < 9; t++) {
                float4 w = a4[t];
                o.av[4 * t] = (double)w.x;
                o.av[4 * t + 1] = (double)w.y;
                o.av[4 * t + 2] = (double)w.z;
                o.av[4 * t + 3] = (double)w.w;
            }
        }
    };
    // acc(r) += sum_j op(A)(r, j) B(j, c)
    auto add = [&](const Ops& o) {
#pragma unroll
        for (int r = 0; r < 6; r++) {
            double s = 0.0;
#pragma unroll
            for (int j = 0; j < 6; j++) s = fma(TA ? o.av[j * 6 + r] : o.av[r * 6 + j], o.bc[j], s);
            acc[r] += s;
        }
    };
    // two contributions' loads in flight, added in list order
    for (; i + 2 <= end; i += 2) {
        Ops o0, o1;
        load(vals[i], o0);
        load(vals[i + 1], o1);
        add(o0);
        add(o1);
    }
    if (i < end) {
        Ops o0;
        load(vals[i], o0);
        add(o0);
    }
#pragma unroll
    for (int r = 0; r < 6; r++) out[36 * q + 6 * r + c] = acc[r];
}

// The same for K P on a matrix-free level 0: the left block of contribution (e << 32 | f)
// is block e of the level-0 pattern, made from the cell template (krow gives its row),
// the right one block f of P. Thread c of a group owns column c of the output block as
// above, but makes only row c of each template block and takes the other rows from its
// group's lanes by shuffles, so the groups sit inside warps: five to a warp, two lanes
// idle. Blocks stay resident, striding over the outputs (the template is staged once
// per block).
constexpr int K0SUM_WARPS = 6;
constexpr int K0SUM_GROUPS = 5 * K0SUM_WARPS;
template <class TB, class TO>
__global__ void __launch_bounds__(32 * K0SUM_WARPS) k_sum_products_k0(int64_t nout, const int64_t* __restrict__ seg,
                                                                     const uint64_t* __restrict__ vals,
                                                                     const TB* __restrict__ B,
                                                                     TO* __restrict__ out, K0View k0,
                                                                     const int32_t* __restrict__ krow) {
    __shared__ double T[36 * 36];
    for (int t = threadIdx.x; t < 36 * 36; t += blockDim.x) T[t] = k0.tpl_s[t];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gl = min(lane / 6, 4), c = lane - 6 * gl;  // lanes 30, 31 shadow group 4's lanes 0, 1
    const bool idle = lane >= 30;
    const int base = 6 * gl;
    const int g = 5 * warp + gl;
    // the whole warp runs the same trip count, so the shuffles always find every lane
    const int64_t first_q = (int64_t)blockIdx.x * K0SUM_GROUPS;
    for (int64_t q0 = first_q; q0 < nout; q0 += (int64_t)gridDim.x * K0SUM_GROUPS) {
        const int64_t q = q0 + g;
        const bool live = !idle && q < nout;
        int64_t i = live ? seg[q] : 0;
        const int64_t end = live ? seg[q + 1] : 0;
        K0Row row{};
        if (i < end) row = k0_row(k0, krow[vals[i] >> 32]);
        // the most contributions of any group of the warp
        int64_t n = end - i, most = n;
#pragma unroll
        for (int o = 16; o; o >>= 1) most = max(most, __shfl_xor_sync(0xffffffffu, most, o));
        double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int64_t t = 0; t < most; t++) {
            const bool has = t < n;
            double bc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, ar[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            if (has) {
                const uint64_t v = vals[i + t];
                const TB* bb = B + 36 * (int64_t)(v & 0xffffffffu);
#pragma unroll
                for (int j = 0; j < 6; j++) bc[j] = (double)bb[j * 6 + c];
                const uint8_t d = k0.desc[v >> 32];
#pragma unroll
                for (int j = 0; j < 6; j++) ar[j] = k0_entry(T, row, d, c, j);  // row c of A
            }
            // acc(r) += sum_j A(r, j) B(j, c), row r of A from lane base + r
#pragma unroll
            for (int r = 0; r < 6; r++) {
                double s = 0.0;
#pragma unroll
                for (int j = 0; j < 6; j++) s = fma(__shfl_sync(0xffffffffu, ar[j], base + r), bc[j], s);
                if (has) acc[r] += s;
            }
        }
        if (live)
#pragma unroll
            for (int r = 0; r < 6; r++) out[36 * q + 6 * r + c] = (TO)acc[r];
    }
}

// P' as its own block rows: block t = transpose of P's block tent[t]
__global__ void k_transpose_gather(int64_t m, const int64_t* __restrict__ tent, const double* __restrict__ pval,
                                   double* __restrict__ ptval) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= 36 * m) return;
    int64_t t = i / 36;
    int e = (int)(i % 36), r = e / 6, c = e % 6;
    ptval[i] = pval[36 * tent[t] + c * 6 + r];
}

// full symmetric storage: entry i of the full pattern copies upper entry src[i] & mask,
// transposed when its top bit is set
__global__ void k_mirror_vals(int64_t m, const int64_t* __restrict__ src, const double* __restrict__ up_val,
                              double* __restrict__ val) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= 36 * m) return;
    int64_t b = i / 36;
    int e = (int)(i % 36);
    int64_t s = src[b];
    bool tr = s < 0;
    int64_t u = tr ? ~s : s;
    int r = e / 6, c = e % 6;
    val[i] = tr ? up_val[36 * u + c * 6 + r] : up_val[36 * u + e];
}
__global__ void k_mirror_keys(int64_t m, const int32_t* __restrict__ row, const int32_t* __restrict__ col,
                              uint64_t* __restrict__ keys, int64_t* __restrict__ src, const int64_t* __restrict__ off) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= m) return;
    int64_t o = off[i];
    uint32_t r = (uint32_t)row[i], c = (uint32_t)col[i];
    keys[o] = ((uint64_t)r << 32) | c;
    src[o] = i;
    if (c != r) {
        keys[o + 1] = ((uint64_t)c << 32) | r;
        src[o + 1] = ~i;
    }
}
__global__ void k_mirror_count(int64_t m, const int32_t* __restrict__ row, const int32_t* __restrict__ col,
                               int64_t* __restrict__ cnt) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= m) return;
    cnt[i] = row[i] == col[i] ? 1 : 2;
}

__global__ void k_rvec(int64_t n, const int32_t* __restrict__ up, const double* __restrict__ centre,
                       const double* __restrict__ centre_c, double* __restrict__ rvec) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    int32_t c = up[k];
    for (int q = 0; q < 3; q++) rvec[3 * k + q] = c >= 0 ? centre[3 * k + q] - centre_c[3 * (int64_t)c + q] : 0.0;
}

// ---- dense top ---------------------------------------------------------------------
// The dense top of each listed piece, block (., i) for top i: its blocks scattered into
// the piece's n x n row-major matrix at A + off[i] (zeroed beforehand).
template <bool K0>
__global__ void k_dense_from_bsr_all(const int32_t* __restrict__ top, const int64_t* __restrict__ pstart,
                                     const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                                     const double* __restrict__ val, K0View k0, const int64_t* __restrict__ off,
                                     double* __restrict__ A_all) {
    int p = top[blockIdx.y];
    int64_t k0p = pstart[p], k1 = pstart[p + 1];
    int64_t n = 6 * (k1 - k0p);
    double* A = A_all + off[blockIdx.y];
    for (int64_t k = k0p + blockIdx.x; k < k1; k += gridDim.x) {
        K0Row row{};
        if (K0) row = k0_row(k0, k);
        for (int64_t e = rowptr[k]; e < rowptr[k + 1]; e++) {
            int64_t j = col[e];
            for (int t = threadIdx.x; t < 36; t += blockDim.x) {
                int r = t / 6, c = t % 6;
                A[(6 * (k - k0p) + r) * n + 6 * (j - k0p) + c] =
                    K0 ? k0_entry(k0.tpl_s, row, k0.desc[e], r, c) : val[36 * e + t];
            }
        }
    }
}

// Left-looking Cholesky in the reference's order (bodies.rs:307-313), then X = L^-1 by
// columns and Kinv = X' X written over A (A is not read once X is complete). One block.
__device__ void cholesky_inverse_block(int n, double* A, double* __restrict__ X, int32_t* __restrict__ status,
                                       int piece) {
    __shared__ double red[32];
    __shared__ double dsh;
    __shared__ int bad;
    if (threadIdx.x == 0) bad = 0;
    const int nw = (int)(blockDim.x + 31) / 32;
    for (int j = 0; j < n; j++) {
        // the diagonal's sum: within each warp by shuffles, then the warps' sums by thread
        // 0 (two barriers a column)
        double s = 0.0;
        for (int k = threadIdx.x; k < j; k += blockDim.x) s = fma(A[(int64_t)j * n + k], A[(int64_t)j * n + k], s);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double sum = 0.0;
            for (int w = 0; w < nw; w++) sum += red[w];
            double v = A[(int64_t)j * n + j] - sum;
            if (!(v > 0.0)) bad = 1;
            dsh = sqrt(v);
            A[(int64_t)j * n + j] = dsh;
        }
        __syncthreads();
        double d = dsh;
        for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
            double t = 0.0;
            for (int k = 0; k < j; k++) t = fma(A[(int64_t)i * n + k], A[(int64_t)j * n + k], t);
            A[(int64_t)i * n + j] = (A[(int64_t)i * n + j] - t) / d;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && bad) atomicMax(status + piece, (int)SC_NOT_SPD);
    // X = L^-1, column j by thread j
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        for (int i = 0; i < j; i++) X[(int64_t)i * n + j] = 0.0;
        X[(int64_t)j * n + j] = 1.0 / A[(int64_t)j * n + j];
        for (int i = j + 1; i < n; i++) {
            double t = 0.0;
            for (int k = j; k < i; k++) t = fma(A[(int64_t)i * n + k], X[(int64_t)k * n + j], t);
            X[(int64_t)i * n + j] = -t / A[(int64_t)i * n + i];
        }
    }
    __syncthreads();
    for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += blockDim.x) {
        int i = (int)(e / n), j = (int)(e % n);
        int k0 = i > j ? i : j;
        double t = 0.0;
        for (int k = k0; k < n; k++) t = fma(X[(int64_t)k * n + i], X[(int64_t)k * n + j], t);
        A[e] = t;
    }
}

// Every listed piece's top at once, one block per piece: A_all[off[i]..] holds the dense
// matrix on entry and its inverse on exit; X_all is scratch of the same layout.
__global__ void __launch_bounds__(1024) k_cholesky_inverse_all(const int32_t* __restrict__ top,
                                                               const int64_t* __restrict__ pstart,
                                                               const int64_t* __restrict__ off, double* A_all,
                                                               double* __restrict__ X_all,
                                                               int32_t* __restrict__ status) {
    int p = top[blockIdx.x];
    int n = (int)(6 * (pstart[p + 1] - pstart[p]));
    if (n == 0) return;
    cholesky_inverse_block(n, A_all + off[blockIdx.x], X_all + off[blockIdx.x], status, p);
}

// each piece's value of a per-part flag at its first part (0 where it has no part)
__global__ void k_first_flags(int np, const int64_t* __restrict__ pstart, const int32_t* __restrict__ flag,
                              int32_t* __restrict__ out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < np) out[p] = pstart[p] < pstart[p + 1] ? flag[pstart[p]] : 0;
}

__global__ void k_fill_i32(int64_t n, int32_t* __restrict__ a, int32_t v) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) a[i] = v;
}

__global__ void k_iota32(int64_t n, int32_t* __restrict__ v) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) v[i] = (int32_t)i;
}
__global__ void k_iota64(int64_t n, int64_t* __restrict__ v) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}
__global__ void k_row_of_entry(int64_t n, const int64_t* __restrict__ rowptr, int32_t* __restrict__ row) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    for (int64_t e = rowptr[k]; e < rowptr[k + 1]; e++) row[e] = (int32_t)k;
}

int bits_for(int64_t v) {
    int b = 1;
    while (b < 63 && (int64_t(1) << b) <= v) b++;
    return b;
}

int64_t d2h_i64(Context& ctx, const int64_t* p) {
    int64_t v = 0;
    SC_CK(cudaMemcpyAsync(&v, p, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx.stream));
    SC_CK(cudaStreamSynchronize(ctx.stream));
    return v;
}

void exclusive_scan(Context& ctx, const int64_t* in, int64_t* out, int64_t n) {
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, n, ctx.stream);
    cub::DeviceScan::ExclusiveSum(ctx.cub_scratch(tb), tb, in, out, n, ctx.stream);
}

// Keys (row << cb | col), cb = bits_for(ncols), sorted and made unique -> CSR pattern.
// The sort ping-pongs between `keys` and a second buffer (no copy of them in scratch).
void keys_to_csr(Context& ctx, DBuf<uint64_t>& keys, int64_t nkeys, int64_t nrows, int64_t ncols, DBuf<int64_t>& rowptr,
                 DBuf<int32_t>& col, int64_t& nnz) {
    cudaStream_t st = ctx.stream;
    MemStats* ms = &ctx.mem;
    const int cb = bits_for(ncols);
    DBuf<uint64_t> other;
    other.alloc(std::max<int64_t>(nkeys, 1), st, ms);
    int end_bit = cb + bits_for(nrows);
    size_t tb = 0;
    if (nkeys > 0) {
        cub::DoubleBuffer<uint64_t> dk(keys.get(), other.get());
        cub::DeviceRadixSort::SortKeys(nullptr, tb, dk, nkeys, 0, end_bit, st);
        cub::DeviceRadixSort::SortKeys(ctx.cub_scratch(tb), tb, dk, nkeys, 0, end_bit, st);
        if (dk.Current() != keys.get()) std::swap(keys, other);  // `keys` holds the sorted keys
    }
    other.release();
    DBuf<uint64_t> uniq;
    uniq.alloc(std::max<int64_t>(nkeys, 1), st, ms);
    DBuf<int64_t> nsel;
    nsel.alloc(1, st, ms);
    nsel.zero();
    if (nkeys > 0) {
        cub::DeviceSelect::Unique(nullptr, tb, keys.get(), uniq.get(), nsel.get(), nkeys, st);
        cub::DeviceSelect::Unique(ctx.cub_scratch(tb), tb, keys.get(), uniq.get(), nsel.get(), nkeys, st);
    }
    nnz = d2h_i64(ctx, nsel.get());
    keys.release();
    col.alloc(std::max<int64_t>(nnz, 1), st, ms);
    DBuf<int32_t> rows;
    rows.alloc(std::max<int64_t>(nnz, 1), st, ms);
    k_unpack_pattern<<<grid_for(nnz, 256), 256, 0, st>>>(nnz, uniq.get(), col.get(), rows.get(), cb);
    SC_LAUNCH_CK();
    rowptr.alloc(nrows + 1, st, ms);
    k_offsets_from_sorted<<<grid_for(nnz + 1, 256), 256, 0, st>>>(nnz, rows.get(), nrows, rowptr.get());
    SC_LAUNCH_CK();
}

__global__ void k_seg_flags(int64_t m, const uint64_t* __restrict__ keys, int64_t* __restrict__ flag) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= m) return;
    flag[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}
__global__ void k_seg_starts(int64_t m, const uint64_t* __restrict__ keys, const int64_t* __restrict__ flag,
                             const int64_t* __restrict__ idx, int64_t* __restrict__ seg, int32_t* __restrict__ col,
                             int32_t* __restrict__ row, int cb) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= m) return;
    if (flag[i]) {
        int64_t u = idx[i];
        seg[u] = i;
        col[u] = (int32_t)(keys[i] & ((uint64_t(1) << cb) - 1));
        row[u] = (int32_t)(keys[i] >> cb);
    }
}

// The same, keeping each candidate's contribution (a << 32 | b): the pattern in CSR,
// and for every stored block the range seg[q] .. seg[q+1] of its contributions in
// `vals` (sorted by output block, candidate order kept within one).
void keys_to_csr_with(Context& ctx, DBuf<uint64_t>& keys, DBuf<uint64_t>& vin, int64_t nkeys, int64_t nrows,
                      int64_t ncols, DBuf<int64_t>& rowptr, DBuf<int32_t>& col, int64_t& nnz, DBuf<int64_t>& seg,
                      DBuf<uint64_t>& vals) {
    cudaStream_t st = ctx.stream;
    MemStats* ms = &ctx.mem;
    const int cb = bits_for(ncols);
    DBuf<uint64_t> sorted;
    sorted.alloc(std::max<int64_t>(nkeys, 1), st, ms);
    vals.alloc(std::max<int64_t>(nkeys, 1), st, ms);
    int end_bit = cb + bits_for(nrows);
    size_t tb = 0;
    if (nkeys > 0) {
        // ping-pong between the inputs and the outputs (no copies in scratch); the sort
        // is stable, so each block's contributions keep their generation order
        cub::DoubleBuffer<uint64_t> dk(keys.get(), sorted.get()), dv(vin.get(), vals.get());
        cub::DeviceRadixSort::SortPairs(nullptr, tb, dk, dv, nkeys, 0, end_bit, st);
        cub::DeviceRadixSort::SortPairs(ctx.cub_scratch(tb), tb, dk, dv, nkeys, 0, end_bit, st);
        if (dk.Current() != sorted.get()) std::swap(keys, sorted);
        if (dv.Current() != vals.get()) std::swap(vin, vals);
    }
    keys.release();
    vin.release();
    DBuf<int64_t> flag, idx;
    flag.alloc(nkeys + 1, st, ms);
    idx.alloc(nkeys + 1, st, ms);
    SC_CK(cudaMemsetAsync(flag.get() + nkeys, 0, sizeof(int64_t), st));
    if (nkeys > 0) {
        k_seg_flags<<<grid_for(nkeys, 256), 256, 0, st>>>(nkeys, sorted.get(), flag.get());
        SC_LAUNCH_CK();
    }
    exclusive_scan(ctx, flag.get(), idx.get(), nkeys + 1);
    nnz = d2h_i64(ctx, idx.get() + nkeys);
    seg.alloc(nnz + 1, st, ms);
    col.alloc(std::max<int64_t>(nnz, 1), st, ms);
    DBuf<int32_t> rows;
    rows.alloc(std::max<int64_t>(nnz, 1), st, ms);
    if (nkeys > 0) {
        k_seg_starts<<<grid_for(nkeys, 256), 256, 0, st>>>(nkeys, sorted.get(), flag.get(), idx.get(), seg.get(),
                                                          col.get(), rows.get(), cb);
        SC_LAUNCH_CK();
    }
    SC_CK(cudaMemcpyAsync(seg.get() + nnz, &nkeys, sizeof(int64_t), cudaMemcpyHostToDevice, st));
    rowptr.alloc(nrows + 1, st, ms);
    k_offsets_from_sorted<<<grid_for(nnz + 1, 256), 256, 0, st>>>(nnz, rows.get(), nrows, rowptr.get());
    SC_LAUNCH_CK();
    SC_CK(cudaStreamSynchronize(st));  // nkeys (a host value) was copied asynchronously
}

}  // namespace

void setup_chunks(Context& ctx, Level& L, int32_t np) {
    std::vector<int64_t> lo;
    std::vector<int32_t> cp;
    std::vector<int64_t> pc(np + 1, 0);
    for (int p = 0; p < np; p++) {
        pc[p] = (int64_t)cp.size();
        for (int64_t a = L.pstart[p]; a < L.pstart[p + 1]; a += CHUNK) {
            lo.push_back(a);
            cp.push_back(p);
        }
    }
    pc[np] = (int64_t)cp.size();
    L.nchunks = (int64_t)cp.size();
    lo.push_back(L.n);
    L.chunk_lo.alloc(lo.size(), ctx.stream, &ctx.mem);
    L.chunk_lo.upload(lo.data(), lo.size());
    L.chunk_piece.alloc(std::max<size_t>(cp.size(), 1), ctx.stream, &ctx.mem);
    L.chunk_piece.upload(cp.data(), cp.size());
    L.piece_chunk.alloc(np + 1, ctx.stream, &ctx.mem);
    L.piece_chunk.upload(pc.data(), np + 1);
}

// The template view of a matrix-free level 0 during setup (all null otherwise).
static K0View k0_view(const Batch& b, const Level& L) {
    K0View v{};
    if (L.matrix_free && L.desc.size()) {
        const Grid0& g = b.grid;
        v = K0View{L.desc.get(), g.axis.get(), g.cella.get(), g.cellb.get(), g.cell.get(), g.tpl_s.get()};
    }
    return v;
}

static void invert_blocks_k0(Context& ctx, const Batch& b, Level& L, int32_t* status) {
    L.inv.alloc(36 * L.n, ctx.stream, &ctx.mem);
    k_diag_invert_k0<<<grid_for(L.n, 128), 128, 0, ctx.stream>>>(L.n, k0_view(b, L), L.inv.get(), L.piece.get(),
                                                                 status);
    SC_LAUNCH_CK();
}

void invert_blocks(Context& ctx, Level& L, int32_t* status) {
    L.inv.alloc(36 * L.n, ctx.stream, &ctx.mem);
    k_find_diag_invert<<<grid_for(L.n, 128), 128, 0, ctx.stream>>>(L.n, L.rowptr.get(), L.col.get(), L.val.get(),
                                                                   L.inv.get(), L.piece.get(), status);
    SC_LAUNCH_CK();
}

void invert_blocks(Context& ctx, Level& L) { invert_blocks(ctx, L, nullptr); }

// step = 4/3 / lambda_max(D^-1 K) per piece (bodies.rs:174, 180-190)
static void smoother_step(Context& ctx, Batch& b, int l) {
    Level& L = b.levels[l];
    cudaStream_t st = ctx.stream;
    int np = b.npieces;
    DBuf<double> v, w, t;
    v.alloc(6 * L.n, st, &ctx.mem);
    w.alloc(6 * L.n, st, &ctx.mem);
    t.alloc(6 * L.n, st, &ctx.mem);
    DBuf<double> ww, vv, most;
    ww.alloc(np, st, &ctx.mem);
    vv.alloc(np, st, &ctx.mem);
    most.alloc(np, st, &ctx.mem);
    k_power_start<<<grid_for(L.n, 256), 256, 0, st>>>(L.n, L.pstart_d.get(), L.piece.get(), v.get());
    SC_LAUNCH_CK();
    for (int it = 0; it < 12; it++) {
        level_apply<double>(ctx, b, l, v.get(), t.get());
        jacobi<double>(ctx, L.n, L.inv.get(), t.get(), w.get(), nullptr, L.piece.get(), nullptr, nullptr);
        seg_dot_t<double>(ctx, L, w.get(), w.get(), ww.get());
        seg_dot_t<double>(ctx, L, v.get(), v.get(), vv.get());
        k_power_most<<<grid_for(np, 128), 128, 0, st>>>(np, ww.get(), vv.get(), most.get());
        SC_LAUNCH_CK();
        k_power_scale<<<grid_for(6 * L.n, 256), 256, 0, st>>>(L.n, L.piece.get(), ww.get(), w.get(), v.get());
        SC_LAUNCH_CK();
    }
    L.step.alloc(np, st, &ctx.mem);
    k_step<<<grid_for(np, 128), 128, 0, st>>>(np, most.get(), L.step.get());
    SC_LAUNCH_CK();
}

void gather_i32(Context& ctx, int64_t n, const int64_t* idx, const int32_t* src, int32_t* dst);

// The next level from level l (bodies.rs:228-282); returns false when every piece tops
// out at level l.
static bool coarsen(Context& ctx, Batch& b, int l, int octree_level, const sc_options& opt) {
    cudaStream_t st = ctx.stream;
    MemStats* ms = &ctx.mem;
    int np = b.npieces;
    Level& F = b.levels[l];
    int64_t n = F.n;
    PhaseTimer pt(ctx);
    // which pieces go on: more than FEW parts (bodies.rs:447)
    std::vector<int32_t> active(np, 0);
    for (int p = 0; p < np; p++) active[p] = (F.pstart[p + 1] - F.pstart[p]) > opt.few ? 1 : 0;
    DBuf<int32_t> active_d;
    active_d.alloc(np, st, ms);
    active_d.upload(active.data(), np);
    // bodies_of (bodies.rs:472-496)
    int64_t mask = ~((int64_t(1) << octree_level) - 1);
    DBuf<int32_t> label;
    label.alloc(n, st, ms);
    k_label_init<<<grid_for(n, 256), 256, 0, st>>>(n, label.get());
    SC_LAUNCH_CK();
    DBuf<int32_t> changed;
    changed.alloc(1, st, ms);
    for (int it = 0; it < 100000; it++) {
        changed.zero();
        k_label_sweep<<<grid_for(n, 256), 256, 0, st>>>(n, F.rowptr.get(), F.col.get(), F.site.get(), mask,
                                                        active_d.get(), F.piece.get(), label.get(), changed.get());
        SC_LAUNCH_CK();
        k_label_jump<<<grid_for(n, 256), 256, 0, st>>>(n, label.get());
        SC_LAUNCH_CK();
        int32_t ch = 0;
        SC_CK(cudaMemcpyAsync(&ch, changed.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        SC_CK(cudaStreamSynchronize(st));
        if (!ch) break;
    }
    DBuf<int64_t> root, id;
    root.alloc(n + 1, st, ms);
    id.alloc(n + 1, st, ms);
    DBuf<int32_t> bodies_d;
    bodies_d.alloc(np, st, ms);
    bodies_d.zero();
    SC_CK(cudaMemsetAsync(root.get() + n, 0, sizeof(int64_t), st));
    k_roots<<<grid_for(n, 256), 256, 0, st>>>(n, label.get(), F.piece.get(), root.get(), bodies_d.get());
    SC_LAUNCH_CK();
    std::vector<int32_t> bodies = bodies_d.to_host();
    bool any = false;
    for (int p = 0; p < np; p++) {
        if (active[p] && bodies[p] == (int32_t)(F.pstart[p + 1] - F.pstart[p])) active[p] = 0;  // bodies.rs:453-455
        any = any || active[p];
    }
    F.top_of_part.alloc(n, st, ms);
    F.up.alloc(n, st, ms);
    if (!any) {
        k_fill_i32<<<grid_for(n, 256), 256, 0, st>>>(n, F.top_of_part.get(), 1);
        k_fill_i32<<<grid_for(n, 256), 256, 0, st>>>(n, F.up.get(), -1);
        SC_LAUNCH_CK();
        return false;
    }
    active_d.upload(active.data(), np);
    k_mask_roots<<<grid_for(n, 256), 256, 0, st>>>(n, F.piece.get(), active_d.get(), root.get());
    SC_LAUNCH_CK();
    exclusive_scan(ctx, root.get(), id.get(), n + 1);
    int64_t nc = d2h_i64(ctx, id.get() + n);
    k_up<<<grid_for(n, 256), 256, 0, st>>>(n, label.get(), id.get(), F.piece.get(), active_d.get(), F.up.get(),
                                           F.top_of_part.get());
    SC_LAUNCH_CK();
    label.release();
    root.release();
    id.release();
    pt.mark("  bodies");

    Level C;
    C.n = nc;
    C.pstart.assign(np + 1, 0);
    for (int p = 0; p < np; p++) C.pstart[p + 1] = C.pstart[p] + (active[p] ? bodies[p] : 0);
    C.pstart_d.alloc(np + 1, st, ms);
    C.pstart_d.upload(C.pstart.data(), np + 1);
    // members of each body in part order (stable sort by body)
    DBuf<int32_t> mem_part, mem_body;
    {
        DBuf<int32_t> ids;
        ids.alloc(n, st, ms);
        k_iota32<<<grid_for(n, 256), 256, 0, st>>>(n, ids.get());
        SC_LAUNCH_CK();
        DBuf<int32_t> keys_in;
        keys_in.alloc(n, st, ms);
        // parts of stopped pieces (up = -1) sort first as 0xffffffff... use unsigned keys
        SC_CK(cudaMemcpyAsync(keys_in.get(), F.up.get(), n * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
        mem_part.alloc(n, st, ms);
        mem_body.alloc(n, st, ms);
        size_t tb = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, (uint32_t*)keys_in.get(), (uint32_t*)mem_body.get(), ids.get(),
                                        mem_part.get(), n, 0, 32, st);
        cub::DeviceRadixSort::SortPairs(ctx.cub_scratch(tb), tb, (uint32_t*)keys_in.get(), (uint32_t*)mem_body.get(),
                                        ids.get(), mem_part.get(), n, 0, 32, st);
    }
    // active parts are the first m entries (up < 2^31 sorts below 0xffffffff)
    int64_t m = 0;
    for (int p = 0; p < np; p++)
        if (active[p]) m += F.pstart[p + 1] - F.pstart[p];
    DBuf<int64_t> moff;
    moff.alloc(nc + 1, st, ms);
    k_offsets_from_sorted<<<grid_for(m + 1, 256), 256, 0, st>>>(m, mem_body.get(), nc, moff.get());
    SC_LAUNCH_CK();
    C.centre.alloc(3 * nc, st, ms);
    C.site.alloc(3 * nc, st, ms);
    C.piece.alloc(nc, st, ms);
    k_centroid<<<grid_for(nc, 128), 128, 0, st>>>(nc, moff.get(), mem_part.get(), F.centre.get(), F.site.get(),
                                                  F.piece.get(), C.centre.get(), C.site.get(), C.piece.get());
    SC_LAUNCH_CK();
    mem_body.release();
    DBuf<double> rvec;
    rvec.alloc(3 * n, st, ms);
    k_rvec<<<grid_for(n, 256), 256, 0, st>>>(n, F.up.get(), F.centre.get(), C.centre.get(), rvec.get());
    SC_LAUNCH_CK();
    bool keep_mf = l == 0 && F.matrix_free;
    pt.mark("  members, centroids");

    // --- P pattern and values
    DBuf<int64_t> cnt, off;
    cnt.alloc(n + 1, st, ms);
    off.alloc(n + 1, st, ms);
    SC_CK(cudaMemsetAsync(cnt.get() + n, 0, sizeof(int64_t), st));
    k_count_P<<<grid_for(n, 256), 256, 0, st>>>(n, F.rowptr.get(), F.up.get(), cnt.get());
    SC_LAUNCH_CK();
    exclusive_scan(ctx, cnt.get(), off.get(), n + 1);
    int64_t tot = d2h_i64(ctx, off.get() + n);
    {
        DBuf<uint64_t> keys;
        keys.alloc(std::max<int64_t>(tot, 1), st, ms);
        k_fill_P<<<grid_for(n, 256), 256, 0, st>>>(n, F.rowptr.get(), F.col.get(), F.up.get(), off.get(), keys.get(),
                                                   bits_for(nc));
        SC_LAUNCH_CK();
        keys_to_csr(ctx, keys, tot, n, nc, F.prow, F.pcol, F.pnnz);
    }
    cnt.release();
    off.release();
    F.pval.alloc(36 * std::max<int64_t>(F.pnnz, 1), st, ms);
    F.pval.zero();
    const K0View k0 = k0_view(b, F);
    const bool virt = k0.desc != nullptr;  // level-0 blocks made from the cell template
    if (virt)
        k_num_P<true><<<grid_for(n * 32, 256), 256, 0, st>>>(n, F.rowptr.get(), F.col.get(), nullptr, k0, F.up.get(),
                                                             rvec.get(), F.inv.get(), F.step.get(), F.piece.get(),
                                                             F.prow.get(), F.pcol.get(), F.pval.get());
    else
        k_num_P<false><<<grid_for(n * 32, 256), 256, 0, st>>>(n, F.rowptr.get(), F.col.get(), F.val.get(), k0,
                                                              F.up.get(), rvec.get(), F.inv.get(), F.step.get(),
                                                              F.piece.get(), F.prow.get(), F.pcol.get(), F.pval.get());
    SC_LAUNCH_CK();
    if (keep_mf) {
        F.mf_r = std::move(rvec);
        F.mem_off = std::move(moff);
        F.mem = std::move(mem_part);
    } else {
        rvec.release();
        moff.release();
        mem_part.release();
    }
    // P transposed: entries sorted by column, stable (fine-row order within a column)
    DBuf<int32_t> prow_of;  // the row of each P entry
    prow_of.alloc(std::max<int64_t>(F.pnnz, 1), st, ms);
    k_row_of_entry<<<grid_for(n, 256), 256, 0, st>>>(n, F.prow.get(), prow_of.get());
    SC_LAUNCH_CK();
    {
        DBuf<int64_t> ent;
        ent.alloc(std::max<int64_t>(F.pnnz, 1), st, ms);
        k_iota64<<<grid_for(F.pnnz, 256), 256, 0, st>>>(F.pnnz, ent.get());
        SC_LAUNCH_CK();
        DBuf<int32_t> ccol;
        ccol.alloc(std::max<int64_t>(F.pnnz, 1), st, ms);
        F.tent.alloc(std::max<int64_t>(F.pnnz, 1), st, ms);
        size_t tb = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, F.pcol.get(), ccol.get(), ent.get(), F.tent.get(), F.pnnz, 0,
                                        bits_for(nc), st);
        cub::DeviceRadixSort::SortPairs(ctx.cub_scratch(tb), tb, F.pcol.get(), ccol.get(), ent.get(), F.tent.get(),
                                        F.pnnz, 0, bits_for(nc), st);
        F.tptr.alloc(nc + 1, st, ms);
        k_offsets_from_sorted<<<grid_for(F.pnnz + 1, 256), 256, 0, st>>>(F.pnnz, ccol.get(), nc, F.tptr.get());
        SC_LAUNCH_CK();
        F.trow.alloc(std::max<int64_t>(F.pnnz, 1), st, ms);
        // trow[t] = row of entry tent[t]
        gather_i32(ctx, F.pnnz, F.tent.get(), prow_of.get(), F.trow.get());
    }
    // the restriction's blocks, contiguous by coarse row (a matrix-free level 0 needs none)
    if (!keep_mf) {
        F.ptval.alloc(36 * std::max<int64_t>(F.pnnz, 1), st, ms);
        k_transpose_gather<<<grid_for(36 * F.pnnz, 256), 256, 0, st>>>(F.pnnz, F.tent.get(), F.pval.get(),
                                                                       F.ptval.get());
        SC_LAUNCH_CK();
    }
    pt.mark("  prolongator");
    // A product goes row by row (rowprod.cuh) when every piece's coarse level fits the
    // bitmap window and B's rows are long enough to keep a block's 32 groups busy (eight
    // blocks a row or more: levels 1 and up of voxel pieces), else through sorted
    // candidate lists. Both give the same bits; SC_GALERKIN=sort or =rows forces one
    // (rows only where the window fits).
    int64_t widest = 0;
    for (int p = 0; p < np; p++) widest = std::max<int64_t>(widest, C.pstart[p + 1] - C.pstart[p]);
    const char* gal_env = std::getenv("SC_GALERKIN");
    const std::string gal = gal_env ? gal_env : "";
    const bool fits = widest <= ROWS_MAX_WIDTH && gal != "sort";
    const bool by_rows = fits && (gal == "rows" || F.pnnz >= 8 * n);
    // --- K P
    DBuf<int64_t> kprow;
    DBuf<int32_t> kpcol;
    int64_t kpnnz = 0, kp_cands = 0, c_cands = 0;
    DBuf<double> kpval;
    // Under SC_MIXED the V-cycle reads the coarse operators in FP32 only, so a matrix-free
    // level 0's K P blocks (the largest array of the setup: 27.5 M blocks at 128^3) are
    // held in FP32 where both products go through sorted sums; P'(KP) still adds in FP64.
    DBuf<float> kpval32;
    bool kp32 = false;
    if (by_rows) {
        DBuf<int32_t> lo, hi;
        lo.alloc(n, st, ms);
        hi.alloc(n, st, ms);
        kp_windows(ctx, n, F.up.get(), F.prow.get(), F.pcol.get(), F.piece.get(), C.pstart_d.get(), lo.get(), hi.get());
        RowArgs a{};
        a.arow = F.rowptr.get();
        a.acol = F.col.get();
        a.aval = virt ? nullptr : F.val.get();
        a.k0 = k0;
        a.annz = F.nnzb;
        a.brow = F.prow.get();
        a.bcol = F.pcol.get();
        a.bval = F.pval.get();
        a.lo = lo.get();
        a.hi = hi.get();
        row_products(ctx, virt ? ROWS_K0 : ROWS_PLAIN, a, n, widest, kprow, kpcol, kpval, kpnnz, kp_cands);
    } else {
        // one thread per block of K (its row from krow), offsets by a scan over K's entries
        const int64_t knz = F.nnzb;
        DBuf<int32_t> krow;
        DBuf<int64_t> kcnt, koff;
        krow.alloc(std::max<int64_t>(knz, 1), st, ms);
        kcnt.alloc(knz + 1, st, ms);
        koff.alloc(knz + 1, st, ms);
        k_row_of_entry<<<grid_for(n, 256), 256, 0, st>>>(n, F.rowptr.get(), krow.get());
        SC_LAUNCH_CK();
        SC_CK(cudaMemsetAsync(kcnt.get() + knz, 0, sizeof(int64_t), st));
        if (knz > 0) {
            k_count_KP<<<grid_for(knz, 256), 256, 0, st>>>(knz, krow.get(), F.col.get(), F.prow.get(), F.pcol.get(),
                                                          F.up.get(), kcnt.get());
            SC_LAUNCH_CK();
        }
        exclusive_scan(ctx, kcnt.get(), koff.get(), knz + 1);
        tot = d2h_i64(ctx, koff.get() + knz);
        kp_cands = tot;
        kcnt.release();
        DBuf<uint64_t> keys, vin, vals;
        DBuf<int64_t> seg;
        keys.alloc(std::max<int64_t>(tot, 1), st, ms);
        vin.alloc(std::max<int64_t>(tot, 1), st, ms);
        if (knz > 0) {
            k_fill_KP<<<grid_for(knz, 256), 256, 0, st>>>(knz, krow.get(), F.col.get(), F.prow.get(), F.pcol.get(),
                                                         F.up.get(), koff.get(), keys.get(), vin.get(), bits_for(nc));
            SC_LAUNCH_CK();
        }
        koff.release();
        keys_to_csr_with(ctx, keys, vin, tot, n, nc, kprow, kpcol, kpnnz, seg, vals);
        kp32 = virt && opt.precision == SC_MIXED && !(fits && (gal == "rows" || kpnnz >= 12 * n));
        if (kp32) {
            // P too: both products read it, nothing after them (a matrix-free level 0
            // transfers through its rigid part and the stencil)
            to_float(ctx, F.pval, F.pval32);
            F.pval.release();
            kpval32.alloc(36 * std::max<int64_t>(kpnnz, 1), st, ms);
        } else {
            kpval.alloc(36 * std::max<int64_t>(kpnnz, 1), st, ms);
        }
        if (kpnnz > 0) {
            unsigned nb = (unsigned)((kpnnz + SUM_GROUPS - 1) / SUM_GROUPS);
            const unsigned nb0 = std::min((unsigned)((kpnnz + K0SUM_GROUPS - 1) / K0SUM_GROUPS), 148u * 8u);
            if (virt && kp32)
                k_sum_products_k0<float, float><<<nb0, 32 * K0SUM_WARPS, 0, st>>>(
                    kpnnz, seg.get(), vals.get(), F.pval32.get(), kpval32.get(), k0, krow.get());
            else if (virt)
                k_sum_products_k0<double, double><<<nb0, 32 * K0SUM_WARPS, 0, st>>>(
                    kpnnz, seg.get(), vals.get(), F.pval.get(), kpval.get(), k0, krow.get());
            else
                k_sum_products<false, double, double><<<nb, SUM_THREADS, 0, st>>>(
                    kpnnz, seg.get(), vals.get(), F.val.get(), F.pval.get(), kpval.get());
            SC_LAUNCH_CK();
        }
    }
    pt.mark("  K P");
    // --- P' K P, upper triangle (d >= c)
    DBuf<int64_t> urow;
    DBuf<int32_t> ucol;
    DBuf<double> uval;
    int64_t unnz = 0;
    // the upper product's rows see about half of each K P row
    if (fits && (gal == "rows" || kpnnz >= 12 * n)) {
        DBuf<int32_t> lo, hi;
        lo.alloc(nc, st, ms);
        hi.alloc(nc, st, ms);
        upper_windows(ctx, nc, C.piece.get(), C.pstart_d.get(), lo.get(), hi.get());
        RowArgs a{};
        a.arow = F.tptr.get();
        a.acol = F.trow.get();
        a.aent = F.tent.get();
        a.aval = F.pval.get();
        a.annz = F.pnnz;
        a.brow = kprow.get();
        a.bcol = kpcol.get();
        a.bval = kpval.get();
        a.lo = lo.get();
        a.hi = hi.get();
        row_products(ctx, ROWS_TRANSPOSED, a, nc, widest, urow, ucol, uval, unnz, c_cands);
    } else {
        DBuf<int64_t> ecnt, eoff;
        ecnt.alloc(F.pnnz + 1, st, ms);
        eoff.alloc(F.pnnz + 1, st, ms);
        SC_CK(cudaMemsetAsync(ecnt.get() + F.pnnz, 0, sizeof(int64_t), st));
        if (F.pnnz > 0) {
            k_count_C<<<grid_for(F.pnnz, 256), 256, 0, st>>>(F.pnnz, prow_of.get(), F.pcol.get(), kprow.get(),
                                                             kpcol.get(), ecnt.get());
            SC_LAUNCH_CK();
        }
        exclusive_scan(ctx, ecnt.get(), eoff.get(), F.pnnz + 1);
        tot = d2h_i64(ctx, eoff.get() + F.pnnz);
        c_cands = tot;
        eoff.release();
        const int cbc = bits_for(nc);
        // One slice of coarse rows [c0, c1): its candidates made, sorted and summed into
        // its own rows (rp: the slice's entries before each row), columns and blocks.
        auto upper_slice = [&](int32_t c0, int32_t c1, DBuf<int64_t>& rp, DBuf<int32_t>& cl, int64_t& nn,
                               DBuf<double>& vv) {
            DBuf<int64_t> scnt, soff;
            const int64_t* cnt = ecnt.get();
            if (c0 > 0 || c1 < nc) {
                scnt.alloc(F.pnnz + 1, st, ms);
                SC_CK(cudaMemsetAsync(scnt.get() + F.pnnz, 0, sizeof(int64_t), st));
                if (F.pnnz > 0) {
                    k_slice_counts<<<grid_for(F.pnnz, 256), 256, 0, st>>>(F.pnnz, F.pcol.get(), ecnt.get(), c0, c1,
                                                                          scnt.get());
                    SC_LAUNCH_CK();
                }
                cnt = scnt.get();
            }
            soff.alloc(F.pnnz + 1, st, ms);
            exclusive_scan(ctx, cnt, soff.get(), F.pnnz + 1);
            const int64_t ns = d2h_i64(ctx, soff.get() + F.pnnz);
            DBuf<uint64_t> keys, vin, vals;
            DBuf<int64_t> seg;
            keys.alloc(std::max<int64_t>(ns, 1), st, ms);
            vin.alloc(std::max<int64_t>(ns, 1), st, ms);
            if (F.pnnz > 0) {
                k_fill_C<<<grid_for(F.pnnz, 256), 256, 0, st>>>(F.pnnz, prow_of.get(), F.pcol.get(), kprow.get(),
                                                                kpcol.get(), soff.get(), keys.get(), vin.get(), cbc,
                                                                c0, c1);
                SC_LAUNCH_CK();
            }
            scnt.release();
            soff.release();
            keys_to_csr_with(ctx, keys, vin, ns, nc, nc, rp, cl, nn, seg, vals);
            vv.alloc(36 * std::max<int64_t>(nn, 1), st, ms);
            if (nn > 0) {
                const unsigned nbu = (unsigned)((nn + SUM_GROUPS - 1) / SUM_GROUPS);
                if (kp32)
                    k_sum_products<true, float, float><<<nbu, SUM_THREADS, 0, st>>>(
                        nn, seg.get(), vals.get(), F.pval32.get(), kpval32.get(), vv.get());
                else
                    k_sum_products<true, double, double><<<nbu, SUM_THREADS, 0, st>>>(
                        nn, seg.get(), vals.get(), F.pval.get(), kpval.get(), vv.get());
                SC_LAUNCH_CK();
            }
        };
        // All at once, or, where the candidates are many, in slices of coarse rows of at
        // most `slice` candidates each: every output block's candidates are the same and in
        // the same order either way (the same bits), and a slice's lists are gone before
        // the next one's are made. SC_UPPER_SLICE lowers the limit (to test the slices).
        int64_t slice = 96LL << 20;
        if (const char* v = std::getenv("SC_UPPER_SLICE")) slice = std::max<int64_t>(1, std::atoll(v));
        if (tot <= slice) {
            upper_slice(0, (int32_t)nc, urow, ucol, unnz, uval);
        } else {
            DBuf<int64_t> rc;
            rc.alloc(nc + 1, st, ms);
            rc.zero();
            if (F.pnnz > 0) {
                k_row_cands<<<grid_for(F.pnnz, 256), 256, 0, st>>>(F.pnnz, F.pcol.get(), ecnt.get(), rc.get());
                SC_LAUNCH_CK();
            }
            const std::vector<int64_t> rch = rc.to_host();
            std::vector<std::pair<int32_t, int32_t>> sl;
            int32_t c0 = 0;
            int64_t acc = 0;
            for (int32_t c = 0; c < (int32_t)nc; c++) {
                if (c > c0 && acc + rch[c] > slice) {
                    sl.push_back({c0, c});
                    c0 = c;
                    acc = 0;
                }
                acc += rch[c];
            }
            sl.push_back({c0, (int32_t)nc});
            urow.alloc(nc + 1, st, ms);
            urow.zero();
            std::vector<DBuf<int32_t>> cols(sl.size());
            std::vector<DBuf<double>> vls(sl.size());
            std::vector<int64_t> nns(sl.size(), 0);
            for (size_t i = 0; i < sl.size(); i++) {
                DBuf<int64_t> rp;
                upper_slice(sl[i].first, sl[i].second, rp, cols[i], nns[i], vls[i]);
                k_add_i64<<<grid_for(nc + 1, 256), 256, 0, st>>>(nc + 1, urow.get(), rp.get());
                SC_LAUNCH_CK();
            }
            kpval.release();  // the products are done
            kpval32.release();
            unnz = 0;
            for (int64_t v : nns) unnz += v;
            ucol.alloc(std::max<int64_t>(unnz, 1), st, ms);
            uval.alloc(36 * std::max<int64_t>(unnz, 1), st, ms);
            int64_t o = 0;
            for (size_t i = 0; i < sl.size(); i++) {
                if (nns[i] > 0) {
                    SC_CK(cudaMemcpyAsync(ucol.get() + o, cols[i].get(), nns[i] * sizeof(int32_t),
                                          cudaMemcpyDeviceToDevice, st));
                    SC_CK(cudaMemcpyAsync(uval.get() + 36 * o, vls[i].get(), 36 * nns[i] * sizeof(double),
                                          cudaMemcpyDeviceToDevice, st));
                }
                o += nns[i];
                cols[i].release();
                vls[i].release();
            }
        }
    }
    kpval.release();
    kpval32.release();
    kprow.release();
    kpcol.release();
    prow_of.release();
    pt.mark("  P' K P");
    pt.note("  sizes: rows %lld blocks %lld P %lld KP cands %lld KP %lld C cands %lld C upper %lld", (long long)n,
            (long long)F.nnzb, (long long)F.pnnz, (long long)kp_cands, (long long)kpnnz, (long long)c_cands,
            (long long)unnz);
    // --- full symmetric storage
    {
        DBuf<int32_t> urows;
        urows.alloc(std::max<int64_t>(unnz, 1), st, ms);
        k_row_of_entry<<<grid_for(nc, 256), 256, 0, st>>>(nc, urow.get(), urows.get());
        SC_LAUNCH_CK();
        DBuf<int64_t> mc, mo;
        mc.alloc(unnz + 1, st, ms);
        mo.alloc(unnz + 1, st, ms);
        SC_CK(cudaMemsetAsync(mc.get() + unnz, 0, sizeof(int64_t), st));
        k_mirror_count<<<grid_for(unnz, 256), 256, 0, st>>>(unnz, urows.get(), ucol.get(), mc.get());
        SC_LAUNCH_CK();
        exclusive_scan(ctx, mc.get(), mo.get(), unnz + 1);
        int64_t fn = d2h_i64(ctx, mo.get() + unnz);
        DBuf<uint64_t> keys, keys_s;
        DBuf<int64_t> src, src_s;
        keys.alloc(fn, st, ms);
        src.alloc(fn, st, ms);
        k_mirror_keys<<<grid_for(unnz, 256), 256, 0, st>>>(unnz, urows.get(), ucol.get(), keys.get(), src.get(), mo.get());
        SC_LAUNCH_CK();
        keys_s.alloc(fn, st, ms);
        src_s.alloc(fn, st, ms);
        size_t tb = 0;
        int end_bit = 32 + bits_for(nc);
        cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.get(), keys_s.get(), src.get(), src_s.get(), fn, 0, end_bit, st);
        cub::DeviceRadixSort::SortPairs(ctx.cub_scratch(tb), tb, keys.get(), keys_s.get(), src.get(), src_s.get(), fn, 0,
                                        end_bit, st);
        keys.release();
        src.release();
        C.nnzb = fn;
        C.col.alloc(fn, st, ms);
        DBuf<int32_t> rows;
        rows.alloc(fn, st, ms);
        k_unpack_pattern<<<grid_for(fn, 256), 256, 0, st>>>(fn, keys_s.get(), C.col.get(), rows.get(), 32);
        SC_LAUNCH_CK();
        C.rowptr.alloc(nc + 1, st, ms);
        k_offsets_from_sorted<<<grid_for(fn + 1, 256), 256, 0, st>>>(fn, rows.get(), nc, C.rowptr.get());
        SC_LAUNCH_CK();
        C.val.alloc(36 * fn, st, ms);
        k_mirror_vals<<<grid_for(36 * fn, 256), 256, 0, st>>>(fn, src_s.get(), uval.get(), C.val.get());
        SC_LAUNCH_CK();
    }
    pt.mark("  mirror");
    b.levels.push_back(std::move(C));
    return true;
}

void gather_i32(Context& ctx, int64_t n, const int64_t* idx, const int32_t* src, int32_t* dst);

static void build_top(Context& ctx, Batch& b, int l, const std::vector<int32_t>& pieces) {
    Level& L = b.levels[l];
    cudaStream_t st = ctx.stream;
    L.top_h = pieces;
    if (pieces.empty()) return;
    L.top.alloc(pieces.size(), st, &ctx.mem);
    L.top.upload(pieces.data(), pieces.size());
    std::vector<int64_t> off(pieces.size() + 1, 0);
    for (size_t i = 0; i < pieces.size(); i++) {
        int64_t nn = 6 * (L.pstart[pieces[i] + 1] - L.pstart[pieces[i]]);
        off[i + 1] = off[i] + nn * nn;
    }
    L.kinv_off.alloc(off.size(), st, &ctx.mem);
    L.kinv_off.upload(off.data(), off.size());
    L.kinv.alloc(std::max<int64_t>(off.back(), 1), st, &ctx.mem);
    // all tops factored together, one block per piece, the inverse written in place
    SC_CK(cudaMemsetAsync(L.kinv.get(), 0, std::max<int64_t>(off.back(), 1) * sizeof(double), st));
    DBuf<double> X;
    X.alloc(std::max<int64_t>(off.back(), 1), st, &ctx.mem);
    unsigned nt = (unsigned)pieces.size();
    for (unsigned first = 0; first < nt; first += 65535u) {  // gridDim.y <= 65535
        unsigned m = std::min(nt - first, 65535u);
        const K0View k0 = k0_view(b, L);
        if (k0.desc)
            k_dense_from_bsr_all<true><<<dim3(64, m), 64, 0, st>>>(L.top.get() + first, L.pstart_d.get(),
                                                                   L.rowptr.get(), L.col.get(), nullptr, k0,
                                                                   L.kinv_off.get() + first, L.kinv.get());
        else
            k_dense_from_bsr_all<false><<<dim3(64, m), 64, 0, st>>>(L.top.get() + first, L.pstart_d.get(),
                                                                    L.rowptr.get(), L.col.get(), L.val.get(), k0,
                                                                    L.kinv_off.get() + first, L.kinv.get());
        SC_LAUNCH_CK();
    }
    k_cholesky_inverse_all<<<nt, 1024, 0, st>>>(L.top.get(), L.pstart_d.get(), L.kinv_off.get(), L.kinv.get(),
                                                 X.get(), b.status_d.get());
    SC_LAUNCH_CK();
}

template <class T>
__global__ void k_gather(int64_t n, const int64_t* __restrict__ idx, const T* __restrict__ src, T* __restrict__ dst) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[idx[i]];
}
void gather_i32(Context& ctx, int64_t n, const int64_t* idx, const int32_t* src, int32_t* dst) {
    if (n <= 0) return;
    k_gather<int32_t><<<grid_for(n, 256), 256, 0, ctx.stream>>>(n, idx, src, dst);
    SC_LAUNCH_CK();
}

void to_float(Context& ctx, const DBuf<double>& a, DBuf<float>& b) {
    b.alloc(a.size(), ctx.stream, &ctx.mem);
    if (a.size()) {
        k_to_float<<<grid_for((int64_t)a.size(), 256), 256, 0, ctx.stream>>>((int64_t)a.size(), a.get(), b.get());
        SC_LAUNCH_CK();
    }
}

// Levels for every piece: while a piece has more than FEW parts and its bodies are fewer
// than its parts, coarsen it (bodies.rs:444-461); then factor each piece's top.
// A matrix-free level 0 keeps only what the solve reads: the assembled blocks, their
// inverses and the explicit prolongator serve the setup alone.
static void release_level0_setup(Batch& b) {
    if (!b.levels[0].matrix_free || b.levels.size() < 2) return;
    Level& L0 = b.levels[0];
    L0.val.release();
    L0.desc.release();
    b.grid.tpl_s.release();
    L0.col.release();
    L0.rowptr.release();
    L0.inv.release();
    L0.pval.release();
    L0.pval32.release();
    L0.pcol.release();
    L0.prow.release();
    L0.tptr.release();
    L0.tent.release();
    L0.trow.release();
}

void build_hierarchy(Context& ctx, Batch& b, const sc_options& opt) {
    auto t0 = std::chrono::steady_clock::now();
    PhaseTimer pt(ctx);
    int np = b.npieces;
    b.levels.reserve(SC_MAX_LEVELS + 1);
    b.status_d.alloc(np, ctx.stream, &ctx.mem);
    b.status_d.zero();
    int octree = b.base_level;
    for (int l = 0;; l++) {
        Level& L = b.levels[l];
        setup_chunks(ctx, L, np);
        if (L.matrix_free && L.desc.size())
            invert_blocks_k0(ctx, b, L, b.status_d.get());
        else
            invert_blocks(ctx, L, b.status_d.get());
        pt.mark("chunks + inverses");
        smoother_step(ctx, b, l);
        pt.mark("smoother step");
        octree += 1;
        bool more = l + 1 < SC_MAX_LEVELS && coarsen(ctx, b, l, octree, opt);
        pt.mark("coarsen");
        Level& F = b.levels[l];  // reference may have moved
        // pieces whose top is this level (each piece's flag read at its first part)
        std::vector<int32_t> tops;
        {
            std::vector<int32_t> topp;
            if (F.top_of_part.size() && np > 0) {
                DBuf<int32_t> first;
                first.alloc(np, ctx.stream, &ctx.mem);
                k_first_flags<<<grid_for(np, 128), 128, 0, ctx.stream>>>(np, F.pstart_d.get(), F.top_of_part.get(),
                                                                       first.get());
                SC_LAUNCH_CK();
                topp = first.to_host();
            }
            for (int p = 0; p < np; p++) {
                int64_t a = F.pstart[p], e = F.pstart[p + 1];
                if (a == e) continue;  // not on this level
                bool top = !more || topp.empty() || topp[p];
                if (top) tops.push_back(p);
            }
        }
        build_top(ctx, b, l, tops);
        pt.mark("tops");
        // Level l is finished: the levels above it are made from their own operators. Its
        // setup-only arrays go now rather than at the end, so the next products run with
        // less memory held. Under SC_MIXED the V-cycle reads a coarse level's operator,
        // inverses and transfers in FP32 only (the FP64 conjugate gradients read level 0
        // alone), so a coarse level keeps just those.
        if (l == 0) release_level0_setup(b);
        if (l >= 1 && opt.precision == SC_MIXED) {
            Level& D = b.levels[l];
            to_float(ctx, D.val, D.val32);
            to_float(ctx, D.inv, D.inv32);
            if (D.pval.size()) to_float(ctx, D.pval, D.pval32);
            if (D.ptval.size()) to_float(ctx, D.ptval, D.ptval32);
            D.val.release();
            D.inv.release();
            D.pval.release();
            D.ptval.release();
        }
        pt.mark("release");
        if (!more) break;
    }
    b.piece_levels.assign(np, 0);
    for (size_t l = 0; l < b.levels.size(); l++)
        for (int p = 0; p < np; p++)
            if (b.levels[l].pstart[p + 1] > b.levels[l].pstart[p]) b.piece_levels[p] = (int32_t)l + 1;
    SC_CK(cudaStreamSynchronize(ctx.stream));
    b.setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace sc
