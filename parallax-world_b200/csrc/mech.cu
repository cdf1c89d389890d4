// The engine's solver, mechanics::solve::Solver (mechanics/src/solve.rs:356-538), on the
// device. Its levels (Solver::new, solve.rs:241-271, 361-386: rigid aggregates of the parts
// joined within each octree cell a level up, their Galerkin blocks T(r)' M T(s), block
// inverses by Cholesky with dropped pivots, the turn regularisation, the smoother step by
// ten power steps, a direct top) are made on the device by mech_levels.cu and kept there
// as block-sparse rows (3x3 at the cells' nodes, 6x6 above, both triangles). This file
// keeps a host copy of that construction (sc_mech_levels, no device) and runs the
// conjugate gradients and V-cycles (solve.rs:403-538) as a device-side loop: block
// products, block-Jacobi smoothing, the rigid restriction and prolongation, the top's
// dense inverse, and deterministic dot products. Coarse pairs are kept in (a, c) order (the reference
// collects them from a hash map, solve.rs:249-262): sums over pairs add in another order,
// equal up to rounding.
#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "kernels.cuh"
#include "mech.cuh"

namespace sc {

namespace {

typedef std::array<double, 3> H3;
typedef std::array<H3, 3> HM3;
typedef std::array<double, 6> H6;
typedef std::array<H6, 6> HM6;

constexpr int MECH_ROUNDS = 300;  // solve.rs:21

// ---- the levels, on the host ------------------------------------------------------
struct HPair {
    uint32_t i, j;
    HM6 m;
};

struct HSys {  // the system with its blocks embedded as 6x6 (solve.rs:97-103)
    std::vector<std::array<int64_t, 3>> keys;
    std::vector<H3> at;
    std::vector<HM6> diag;
    std::vector<HPair> pairs;
};

HM6 lift6(const HM6& m, const H3& r, const H3& s) {  // solve.rs:77-94
    auto X = [](const H3& v) { return HM3{H3{0.0, v[2], -v[1]}, H3{-v[2], 0.0, v[0]}, H3{v[1], -v[0], 0.0}}; };
    const HM3 xr = X(r), xs = X(s);
    HM6 t = m;
    for (int row = 0; row < 6; row++)
        for (int c = 0; c < 3; c++) {
            double acc = 0.0;
            for (int k = 0; k < 3; k++) acc += m[row][k] * xs[k][c];
            t[row][3 + c] += acc;
        }
    HM6 out = t;
    for (int r3 = 0; r3 < 3; r3++)
        for (int col = 0; col < 6; col++) {
            double acc = 0.0;
            for (int k = 0; k < 3; k++) acc += xr[k][r3] * t[k][col];
            out[3 + r3][col] += acc;
        }
    return out;
}

// L L' in place, pivots below 1e-12 of the largest dropped (solve.rs:138-165)
std::vector<bool> chol(std::vector<double>& a, size_t n) {
    double largest = 0.0;
    for (size_t i = 0; i < n; i++) largest = std::fmax(largest, a[i * n + i]);
    std::vector<bool> dropped(n, false);
    for (size_t j = 0; j < n; j++) {
        double d = a[j * n + j];
        for (size_t k = 0; k < j; k++) d -= a[j * n + k] * a[j * n + k];
        if (d <= largest * 1e-12) {
            dropped[j] = true;
            for (size_t i = j; i < n; i++) a[i * n + j] = 0.0;
            continue;
        }
        d = std::sqrt(d);
        a[j * n + j] = d;
        for (size_t i = j + 1; i < n; i++) {
            double s = a[i * n + j];
            for (size_t k = 0; k < j; k++) s -= a[i * n + k] * a[j * n + k];
            a[i * n + j] = s / d;
        }
    }
    return dropped;
}

void chol_solve(const std::vector<double>& a, const std::vector<bool>& dropped, size_t n, double* b) {  // :167-186
    for (size_t i = 0; i < n; i++) {
        if (dropped[i]) {
            b[i] = 0.0;
            continue;
        }
        double s = 0.0;
        for (size_t k = 0; k < i; k++) s += a[i * n + k] * b[k];
        b[i] = (b[i] - s) / a[i * n + i];
    }
    for (size_t i = n; i-- > 0;) {
        if (dropped[i]) {
            b[i] = 0.0;
            continue;
        }
        double s = 0.0;
        for (size_t k = i + 1; k < n; k++) s += a[k * n + i] * b[k];
        b[i] = (b[i] - s) / a[i * n + i];
    }
}

// the inverse operator of a factored n x n matrix: row-major, out[c * n + r] = (A^-1 e_c)[r]
// as solve.rs:123-135 lays it out (the same matrix, A being symmetric)
std::vector<double> chol_inverse(std::vector<double> a, size_t n) {
    std::vector<bool> l = chol(a, n);
    std::vector<double> out(n * n);
    std::vector<double> e(n);
    for (size_t c = 0; c < n; c++) {
        std::fill(e.begin(), e.end(), 0.0);
        e[c] = 1.0;
        chol_solve(a, l, n, e.data());
        for (size_t r = 0; r < n; r++) out[c * n + r] = e[r];
    }
    return out;
}

size_t uf_find(std::vector<size_t>& up, size_t i) {
    while (up[i] != i) {
        up[i] = up[up[i]];
        i = up[i];
    }
    return i;
}

int64_t half(int64_t v) { return v >= 0 ? v / 2 : -((-v + 1) / 2); }  // div_euclid(2)
std::array<int64_t, 3> parent_key(const std::array<int64_t, 3>& k) { return {half(k[0]), half(k[1]), half(k[2])}; }

struct HLevel {  // solve.rs:188-203
    std::vector<uint32_t> of;
    std::vector<H3> r;
    HSys sys;  // keys, centres, blocks
    std::vector<double> inv;  // 36 per part
    double size = 0.0, step = 1.0;
    bool direct = false;
    std::vector<double> top_inv;  // (6n)^2, the direct level's inverse operator
};

// 4/3 over the largest eigenvalue of over(apply), ten power steps from the reference's
// start (solve.rs:274-296)
template <size_t N, class Apply, class Over>
double power_step(size_t n, Apply apply, Over over) {
    typedef std::array<double, N> VN;
    auto norm = [](const std::vector<VN>& v) {
        double s = 0.0;
        for (const VN& e : v)
            for (double x : e) s += x * x;
        return std::sqrt(s);
    };
    std::vector<VN> v(n), a(n, VN{}), w(n, VN{});
    for (size_t k = 0; k < n; k++)
        for (size_t s = 0; s < N; s++) v[k][s] = 1.0 + (double)((7 * k + 3 * s) % 11) / 11.0;
    double most = 1.0;
    for (int it = 0; it < 10; it++) {
        apply(v, a);
        over(a, w);
        const double nw = norm(w), nv = norm(v);
        if (nw == 0.0) break;
        most = nw / nv;
        for (size_t k = 0; k < n; k++)
            for (size_t s = 0; s < N; s++) v[k][s] = w[k][s] / nw;
    }
    return 4.0 / 3.0 / most;
}

void factor_top(HLevel& L) {  // solve.rs:320-347
    const size_t n = L.sys.diag.size(), m = 6 * n;
    std::vector<double> a(36 * n * n, 0.0);
    for (size_t p = 0; p < n; p++) {
        const HM6& d = L.sys.diag[p];
        for (int r = 0; r < 6; r++)
            for (int c = 0; c < 6; c++) a[(6 * p + r) * m + 6 * p + c] += d[r][c];
        const double t = (d[0][0] + d[1][1] + d[2][2]) / 3.0;
        for (int k = 3; k < 6; k++) a[(6 * p + k) * m + 6 * p + k] += 1e-6 * t * L.size * L.size;
    }
    for (const HPair& e : L.sys.pairs)
        for (int r = 0; r < 6; r++)
            for (int c = 0; c < 6; c++) {
                a[(6 * e.i + r) * m + 6 * e.j + c] += e.m[r][c];
                a[(6 * e.j + c) * m + 6 * e.i + r] += e.m[r][c];
            }
    L.top_inv = chol_inverse(std::move(a), m);
    L.direct = true;
}

// The finer level seen by coarsen: a coarse HSys, or the nodes' arrays with their 3x3
// blocks embedded as 6x6 when read (solve.rs:97-103) rather than stored.
struct FineHSys {
    const HSys& s;
    size_t n() const { return s.keys.size(); }
    size_t npairs() const { return s.pairs.size(); }
    const std::array<int64_t, 3>& key(size_t i) const { return s.keys[i]; }
    H3 at(size_t i) const { return s.at[i]; }
    HM6 diag(size_t i) const { return s.diag[i]; }
    uint32_t pi(size_t q) const { return s.pairs[q].i; }
    uint32_t pj(size_t q) const { return s.pairs[q].j; }
    HM6 pair(size_t q) const { return s.pairs[q].m; }
};
struct FineNodes {
    int64_t nn, np;
    const int64_t* sites;
    const double *at_, *diag_;
    const uint32_t *pi_, *pj_;
    const double* pb;
    std::vector<std::array<int64_t, 3>> keys;
    FineNodes(int64_t n, const int64_t* s, const double* a, const double* d, int64_t m, const uint32_t* i,
              const uint32_t* j, const double* b)
        : nn(n), np(m), sites(s), at_(a), diag_(d), pi_(i), pj_(j), pb(b), keys(n) {
        for (int64_t q = 0; q < n; q++) keys[q] = {s[3 * q], s[3 * q + 1], s[3 * q + 2]};
    }
    static HM6 embed(const double* m) {
        HM6 e{};
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) e[r][c] = m[3 * r + c];
        return e;
    }
    size_t n() const { return (size_t)nn; }
    size_t npairs() const { return (size_t)np; }
    const std::array<int64_t, 3>& key(size_t i) const { return keys[i]; }
    H3 at(size_t i) const { return H3{at_[3 * i], at_[3 * i + 1], at_[3 * i + 2]}; }
    HM6 diag(size_t i) const { return embed(diag_ + 9 * i); }
    uint32_t pi(size_t q) const { return pi_[q]; }
    uint32_t pj(size_t q) const { return pj_[q]; }
    HM6 pair(size_t q) const { return embed(pb + 9 * q); }
};

// f(lo, hi) over [0, n) split among the host's cores
template <class F>
void parallel_ranges(size_t n, F f) {
    const size_t T = std::max<size_t>(1, std::min<size_t>(16, std::thread::hardware_concurrency()));
    if (n < 4096 || T == 1) {
        f(0, n);
        return;
    }
    std::vector<std::thread> th;
    for (size_t t = 0; t < T; t++) th.emplace_back(f, n * t / T, n * (t + 1) / T);
    for (auto& x : th) x.join();
}

// Each part's pairs in pair order (entry 2 q + side: side 0 where the part is the pair's
// first, 1 its second), so a product can run part by part on the host's cores and still
// add each part's terms in the order the reference's pair loop adds them
// (solve.rs:63-73, 306-317): the same values, bit for bit.
struct Incidence {
    std::vector<int64_t> ptr;
    std::vector<uint64_t> ent;
    template <class PI, class PJ>
    Incidence(size_t n, size_t np, PI pi, PJ pj) : ptr(n + 1, 0), ent(2 * np) {
        for (size_t q = 0; q < np; q++) {
            ptr[pi(q) + 1]++;
            ptr[pj(q) + 1]++;
        }
        for (size_t i = 0; i < n; i++) ptr[i + 1] += ptr[i];
        std::vector<int64_t> fill(ptr.begin(), ptr.end() - 1);
        for (size_t q = 0; q < np; q++) {
            ent[fill[pi(q)]++] = 2 * (uint64_t)q;
            ent[fill[pj(q)]++] = 2 * (uint64_t)q + 1;
        }
    }
};

// y = S x over B-vectors: diag(i, r, c) the diagonal blocks, pair(q, r, c) the pairs'
template <int B, class Diag, class Pair, class PI, class PJ>
void apply_rows(size_t n, const Incidence& inc, Diag diag, Pair pair, PI pi, PJ pj,
                const std::vector<std::array<double, B>>& x, std::vector<std::array<double, B>>& y) {
    parallel_ranges(n, [&](size_t lo, size_t hi) {
        for (size_t i = lo; i < hi; i++) {
            for (int r = 0; r < B; r++) {
                double acc = 0.0;
                for (int c = 0; c < B; c++) acc += diag(i, r, c) * x[i][c];
                y[i][r] = acc;
            }
            for (int64_t t = inc.ptr[i]; t < inc.ptr[i + 1]; t++) {
                const size_t q = (size_t)(inc.ent[t] >> 1);
                if ((inc.ent[t] & 1) == 0) {
                    const size_t j = pj(q);
                    for (int r = 0; r < B; r++) {
                        double a = 0.0;
                        for (int c = 0; c < B; c++) a += pair(q, r, c) * x[j][c];
                        y[i][r] += a;
                    }
                } else {
                    const size_t j = pi(q);
                    for (int r = 0; r < B; r++) {
                        double a = 0.0;
                        for (int c = 0; c < B; c++) a += pair(q, c, r) * x[j][c];
                        y[i][r] += a;
                    }
                }
            }
        }
    });
}

template <class Fine>
HLevel coarsen(const Fine& f, double size) {  // solve.rs:241-271
    const size_t nf = f.n();
    std::vector<size_t> up(nf);
    for (size_t i = 0; i < nf; i++) up[i] = i;
    for (size_t q = 0; q < f.npairs(); q++)
        if (parent_key(f.key(f.pi(q))) == parent_key(f.key(f.pj(q)))) {
            size_t r = uf_find(up, f.pi(q)), s = uf_find(up, f.pj(q));
            up[std::max(r, s)] = std::min(r, s);
        }
    HLevel L;
    L.of.resize(nf);
    std::vector<uint32_t> index(nf, UINT32_MAX);
    uint32_t n = 0;
    for (size_t i = 0; i < nf; i++) {
        size_t root = uf_find(up, i);
        if (index[root] == UINT32_MAX) index[root] = n++;
        L.of[i] = index[root];
    }
    HSys& c = L.sys;
    c.at.assign(n, H3{0.0, 0.0, 0.0});
    c.keys.assign(n, std::array<int64_t, 3>{0, 0, 0});
    std::vector<double> count(n, 0.0);
    for (size_t i = 0; i < nf; i++) {
        const uint32_t a = L.of[i];
        const H3 x = f.at(i);
        for (int k = 0; k < 3; k++) c.at[a][k] = c.at[a][k] + x[k];
        count[a] += 1.0;
        c.keys[a] = parent_key(f.key(i));
    }
    for (uint32_t a = 0; a < n; a++)
        for (int k = 0; k < 3; k++) c.at[a][k] = c.at[a][k] * (1.0 / count[a]);
    L.r.resize(nf);
    for (size_t i = 0; i < nf; i++) {
        const H3 x = f.at(i);
        for (int k = 0; k < 3; k++) L.r[i][k] = x[k] - c.at[L.of[i]][k];
    }
    c.diag.assign(n, HM6{});
    auto plus = [](HM6& a, const HM6& b) {
        for (int r = 0; r < 6; r++)
            for (int cc = 0; cc < 6; cc++) a[r][cc] += b[r][cc];
    };
    auto tr = [](const HM6& m) {
        HM6 t;
        for (int r = 0; r < 6; r++)
            for (int cc = 0; cc < 6; cc++) t[r][cc] = m[cc][r];
        return t;
    };
    // Each aggregate's block: its members' lifted blocks in member order, then its inner
    // pairs' (m + m') in pair order; each pair across two aggregates (a < c) summed in
    // pair order into block (a, c); blocks in (a, c) order. That is the order the
    // reference adds them in (solve.rs:254-262), here computed aggregate by aggregate and
    // group by group on the host's cores.
    std::vector<std::pair<uint64_t, uint32_t>> pairs_by;  // ((lesser, greater) part, fine pair)
    pairs_by.reserve(f.npairs());
    for (size_t q = 0; q < f.npairs(); q++) {
        const uint32_t a = L.of[f.pi(q)], b = L.of[f.pj(q)];
        pairs_by.push_back({((uint64_t)std::min(a, b) << 32) | std::max(a, b), (uint32_t)q});
    }
    std::sort(pairs_by.begin(), pairs_by.end());
    std::vector<int64_t> mptr(n + 1, 0);
    for (size_t i = 0; i < nf; i++) mptr[L.of[i] + 1]++;
    for (uint32_t a = 0; a < n; a++) mptr[a + 1] += mptr[a];
    std::vector<uint32_t> mem(nf);
    {
        std::vector<int64_t> fill(mptr.begin(), mptr.end() - 1);
        for (size_t i = 0; i < nf; i++) mem[fill[L.of[i]]++] = (uint32_t)i;
    }
    parallel_ranges(n, [&](size_t lo, size_t hi) {
        for (size_t a = lo; a < hi; a++)
            for (int64_t t = mptr[a]; t < mptr[a + 1]; t++) {
                const uint32_t i = mem[t];
                plus(c.diag[a], lift6(f.diag(i), L.r[i], L.r[i]));
            }
    });
    // group starts, then the groups on the cores (each thread's blocks in order)
    std::vector<size_t> gstart;
    for (size_t g = 0; g < pairs_by.size(); g++)
        if (g == 0 || pairs_by[g].first != pairs_by[g - 1].first) gstart.push_back(g);
    gstart.push_back(pairs_by.size());
    const size_t ng = gstart.size() - 1;
    std::vector<std::vector<HPair>> part_pairs(std::max<size_t>(1, std::min<size_t>(16, std::thread::hardware_concurrency())));
    std::vector<size_t> part_of_lo;
    std::mutex mu;
    parallel_ranges(ng, [&](size_t lo, size_t hi) {
        std::vector<HPair> mine;
        for (size_t gi = lo; gi < hi; gi++) {
            const uint64_t key = pairs_by[gstart[gi]].first;
            const uint32_t a = (uint32_t)(key >> 32), b = (uint32_t)key;
            HM6 acc{};
            for (size_t g = gstart[gi]; g < gstart[gi + 1]; g++) {
                const uint32_t q = pairs_by[g].second;
                const HM6 m = lift6(f.pair(q), L.r[f.pi(q)], L.r[f.pj(q)]);
                if (a == b) {
                    plus(c.diag[a], m);
                    plus(c.diag[a], tr(m));
                } else {
                    plus(acc, L.of[f.pi(q)] < L.of[f.pj(q)] ? m : tr(m));
                }
            }
            if (a != b) mine.push_back(HPair{a, b, acc});
        }
        std::lock_guard<std::mutex> lock(mu);
        part_of_lo.push_back(lo);
        part_pairs[part_of_lo.size() - 1] = std::move(mine);
    });
    {
        std::vector<size_t> order(part_of_lo.size());
        for (size_t t = 0; t < order.size(); t++) order[t] = t;
        std::sort(order.begin(), order.end(), [&](size_t u, size_t v) { return part_of_lo[u] < part_of_lo[v]; });
        for (size_t t : order) c.pairs.insert(c.pairs.end(), part_pairs[t].begin(), part_pairs[t].end());
    }
    L.inv.resize(36 * (size_t)n);
    for (uint32_t p = 0; p < n; p++) {
        HM6 d = c.diag[p];
        const double t = (d[0][0] + d[1][1] + d[2][2]) / 3.0;
        for (int k = 3; k < 6; k++) d[k][k] += 1e-6 * t * size * size;
        std::vector<double> a(36);
        for (int r = 0; r < 6; r++)
            for (int cc = 0; cc < 6; cc++) a[6 * r + cc] = d[r][cc];
        std::vector<double> iv = chol_inverse(std::move(a), 6);
        std::copy(iv.begin(), iv.end(), L.inv.begin() + 36 * (size_t)p);
    }
    L.size = size;
    const Incidence inc(n, c.pairs.size(), [&](size_t q) { return c.pairs[q].i; },
                        [&](size_t q) { return c.pairs[q].j; });
    L.step = power_step<6>(
        n,
        [&](const std::vector<H6>& x, std::vector<H6>& y) {
            apply_rows<6>(
                n, inc, [&](size_t i, int r, int cc) { return c.diag[i][r][cc]; },
                [&](size_t q, int r, int cc) { return c.pairs[q].m[r][cc]; }, [&](size_t q) { return c.pairs[q].i; },
                [&](size_t q) { return c.pairs[q].j; }, x, y);
        },
        [&](const std::vector<H6>& x, std::vector<H6>& y) {
            for (uint32_t p = 0; p < n; p++)
                for (int r = 0; r < 6; r++) {
                    double acc = 0.0;
                    for (int cc = 0; cc < 6; cc++) acc += L.inv[36 * (size_t)p + 6 * r + cc] * x[p][cc];
                    y[p][r] = acc;
                }
        });
    if (n <= MECH_DIRECT) factor_top(L);
    return L;
}

// ---- the device ---------------------------------------------------------------------
// y = S x (resid: y = b - S x) over the nodes' 3x3 block rows
__global__ void k_bsr3(int64_t n, const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                       const double* __restrict__ val, const double* __restrict__ x, const double* __restrict__ b,
                       double* __restrict__ y) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int64_t e = rowptr[i]; e < rowptr[i + 1]; e++) {
        const double* m = val + 9 * e;
        const double* xv = x + 3 * (int64_t)col[e];
        const double x0 = xv[0], x1 = xv[1], x2 = xv[2];
        a0 += m[0] * x0 + m[1] * x1 + m[2] * x2;
        a1 += m[3] * x0 + m[4] * x1 + m[5] * x2;
        a2 += m[6] * x0 + m[7] * x1 + m[8] * x2;
    }
    if (b) {
        y[3 * i] = b[3 * i] - a0;
        y[3 * i + 1] = b[3 * i + 1] - a1;
        y[3 * i + 2] = b[3 * i + 2] - a2;
    } else {
        y[3 * i] = a0;
        y[3 * i + 1] = a1;
        y[3 * i + 2] = a2;
    }
}

// out = base + step * inv (v - w) per node (base, w nullable: 0; base may be out)
__global__ void k_jacobi3(int64_t n, const double* __restrict__ inv, double step, const double* __restrict__ v,
                          const double* __restrict__ w, const double* base, double* out) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d[3];
    for (int k = 0; k < 3; k++) d[k] = w ? v[3 * i + k] - w[3 * i + k] : v[3 * i + k];
    const double* m = inv + 9 * i;
    for (int r = 0; r < 3; r++) {
        double s = m[3 * r] * d[0] + m[3 * r + 1] * d[1] + m[3 * r + 2] * d[2];
        out[3 * i + r] = (base ? base[3 * i + r] : 0.0) + s * step;
    }
}

// rb[a] = sum over a's members p of (r_t, r_w + rp x r_t); W = 3 (nodes: r_w = 0) or 6
template <int W>
__global__ void k_restrict(int64_t nc, const int64_t* __restrict__ mptr, const int32_t* __restrict__ mem,
                           const double* __restrict__ rr, const double* __restrict__ v, const double* __restrict__ w,
                           double* __restrict__ rb) {
    int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (a >= nc) return;
    double o[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int64_t t = mptr[a]; t < mptr[a + 1]; t++) {
        const int64_t p = mem[t];
        double f[6];
        for (int k = 0; k < W; k++) f[k] = w ? v[W * p + k] - w[W * p + k] : v[W * p + k];
        const double r0 = rr[3 * p], r1 = rr[3 * p + 1], r2 = rr[3 * p + 2];
        const double t0 = r1 * f[2] - r2 * f[1], t1 = r2 * f[0] - r0 * f[2], t2 = r0 * f[1] - r1 * f[0];
        o[0] += f[0];
        o[1] += f[1];
        o[2] += f[2];
        if (W == 6) {
            o[3] += f[3] + t0;
            o[4] += f[4] + t1;
            o[5] += f[5] + t2;
        } else {
            o[3] += t0;
            o[4] += t1;
            o[5] += t2;
        }
    }
    for (int k = 0; k < 6; k++) rb[6 * a + k] = o[k];
}

// x[p] += (e_t + e_w x r_p, e_w) of its part (W = 3: the translation only)
template <int W>
__global__ void k_prolong(int64_t nf, const int32_t* __restrict__ of, const double* __restrict__ rr,
                          const double* __restrict__ e, double* __restrict__ x) {
    int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= nf) return;
    const double* ea = e + 6 * (int64_t)of[p];
    const double r0 = rr[3 * p], r1 = rr[3 * p + 1], r2 = rr[3 * p + 2];
    const double u0 = ea[4] * r2 - ea[5] * r1, u1 = ea[5] * r0 - ea[3] * r2, u2 = ea[3] * r1 - ea[4] * r0;
    x[W * p] += ea[0] + u0;
    x[W * p + 1] += ea[1] + u1;
    x[W * p + 2] += ea[2] + u2;
    if (W == 6)
        for (int k = 3; k < 6; k++) x[W * p + k] += ea[k];
}

// x = A^-1 b, A^-1 (m x m) laid out as out[c * m + r]
__global__ void k_top(int64_t m, const double* __restrict__ ainv, const double* __restrict__ b, double* __restrict__ x) {
    for (int64_t r = threadIdx.x; r < m; r += blockDim.x) {
        double s = 0.0;
        for (int64_t c = 0; c < m; c++) s += ainv[c * m + r] * b[c];
        x[r] = s;
    }
}

// per-block partial sums of a . b, a fixed order
constexpr int MDOT_BLOCKS = 256;
__global__ void __launch_bounds__(256) k_mdot(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                                              double* __restrict__ part) {
    __shared__ double red[256];
    const int64_t per = (n + MDOT_BLOCKS - 1) / MDOT_BLOCKS;
    const int64_t lo = blockIdx.x * per, hi = min(n, lo + per);
    double s = 0.0;
    for (int64_t i = lo + threadIdx.x; i < hi; i += 256) s += a[i] * b[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// The PCG's scalars (solve.rs:485-538) where the iterations run on the device: the loop
// goes on until `stop`, with `rounds` the rounds the reference would report.
struct MechCG {
    double rz, target, pap, alpha, beta, nx;
    int32_t stop, round, rounds;
    uint32_t count;  // rounds since the graph's launch
};

// *out = the partial sums of k_mdot, added in order (as the host adds them)
__global__ void k_mdot_sum(const double* __restrict__ part, double* __restrict__ out) {
    double s = 0.0;
    for (int i = 0; i < MDOT_BLOCKS; i++) s += part[i];
    *out = s;
}

// after p'Ap: a round that meets p'Ap <= 0 stops (and counts), else alpha = rz / p'Ap
__global__ void k_mcg_alpha(MechCG* c) {
    if (c->stop) return;
    if (c->pap <= 0.0) {
        c->rounds = c->round;
        c->stop = 1;
    } else {
        c->alpha = c->rz / c->pap;
    }
}

// after r'z: beta = r'z / rz, rz = r'z, the round done, and the next round's tests
// (solve.rs: the cap stops, rz < 0 gives None, rz <= target stops)
__global__ void k_mcg_beta(MechCG* c) {
    if (c->stop) return;
    c->beta = c->nx / c->rz;
    c->rz = c->nx;
    c->round += 1;
    if (c->round >= MECH_ROUNDS) {  // the cap ends the loop before its tests
        c->rounds = MECH_ROUNDS;
        c->stop = 1;
    } else if (c->rz < 0.0) {
        c->rounds = -1;
        c->stop = 1;
    } else if (c->rz <= c->target) {
        c->rounds = c->round;
        c->stop = 1;
    }
}

// the loop's condition: on while not stopped and fewer than `chunk` rounds ran since the
// launch (so the host looks in now and then)
__global__ void k_mcg_more(cudaGraphConditionalHandle h, MechCG* c, uint32_t chunk) {
    const uint32_t n = c->count + 1u;
    c->count = n;
    cudaGraphSetConditional(h, (!c->stop && n < chunk) ? 1u : 0u);
}

// k_mupdate with the step from the device's scalars; nothing once stopped
__global__ void k_mupdate_d(int64_t n, int update, const MechCG* __restrict__ c, double* __restrict__ x,
                            double* __restrict__ r, const double* __restrict__ p, const double* __restrict__ ap) {
    if (c->stop) return;
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (update == 0) {
        const double s = c->alpha;
        x[i] = x[i] + p[i] * s;
        r[i] = r[i] - ap[i] * s;
    } else {
        x[i] = r[i] + x[i] * c->beta;  // x = p, r = z
    }
}

struct MechSolver {
    Context& ctx;
    MechLevels& M;
    DBuf<double> part;
    std::vector<double> hpart;

    MechSolver(Context& c, MechLevels& m) : ctx(c), M(m) {}

    double dot(const double* a, const double* b, int64_t n) {
        k_mdot<<<MDOT_BLOCKS, 256, 0, ctx.stream>>>(n, a, b, part.get());
        SC_LAUNCH_CK();
        part.download(hpart.data(), MDOT_BLOCKS);
        SC_CK(cudaStreamSynchronize(ctx.stream));
        double s = 0.0;
        for (int i = 0; i < MDOT_BLOCKS; i++) s += hpart[i];
        return s;
    }
    // *out = a . b on the device (the same partial sums, added in the same order, as dot)
    void dot_d(const double* a, const double* b, int64_t n, double* out) {
        k_mdot<<<MDOT_BLOCKS, 256, 0, ctx.stream>>>(n, a, b, part.get());
        SC_LAUNCH_CK();
        k_mdot_sum<<<1, 1, 0, ctx.stream>>>(part.get(), out);
        SC_LAUNCH_CK();
    }
    void times(const double* x, double* y, const double* b = nullptr) {
        k_bsr3<<<grid_for(M.n0, 128), 128, 0, ctx.stream>>>(M.n0, M.rowptr0.get(), M.col0.get(), M.val0.get(), x, b,
                                                             y);
        SC_LAUNCH_CK();
    }
    // x = V-cycle of level l for its b (solve.rs:403-447)
    void cycle(size_t l) {
        MechLevel& L = M.lv[l];
        if (L.direct) {
            k_top<<<1, 256, 0, ctx.stream>>>(6 * L.n, L.top_inv.get(), L.b.get(), L.x.get());
            SC_LAUNCH_CK();
            return;
        }
        MechLevel& U = M.lv[l + 1];
        jacobi<double>(ctx, L.n, L.inv.get(), L.b.get(), L.x.get(), L.step.get(), nullptr, nullptr, nullptr);
        spmv<double>(ctx, SPMV_RES, L.n, L.rowptr.get(), L.col.get(), L.val.get(), L.x.get(), L.b.get(), L.res.get(),
                     nullptr, nullptr, nullptr, nullptr, nullptr, L.nnzb);
        k_restrict<6><<<grid_for(U.n, 128), 128, 0, ctx.stream>>>(U.n, U.mptr.get(), U.mem.get(), U.r.get(),
                                                                   L.res.get(), nullptr, U.b.get());
        SC_LAUNCH_CK();
        cycle(l + 1);
        k_prolong<6><<<grid_for(L.n, 256), 256, 0, ctx.stream>>>(L.n, U.of.get(), U.r.get(), U.x.get(), L.x.get());
        SC_LAUNCH_CK();
        spmv<double>(ctx, SPMV_RES, L.n, L.rowptr.get(), L.col.get(), L.val.get(), L.x.get(), L.b.get(), L.res.get(),
                     nullptr, nullptr, nullptr, nullptr, nullptr, L.nnzb);
        jacobi_add<double>(ctx, L.n, L.inv.get(), L.res.get(), L.x.get(), L.t.get(), L.step.get(), nullptr, nullptr,
                           nullptr);
        std::swap(L.x, L.t);
    }
    // out = the preconditioner of b (solve.rs:450-476); scratch: 3 n0
    void precondition(const double* b, double* out, double* scratch) {
        const unsigned g = grid_for(M.n0, 256);
        k_jacobi3<<<g, 256, 0, ctx.stream>>>(M.n0, M.inv0.get(), M.step0, b, nullptr, nullptr, out);
        SC_LAUNCH_CK();
        times(out, scratch);
        MechLevel& U = M.lv[0];
        k_restrict<3><<<grid_for(U.n, 128), 128, 0, ctx.stream>>>(U.n, U.mptr.get(), U.mem.get(), U.r.get(), b,
                                                                   scratch, U.b.get());
        SC_LAUNCH_CK();
        cycle(0);
        k_prolong<3><<<g, 256, 0, ctx.stream>>>(M.n0, U.of.get(), U.r.get(), U.x.get(), out);
        SC_LAUNCH_CK();
        times(out, scratch);
        k_jacobi3<<<g, 256, 0, ctx.stream>>>(M.n0, M.inv0.get(), M.step0, b, scratch, out, out);
        SC_LAUNCH_CK();
    }
};

}  // namespace

// ---- a voxel piece at rest as a system (mechanics/src/lib.rs:375-423, 638-676) ----------
// Every free cell an 8-node element of the unit cube's stiffness (element.rs:44-69, a
// Poisson's ratio of 0.3) times E h, welded to its free neighbours (corners at one lattice
// point are one node, numbered by the first cell and corner that reach it); a corner
// touching a held cell is held. Unknowns: the other nodes in order; diagonal blocks
// m I + (dt^2 + 0.3 dt) E h K_aa; pairs in first-encounter order over cells and corner
// pairs, (min, max), their blocks transposed where the first node is the greater;
// b = m (0, -9.81 dt, 0) (at rest, gravity along -y).
namespace {
const int MCORNERS[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {1, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
typedef std::array<std::array<HM3, 8>, 8> HUnit;
const HUnit& unit_cube() {
    static HUnit k = [] {
        HUnit k{};
        const double NU = 0.3, g = 1.0 / std::sqrt(3.0);
        auto sgn = [](int c) {
            return H3{(double)(2 * MCORNERS[c][0] - 1), (double)(2 * MCORNERS[c][1] - 1),
                      (double)(2 * MCORNERS[c][2] - 1)};
        };
        auto strain = [&](int a, const H3& at) {  // rows xx, yy, zz, 2yz, 2xz, 2xy
            H3 s = sgn(a), gr;
            for (int q = 0; q < 3; q++) {
                double prod = 1.0;
                for (int j = 0; j < 3; j++)
                    if (j != q) prod *= 1.0 + s[j] * at[j];
                gr[q] = s[q] / 4.0 * prod;
            }
            return std::array<H3, 6>{H3{gr[0], 0.0, 0.0}, H3{0.0, gr[1], 0.0}, H3{0.0, 0.0, gr[2]},
                                     H3{0.0, gr[2], gr[1]}, H3{gr[2], 0.0, gr[0]}, H3{gr[1], gr[0], 0.0}};
        };
        const double l = NU / ((1.0 + NU) * (1.0 - 2.0 * NU)), m = 1.0 / (2.0 * (1.0 + NU));
        for (int p = 0; p < 8; p++) {
            const H3 s = sgn(p), at{s[0] * g, s[1] * g, s[2] * g};
            std::array<std::array<H3, 6>, 8> b;
            for (int a = 0; a < 8; a++) b[a] = strain(a, at);
            for (int a = 0; a < 8; a++)
                for (int c = 0; c < 8; c++)
                    for (int j = 0; j < 3; j++) {
                        double e[6];
                        for (int r = 0; r < 6; r++) e[r] = b[c][r][j];
                        const double tr = e[0] + e[1] + e[2];
                        const double st[6] = {l * tr + 2.0 * m * e[0], l * tr + 2.0 * m * e[1], l * tr + 2.0 * m * e[2],
                                              m * e[3], m * e[4], m * e[5]};
                        for (int i = 0; i < 3; i++) {
                            double acc = 0.0;
                            for (int r = 0; r < 6; r++) acc += b[a][r][i] * st[r];
                            k[a][c][i][j] += acc / 8.0;
                        }
                    }
        }
        return k;
    }();
    return k;
}
}  // namespace

void mech_voxel_system(const uint8_t* state, const float* e, int nx, int ny, int nz, double h, double dt,
                       double mass, std::vector<int64_t>& sites, std::vector<double>& at, std::vector<double>& diag,
                       std::vector<uint32_t>& pi, std::vector<uint32_t>& pj, std::vector<double>& pb,
                       std::vector<double>& b) {
    auto st = [&](int x, int y, int z) -> int {
        if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) return 0;
        return state[((int64_t)x * ny + y) * nz + z];
    };
    std::vector<std::array<int, 3>> cells;
    std::vector<double> ke;
    for (int x = 0; x < nx; x++)
        for (int y = 0; y < ny; y++)
            for (int z = 0; z < nz; z++)
                if (st(x, y, z) == 1) {
                    cells.push_back({x, y, z});
                    ke.push_back((double)e[((int64_t)x * ny + y) * nz + z]);
                }
    const int64_t NY = ny + 1, NZ = nz + 1;
    std::vector<int64_t> node_of((size_t)((int64_t)(nx + 1) * NY * NZ), -1);
    std::vector<std::array<int64_t, 3>> nsite;
    std::vector<double> nmass;
    std::vector<char> nheld;
    std::vector<std::array<uint32_t, 8>> corners(cells.size());
    for (size_t i = 0; i < cells.size(); i++)
        for (int c = 0; c < 8; c++) {
            const int px = cells[i][0] + MCORNERS[c][0], py = cells[i][1] + MCORNERS[c][1],
                      pz = cells[i][2] + MCORNERS[c][2];
            const int64_t g = (px * NY + py) * NZ + pz;
            if (node_of[g] < 0) {
                node_of[g] = (int64_t)nsite.size();
                nsite.push_back({px, py, pz});
                nmass.push_back(0.0);
                bool held = false;
                for (int dx = -1; dx <= 0; dx++)
                    for (int dy = -1; dy <= 0; dy++)
                        for (int dz = -1; dz <= 0; dz++) held = held || st(px + dx, py + dy, pz + dz) == 2;
                nheld.push_back(held);
            }
            corners[i][c] = (uint32_t)node_of[g];
            nmass[node_of[g]] += mass / 8.0;
        }
    const uint32_t NONE = UINT32_MAX, TURNED = 1u << 31;
    std::vector<uint32_t> fr(nsite.size());
    uint32_t count = 0;
    for (size_t k = 0; k < nsite.size(); k++) fr[k] = nheld[k] ? NONE : count++;
    sites.clear(), at.clear(), diag.clear(), pi.clear(), pj.clear(), pb.clear(), b.clear();
    for (size_t k = 0; k < nsite.size(); k++) {
        if (fr[k] == NONE) continue;
        for (int q = 0; q < 3; q++) {
            sites.push_back(nsite[k][q]);
            at.push_back(nsite[k][q] * h);
        }
        const double m = nmass[k];
        const double d[9] = {m, 0.0, 0.0, 0.0, m, 0.0, 0.0, 0.0, m};
        diag.insert(diag.end(), d, d + 9);
        b.push_back(0.0 * m);
        b.push_back(-9.81 * dt * m);
        b.push_back(0.0 * m);
    }
    std::map<std::pair<uint32_t, uint32_t>, uint32_t> index;
    std::vector<std::array<uint32_t, 64>> slots(cells.size());
    for (size_t i = 0; i < cells.size(); i++) {
        slots[i].fill(NONE);
        for (int a = 0; a < 8; a++)
            for (int c = a + 1; c < 8; c++) {
                const uint32_t p = fr[corners[i][a]], q = fr[corners[i][c]];
                if (p == NONE || q == NONE) continue;
                const auto key = std::make_pair(std::min(p, q), std::max(p, q));
                auto it = index.find(key);
                uint32_t k;
                if (it == index.end()) {
                    k = (uint32_t)pi.size();
                    index.emplace(key, k);
                    pi.push_back(key.first);
                    pj.push_back(key.second);
                    pb.insert(pb.end(), 9, 0.0);
                } else {
                    k = it->second;
                }
                slots[i][8 * a + c] = k | (p > q ? TURNED : 0u);
            }
    }
    const double stiff = dt * dt + 0.3 * dt;
    const HUnit& K = unit_cube();
    for (size_t i = 0; i < cells.size(); i++) {
        const double k = ke[i] * h;
        for (int a = 0; a < 8; a++) {
            const uint32_t p = fr[corners[i][a]];
            if (p != NONE)
                for (int r = 0; r < 3; r++)
                    for (int c = 0; c < 3; c++) diag[9 * (size_t)p + 3 * r + c] += K[a][a][r][c] * k * stiff;
            for (int c = a + 1; c < 8; c++) {
                const uint32_t slot = slots[i][8 * a + c];
                if (slot == NONE) continue;
                double* into = pb.data() + 9 * (size_t)(slot & ~TURNED);
                const bool turned = (slot & TURNED) != 0;
                for (int r = 0; r < 3; r++)
                    for (int cc = 0; cc < 3; cc++) into[3 * r + cc] += (turned ? K[a][c][cc][r] : K[a][c][r][cc]) * k * stiff;
            }
        }
    }
}

// Solver::new on the host (solve.rs:361-386): level 0's block inverses and step, then the
// coarse levels.
struct HostLevels {
    std::vector<double> inv0;
    double step0 = 1.0;
    std::vector<HLevel> levels;
};

static HostLevels make_levels(int64_t n, const int64_t* sites, const double* at, const double* diag, int64_t npairs,
                              const uint32_t* pi, const uint32_t* pj, const double* pb, double size) {
    HostLevels H;
    std::vector<double>& inv0 = H.inv0;
    inv0.resize(9 * (size_t)n);
    for (int64_t i = 0; i < n; i++) {
        std::vector<double> a(diag + 9 * i, diag + 9 * i + 9);
        std::vector<double> iv = chol_inverse(std::move(a), 3);
        std::copy(iv.begin(), iv.end(), inv0.begin() + 9 * i);
    }
    const Incidence inc0((size_t)n, (size_t)npairs, [&](size_t q) { return pi[q]; }, [&](size_t q) { return pj[q]; });
    auto times0 = [&](const std::vector<H3>& xv, std::vector<H3>& yv) {  // solve.rs:63-73
        apply_rows<3>(
            (size_t)n, inc0, [&](size_t i, int r, int c) { return diag[9 * i + 3 * r + c]; },
            [&](size_t q, int r, int c) { return pb[9 * q + 3 * r + c]; }, [&](size_t q) { return pi[q]; },
            [&](size_t q) { return pj[q]; }, xv, yv);
    };
    H.step0 = power_step<3>(n, times0, [&](const std::vector<H3>& xv, std::vector<H3>& yv) {
        for (int64_t i = 0; i < n; i++)
            for (int r = 0; r < 3; r++) {
                double acc = 0.0;
                for (int c = 0; c < 3; c++) acc += inv0[9 * i + 3 * r + c] * xv[i][c];
                yv[i][r] = acc;
            }
    });
    // the coarse levels (solve.rs:365-385)
    std::vector<HLevel>& levels = H.levels;
    double sz = size;
    HLevel next = coarsen(FineNodes(n, sites, at, diag, npairs, pi, pj, pb), sz * 2.0);
    for (;;) {
        sz *= 2.0;
        const size_t nn = next.sys.diag.size(), before = levels.empty() ? (size_t)n : levels.back().sys.diag.size();
        if (next.direct) {
            levels.push_back(std::move(next));
            break;
        }
        if (nn == before) {
            factor_top(next);
            levels.push_back(std::move(next));
            break;
        }
        levels.push_back(std::move(next));
        next = coarsen(FineHSys{levels.back().sys}, sz * 2.0);
    }
    return H;
}

void mech_levels(int64_t n, const int64_t* sites, const double* at, const double* diag, int64_t npairs,
                 const uint32_t* pi, const uint32_t* pj, const double* pb, double size, std::vector<int64_t>& sizes,
                 std::vector<double>& steps) {
    HostLevels H = make_levels(n, sites, at, diag, npairs, pi, pj, pb, size);
    sizes.clear();
    steps.assign(1, H.step0);
    for (const HLevel& L : H.levels) {
        sizes.push_back((int64_t)L.sys.diag.size());
        steps.push_back(L.direct ? 0.0 : L.step);
    }
}

// The same, made on the device as mech_solve makes them.
void mech_levels_device(Context& ctx, int64_t n, const int64_t* sites, const double* at, const double* diag,
                        int64_t npairs, const uint32_t* pi, const uint32_t* pj, const double* pb, double size,
                        std::vector<int64_t>& sizes, std::vector<double>& steps) {
    MechLevels M;
    mech_device_levels(ctx, n, sites, at, diag, npairs, pi, pj, pb, size, M);
    sizes.clear();
    steps.assign(1, M.step0);
    for (const MechLevel& L : M.lv) {
        sizes.push_back(L.n);
        steps.push_back(L.direct ? 0.0 : L.step_h);
    }
}

std::vector<double> mech_top_inverse(int64_t n, const double* diag36, int64_t npairs, const uint32_t* pi,
                                     const uint32_t* pj, const double* pm36, double size) {
    HLevel L;
    L.size = size;
    L.sys.diag.resize((size_t)n);
    for (int64_t p = 0; p < n; p++)
        for (int r = 0; r < 6; r++)
            for (int c = 0; c < 6; c++) L.sys.diag[p][r][c] = diag36[36 * p + 6 * r + c];
    L.sys.pairs.resize((size_t)npairs);
    for (int64_t e = 0; e < npairs; e++) {
        HPair& q = L.sys.pairs[e];
        q.i = pi[e];
        q.j = pj[e];
        for (int r = 0; r < 6; r++)
            for (int c = 0; c < 6; c++) q.m[r][c] = pm36[36 * e + 6 * r + c];
    }
    factor_top(L);
    return std::move(L.top_inv);
}

// The PCG's rounds from the first one on (solve.rs:495-536), all on the device: a round
// is captured once into a graph whose conditional WHILE node replays it until the scalars
// say stop (or `chunk` rounds ran, when the host looks in); without conditional nodes the
// round is launched from the host, which looks in after each. The same kernels and the
// same additions in the same order as rounds driven from the host.
static int device_rounds(Context& ctx, MechSolver& S, int64_t m, double rz, double target, double* x, double* r,
                         double* z, double* p, double* ap, double* scratch) {
    cudaStream_t st = ctx.stream;
    DBuf<MechCG> cg;
    cg.alloc(1, st, &ctx.mem);
    MechCG c0{};
    c0.rz = rz;
    c0.target = target;
    c0.rounds = MECH_ROUNDS;
    cg.upload(&c0, 1);
    MechCG* c = cg.get();
    const unsigned g = grid_for(m, 256);
    auto round = [&] {
        S.times(p, ap);
        S.dot_d(p, ap, m, &c->pap);
        k_mcg_alpha<<<1, 1, 0, st>>>(c);
        SC_LAUNCH_CK();
        k_mupdate_d<<<g, 256, 0, st>>>(m, 0, c, x, r, p, ap);
        SC_LAUNCH_CK();
        S.precondition(r, z, scratch);
        S.dot_d(r, z, m, &c->nx);
        k_mcg_beta<<<1, 1, 0, st>>>(c);
        SC_LAUNCH_CK();
        k_mupdate_d<<<g, 256, 0, st>>>(m, 1, c, p, z, nullptr, nullptr);
        SC_LAUNCH_CK();
    };
    const uint32_t chunk = 64;
    cudaGraphExec_t exec = nullptr;
    {
        cudaGraph_t graph = nullptr;
        cudaGraphConditionalHandle h = 0;
        cudaGraphNodeParams prm = {};
        prm.type = cudaGraphNodeTypeConditional;
        prm.conditional.type = cudaGraphCondTypeWhile;
        prm.conditional.size = 1;
        cudaGraphNode_t node;
        if (cudaGraphCreate(&graph, 0) == cudaSuccess &&
            cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault) == cudaSuccess &&
            (prm.conditional.handle = h, cudaGraphAddNode(&node, graph, nullptr, 0, &prm) == cudaSuccess) &&
            cudaStreamBeginCaptureToGraph(st, prm.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            cudaGraph_t body = nullptr;
            try {
                round();
                k_mcg_more<<<1, 1, 0, st>>>(h, c, chunk);
                SC_LAUNCH_CK();
            } catch (...) {
                cudaStreamEndCapture(st, &body);
                cudaGraphDestroy(graph);
                throw;
            }
            if (cudaStreamEndCapture(st, &body) == cudaSuccess && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess)
                exec = nullptr;
        }
        cudaGetLastError();
        if (graph) cudaGraphDestroy(graph);
    }
    MechCG now{};
    try {
        for (;;) {
            if (exec) {
                SC_CK(cudaMemsetAsync(&c->count, 0, sizeof(uint32_t), st));
                SC_CK(cudaGraphLaunch(exec, st));
            } else {
                round();
            }
            cg.download(&now, 1);
            SC_CK(cudaStreamSynchronize(st));
            if (now.stop) break;
        }
    } catch (...) {
        if (exec) cudaGraphExecDestroy(exec);
        throw;
    }
    if (exec) cudaGraphExecDestroy(exec);
    return now.rounds;
}

// The levels of the system, then PCG from x (solve.rs:356-386, 485-538): the rounds taken,
// -1 where the levels do not fit the system (not positive).
int mech_solve(Context& ctx, int64_t n, const int64_t* sites, const double* at, const double* diag, int64_t npairs,
               const uint32_t* pi, const uint32_t* pj, const double* pb, const double* b, double* x, double tol,
               double size, int32_t* nlevels) {
    cudaStream_t st = ctx.stream;
    MemStats* ms = &ctx.mem;
    if (n == 0) return 0;
    PhaseTimer pt(ctx);  // SC_TIMING=1 prints the phases
    MechLevels levels;
    mech_device_levels(ctx, n, sites, at, diag, npairs, pi, pj, pb, size, levels);
    *nlevels = (int32_t)levels.lv.size();
    pt.mark("mech: levels (device)");
    MechSolver S(ctx, levels);
    S.part.alloc(MDOT_BLOCKS, st, ms);
    S.hpart.resize(MDOT_BLOCKS);
    // PCG from x (solve.rs:485-538)
    const int64_t m = 3 * n;
    DBuf<double> db, dx, r, z, p, ap, scratch;
    for (DBuf<double>* v : {&db, &dx, &r, &z, &p, &ap, &scratch}) v->alloc(m, st, ms);
    db.upload(b, m);
    dx.upload(x, m);
    S.precondition(db.get(), z.get(), scratch.get());
    const double target = tol * tol * S.dot(db.get(), z.get(), m);
    int rounds = -1;
    if (!(std::isnan(target) || target < 0.0)) {
        S.times(dx.get(), r.get(), db.get());  // r = b - S x
        S.precondition(r.get(), z.get(), scratch.get());
        SC_CK(cudaMemcpyAsync(p.get(), z.get(), m * sizeof(double), cudaMemcpyDeviceToDevice, st));
        const double rz = S.dot(r.get(), z.get(), m);
        rounds = rz < 0.0 ? -1 : rz <= target ? 0 : MECH_ROUNDS;
        if (rounds == MECH_ROUNDS) rounds = device_rounds(ctx, S, m, rz, target, dx.get(), r.get(), z.get(), p.get(),
                                                          ap.get(), scratch.get());
    }
    dx.download(x, m);
    SC_CK(cudaStreamSynchronize(st));
    pt.note("mech: %d rounds", rounds);
    pt.mark("mech: conjugate gradients");
    return rounds;
}

}  // namespace sc
