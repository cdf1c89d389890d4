// statics::gather (statics/src/gather.rs:193-395): a coarser level measured from a finer
// one.
//
// Each coarse cell of 2^l Z^3 becomes a small problem of its own: its free parts (finer
// nodes inside it, 6 unknowns each), one rigid handle per face (3 unknowns each) and the
// finer bonds between them. Measuring it is one Gauss–Jordan elimination of the free
// parts against every handle axis at once, the handles' reactions, a non-negative
// least-squares fit of beams between the faces, and, beam by beam, the finer bonds' use
// when the beam is pulled alone. In a full lattice a cell has at most 12 free parts and 6
// handles (a 72 x 90 elimination, 480 bonds), so the cells form a batch of fixed-shape
// dense problems. The indexing around them (coarse cells by first appearance, faces in
// key order, handles by first use) runs on the host, in the reference's orders.
//
// The cells are measured in one of two forms. measure_cell is the host's: any size, one
// host thread a cell. gf_measure_cell is the device's (k_gather_cells, one thread block a
// cell, bounded sizes); the host can also run it with one thread a cell
// (SC_GATHER_EMULATE), which is how the CPU tests check the kernel's own code. Each form is
// checked against the CPU restatement of gather.rs.
//
// Every floating-point operation is the reference's, in its order, so the gathered
// lattice is the reference's bit for bit (the CPU restatement checks it). Two places
// differ in form only: row swaps are a permutation of row indices, and the beams' Gram
// products skip the entries where a beam's unit stiffness is zero (adding a zero product
// never changes a non-zero sum; only the sign of an all-zero sum could differ).
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <utility>
#include <vector>

#include "common.cuh"
#include "solver.cuh"

namespace sc {
namespace gth {

using V3 = std::array<double, 3>;
using Site = std::array<int64_t, 3>;

// statics/src/model.rs:16-36, in its operation order
inline V3 add(V3 a, V3 b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
inline V3 sub(V3 a, V3 b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
inline V3 mul(V3 a, double s) { return {a[0] * s, a[1] * s, a[2] * s}; }
inline double dot(V3 a, V3 b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline V3 cross(V3 a, V3 b) { return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]}; }
inline double norm(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 unit(V3 a) { return mul(a, 1.0 / norm(a)); }

constexpr double UNIT = 0.125;                 // lattice.rs:16
constexpr double SECTION[2] = {0.336, 0.336};  // lattice.rs:25
constexpr double PI = 3.14159265358979323846;

inline double spacing(int level) { return UNIT * (double)(uint64_t(1) << level); }  // lattice.rs:34-36
inline V3 centre(const Site& s, int level) {                                         // lattice.rs:39-41
    V3 c;
    for (int k = 0; k < 3; k++) c[k] = ((double)s[k] + 0.5 * (double)(uint64_t(1) << level)) * UNIT;
    return c;
}
inline Site coarse_site(const Site& p, int level) {  // lattice.rs:45-47
    Site q;
    for (int k = 0; k < 3; k++) q[k] = p[k] & ~((int64_t(1) << level) - 1);
    return q;
}
inline size_t beam_class(V3 a, V3 b, V3 c) {  // lattice.rs:29-32
    V3 u = sub(a, c), v = sub(b, c);
    return (size_t)std::round(1.0 + dot(u, v) / (norm(u) * norm(v)));
}

struct Mat {  // the values of statics/src/model.rs:43-51 the gather uses
    double e, g, ft, fc, fs;
    double used(double s1, double s3) const {  // model.rs:66-68
        return std::fmax(std::fmax(s1 / ft, -s3 / fc), (s1 - s3) / (2.0 * fs));
    }
};

// A finer bond inside one cell's problem: its ends renumbered to the cell's places.
struct LBond {
    size_t i, j;
    V3 p, n;
    double a, d, e, g, ft, fc, fs;
    V3 force(V3 delta) const {  // model.rs:115-119
        double along = dot(delta, n);
        double k = a / d;
        return add(mul(n, e * k * along), mul(sub(delta, mul(n, along)), g * k));
    }
    double used(V3 f) const {  // model.rs:123-129
        V3 t = mul(f, 1.0 / a);
        double sigma = dot(t, n);
        double tau2 = std::fmax(dot(t, t) - sigma * sigma, 0.0);
        double r = std::sqrt(sigma * sigma / 4.0 + tau2);
        return Mat{e, g, ft, fc, fs}.used(sigma / 2.0 + r, sigma / 2.0 - r);
    }
    double energy(V3 f) const {  // model.rs:132-136
        double k = a / d;
        double along = dot(f, n);
        return 0.5 * (along * along / (e * k) + (dot(f, f) - along * along) / (g * k));
    }
};

// Rust's f64::total_cmp as an integer key.
inline int64_t total_key(double v) {
    int64_t i;
    std::memcpy(&i, &v, 8);
    return i ^ (int64_t)(((uint64_t)(i >> 63)) >> 1);
}

size_t find(std::vector<size_t>& p, size_t a) {  // bodies.rs:628-634
    while (p[a] != a) {
        p[a] = p[p[a]];
        a = p[a];
    }
    return a;
}

// gather.rs:164-184 on a row-major n x (n + rhs) matrix: Gauss–Jordan with the largest
// pivot (the last of equals), a pivot below 1e-12 of the largest diagonal skipped; the
// answer's rows into x (n x rhs), 0 where the pivot was skipped.
void eliminate(std::vector<double>& a, size_t n, size_t rhs, std::vector<size_t>& row, std::vector<double>& x) {
    const size_t w = n + rhs;
    double scale = 0.0;
    for (size_t r = 0; r < n; r++) scale = std::fmax(scale, std::fabs(a[r * w + r]));
    auto small = [&](double v) { return std::fabs(v) <= 1e-12 * scale; };
    row.resize(n);
    for (size_t r = 0; r < n; r++) row[r] = r;
    for (size_t c = 0; c < n; c++) {
        size_t p = c;
        int64_t best = total_key(std::fabs(a[row[c] * w + c]));
        for (size_t q = c + 1; q < n; q++) {
            int64_t k = total_key(std::fabs(a[row[q] * w + c]));
            if (k >= best) {
                best = k;
                p = q;
            }
        }
        std::swap(row[c], row[p]);
        const double* piv = &a[row[c] * w];
        if (small(piv[c])) continue;
        for (size_t r = 0; r < n; r++) {
            if (r == c) continue;
            double* ar = &a[row[r] * w];
            double f = ar[c] / piv[c];
            if (f != 0.0)
                for (size_t k = c; k < w; k++) ar[k] -= f * piv[k];
        }
    }
    x.assign(n * rhs, 0.0);
    for (size_t r = 0; r < n; r++) {
        const double* ar = &a[row[r] * w];
        for (size_t k = 0; k < rhs; k++) x[r * rhs + k] = small(ar[r]) ? 0.0 : ar[n + k] / ar[r];
    }
}

// One coarse cell's problem: places 0..nf-1 its free parts, nf.. its handles (one a face).
struct CellProblem {
    size_t nf = 0;
    std::vector<V3> place;  // each place's position: a free part's node centre, a handle's face centre
    std::vector<LBond> bonds;
};

struct Beam {
    size_t a, b;
    double k, stronger;
};

using Full = std::array<std::pair<double, double>, 2>;

struct Scratch {
    std::vector<double> a, x, k, g, sol, target, forces;
    std::vector<size_t> row;
};

// gather.rs:119-161: the beams (a < b, their stiffness along them) nearest the handles'
// stiffness k (m x m, m = 3 handles), none negative, only between joined handles.
template <class J>
std::vector<std::tuple<size_t, size_t, double>> fit_beams(const std::vector<double>& k, const std::vector<V3>& at,
                                                          J joined, Scratch& s) {
    const size_t nh = at.size(), n = 3 * nh;
    std::vector<std::pair<size_t, size_t>> pairs;
    for (size_t a = 0; a < nh; a++)
        for (size_t b = a + 1; b < nh; b++)
            if (joined(a, b)) pairs.push_back({a, b});
    // A unit of each beam's stiffness: four 3x3 blocks, kept as (flat index, value) in
    // flat order, the order the dense products add them in.
    std::vector<std::vector<std::pair<size_t, double>>> units(pairs.size());
    for (size_t q = 0; q < pairs.size(); q++) {
        auto [a, b] = pairs[q];
        V3 e = unit(sub(at[b], at[a]));
        auto& u = units[q];
        for (int half = 0; half < 2; half++) {
            size_t r0 = half == 0 ? 3 * a : 3 * b;
            for (size_t r = 0; r < 3; r++) {
                // row r0 + r: column blocks a then b (a < b), + on the diagonal block
                for (int side = 0; side < 2; side++) {
                    size_t c0 = side == 0 ? 3 * a : 3 * b;
                    double sign = (side == half) ? 1.0 : -1.0;
                    for (size_t c = 0; c < 3; c++) {
                        double v = e[r] * e[c];
                        u.push_back({(r0 + r) * n + c0 + c, sign > 0 ? 0.0 + v : 0.0 - v});
                    }
                }
            }
        }
    }
    s.target.resize(n * n);
    for (size_t i = 0; i < n * n; i++) s.target[i] = 0.5 * (k[(i / n) * n + i % n] + k[(i % n) * n + i / n]);
    auto udot = [](const std::vector<std::pair<size_t, double>>& p, const std::vector<std::pair<size_t, double>>& q) {
        double acc = 0.0;
        size_t i = 0, j = 0;
        while (i < p.size() && j < q.size()) {
            if (p[i].first < q[j].first)
                i++;
            else if (q[j].first < p[i].first)
                j++;
            else {
                acc += p[i].second * q[j].second;
                i++;
                j++;
            }
        }
        return acc;
    };
    std::vector<bool> on(pairs.size(), true);
    std::vector<size_t> idx;
    for (;;) {
        idx.clear();
        for (size_t p = 0; p < pairs.size(); p++)
            if (on[p]) idx.push_back(p);
        const size_t m = idx.size();
        s.g.assign(m * (m + 1), 0.0);
        for (size_t r = 0; r < m; r++) {
            for (size_t c = 0; c < m; c++) s.g[r * (m + 1) + c] = udot(units[idx[r]], units[idx[c]]);
            double acc = 0.0;
            for (const auto& [f, v] : units[idx[r]]) acc += v * s.target[f];
            s.g[r * (m + 1) + m] = acc;
        }
        eliminate(s.g, m, 1, s.row, s.sol);
        int64_t worst = -1;  // the most negative, the first of equals
        for (size_t r = 0; r < m; r++)
            if (s.sol[r] < 0.0 && (worst < 0 || total_key(s.sol[r]) < total_key(s.sol[(size_t)worst]))) worst = (int64_t)r;
        if (worst >= 0) {
            on[idx[(size_t)worst]] = false;
            continue;
        }
        std::vector<std::tuple<size_t, size_t, double>> out;
        for (size_t r = 0; r < m; r++)
            if (s.sol[r] > 0.0) out.emplace_back(pairs[idx[r]].first, pairs[idx[r]].second, s.sol[r]);
        return out;
    }
}

// gather.rs:58-114 and 321-361: one cell measured. `at` = its handles' positions.
std::vector<Beam> measure_cell(const CellProblem& cp, const std::vector<V3>& at, const Mat& mat, const Full& full,
                               V3 middle, double s, bool against_full, Scratch& sc) {
    const size_t nf = cp.nf, nh = at.size(), n = 6 * nf, m = 3 * nh, w = n + m, nb = cp.bonds.size();
    auto column = [&](size_t v, size_t d, V3 p) -> V3 {
        V3 e{0.0, 0.0, 0.0};
        e[d % 3] = 1.0;
        return d < 3 ? e : cross(e, sub(p, cp.place[v]));
    };
    auto dof = [&](size_t v, size_t d) -> int64_t {
        if (v < nf) return (int64_t)(6 * v + d);
        if (d < 3) return (int64_t)(n + 3 * (v - nf) + d);
        return -1;
    };
    // The free parts' rows: their stiffness, the handles' columns on the right side.
    sc.a.assign(n * w, 0.0);
    for (const LBond& b : cp.bonds) {
        const double k = b.a / b.d;
        V3 srow[3];
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) {
                double nn = b.n[r] * b.n[c];
                srow[r][c] = b.e * k * nn + b.g * k * ((r == c ? 1.0 : 0.0) - nn);
            }
        const std::pair<size_t, double> ends[2] = {{b.i, -1.0}, {b.j, 1.0}};
        for (const auto& [v, sv] : ends)
            for (size_t d = 0; d < 6; d++) {
                int64_t r = dof(v, d);
                if (r < 0 || (size_t)r >= n) continue;
                V3 cv = column(v, d, b.p);
                V3 scv{dot(srow[0], cv), dot(srow[1], cv), dot(srow[2], cv)};
                for (const auto& [u, su] : ends)
                    for (size_t e = 0; e < 6; e++) {
                        int64_t c = dof(u, e);
                        if (c < 0) continue;
                        double sign = (size_t)c < n ? 1.0 : -1.0;
                        sc.a[(size_t)r * w + (size_t)c] += sign * sv * su * dot(scv, column(u, e, b.p));
                    }
            }
    }
    eliminate(sc.a, n, m, sc.row, sc.x);
    // Each handle axis moved alone: the finer bonds' forces (bodies.rs:420-423), case-major.
    sc.forces.resize(m * nb * 3);
    for (size_t c = 0; c < m; c++) {
        auto motion_at = [&](size_t v, V3 p) -> V3 {
            V3 t{0.0, 0.0, 0.0}, r{0.0, 0.0, 0.0};
            if (v < nf) {
                for (int q = 0; q < 3; q++) {
                    t[q] = sc.x[(6 * v + q) * m + c];
                    r[q] = sc.x[(6 * v + 3 + q) * m + c];
                }
            } else if (v - nf == c / 3) {
                t[c % 3] = 1.0;
            }
            return add(t, cross(r, sub(p, cp.place[v])));  // bodies.rs:44-47
        };
        for (size_t q = 0; q < nb; q++) {
            const LBond& b = cp.bonds[q];
            V3 f = b.force(sub(motion_at(b.j, b.p), motion_at(b.i, b.p)));
            for (int t = 0; t < 3; t++) sc.forces[(c * nb + q) * 3 + t] = f[t];
        }
    }
    auto force = [&](size_t c, size_t q) -> V3 {
        const double* f = &sc.forces[(c * nb + q) * 3];
        return {f[0], f[1], f[2]};
    };
    // The stiffness between handles: what holds each, each case.
    sc.k.assign(m * m, 0.0);
    for (size_t c = 0; c < m; c++)
        for (size_t q = 0; q < nb; q++) {
            V3 f = force(c, q);
            const std::pair<size_t, double> sides[2] = {{cp.bonds[q].j, 1.0}, {cp.bonds[q].i, -1.0}};
            for (const auto& [v, sign] : sides)
                if (v >= nf)
                    for (size_t t = 0; t < 3; t++) sc.k[(3 * (v - nf) + t) * m + c] += sign * f[t];
        }
    // Which handles the cell's matter joins (gather.rs:43-51).
    std::vector<size_t> parent(nf + nh);
    for (size_t t = 0; t < parent.size(); t++) parent[t] = t;
    for (const LBond& b : cp.bonds) {
        size_t x = find(parent, b.i), y = find(parent, b.j);
        parent[x] = y;
    }
    std::vector<size_t> piece(nh);
    for (size_t h = 0; h < nh; h++) piece[h] = find(parent, nf + h);
    std::vector<Beam> found;
    std::vector<V3> pulled(nb);
    for (const auto& [a, b, stiff] : fit_beams(sc.k, at, [&](size_t p, size_t q) { return piece[p] == piece[q]; }, sc)) {
        // The beam pulled alone, a unit apart; each finer bond as much as it holds of
        // the work done.
        V3 e = unit(sub(at[b], at[a]));
        for (size_t q = 0; q < nb; q++) {
            V3 f{0.0, 0.0, 0.0};
            for (size_t t = 0; t < 3; t++)
                f = add(f, add(mul(force(3 * b + t, q), e[t] / 2.0), mul(force(3 * a + t, q), -e[t] / 2.0)));
            pulled[q] = f;
        }
        double hold = 0.0, work = 0.0;
        for (size_t q = 0; q < nb; q++) {
            double u = cp.bonds[q].used(pulled[q]);
            double wq = cp.bonds[q].energy(pulled[q]);
            hold += wq * u;
            work += wq;
        }
        double fine_used = work > 0.0 ? hold / work : 0.0;
        double length = norm(sub(at[b], at[a]));
        double own = mat.used(mat.e / length, 0.0);
        double stronger = fine_used > 0.0 ? own / fine_used : 1.0;
        size_t cls = beam_class(at[a], at[b], middle);
        double section = stiff * length / mat.e / (s * s);
        if (against_full) section = section * SECTION[cls] / full[cls].first;
        found.push_back(Beam{a, b, section * s * s * mat.e / length, stronger / full[cls].second});
    }
    return found;
}

// ---- one cell as the phases of a thread block ---------------------------------------
// The same measurement as measure_cell, written for a CTA: every phase a loop strided by
// the thread index, a barrier between phases, each entry still summed in bond order by
// one thread, and the reductions (the pivot, the most negative beam) taken in a fixed
// order. The kernel runs it with GF_THREADS threads a cell; the host can run it with one
// thread (gf_emulate), the same code with no barriers, so the CPU can check it against
// the reference's order bit for bit. The file is compiled without contraction of
// multiplies and adds (-fmad=false), so the device rounds each operation as the host
// does. Sizes: a cell of a lattice that build (lattice.rs:124-163) or a gather made has
// at most 12 free parts (the inner faces of 2 x 2 x 2 finer cells), 6 handles and 480
// finer bonds (8 finer cells of 15 beams of 4 bonds).
constexpr int GF_MAXF = 12, GF_MAXH = 6, GF_MAXB = 480, GF_MAXP = 15;
constexpr int GF_MAXN = 6 * GF_MAXF, GF_MAXM = 3 * GF_MAXH, GF_MAXW = GF_MAXN + GF_MAXM;
constexpr int GF_THREADS = 256;

#ifdef __CUDA_ARCH__
#define GF_TID ((int)threadIdx.x)
#define GF_NT ((int)blockDim.x)
#define GF_LANES 32
#define GF_SYNC() __syncthreads()
#else
#define GF_TID 0
#define GF_NT 1
#define GF_LANES 1
#define GF_SYNC() ((void)0)
#endif

struct D3 {
    double v[3];
};
__host__ __device__ inline D3 d3(double a, double b, double c) { return D3{{a, b, c}}; }
__host__ __device__ inline D3 d_add(D3 a, D3 b) { return d3(a.v[0] + b.v[0], a.v[1] + b.v[1], a.v[2] + b.v[2]); }
__host__ __device__ inline D3 d_sub(D3 a, D3 b) { return d3(a.v[0] - b.v[0], a.v[1] - b.v[1], a.v[2] - b.v[2]); }
__host__ __device__ inline D3 d_mul(D3 a, double s) { return d3(a.v[0] * s, a.v[1] * s, a.v[2] * s); }
__host__ __device__ inline double d_dot(D3 a, D3 b) { return a.v[0] * b.v[0] + a.v[1] * b.v[1] + a.v[2] * b.v[2]; }
__host__ __device__ inline D3 d_cross(D3 a, D3 b) {
    return d3(a.v[1] * b.v[2] - a.v[2] * b.v[1], a.v[2] * b.v[0] - a.v[0] * b.v[2], a.v[0] * b.v[1] - a.v[1] * b.v[0]);
}
__host__ __device__ inline double d_norm(D3 a) { return sqrt(d_dot(a, a)); }
__host__ __device__ inline D3 d_unit(D3 a) { return d_mul(a, 1.0 / d_norm(a)); }
__host__ __device__ inline int64_t d_total_key(double v) {
#ifdef __CUDA_ARCH__
    int64_t i = __double_as_longlong(v);
#else
    int64_t i;
    std::memcpy(&i, &v, 8);
#endif
    return i ^ (int64_t)(((uint64_t)(i >> 63)) >> 1);
}

// A finer bond: its point, direction, section, length, E, G, strengths.
struct GBond {
    double p[3], n[3], a, d, e, g, ft, fc, fs;
};
// The finer lattice's bonds as the caller holds them (structure of arrays).
struct BondsSoA {
    const double *p, *n, *a, *d, *e, *g, *ft, *fc, *fs;
    __host__ __device__ GBond at(int64_t b) const {
        GBond r;
        for (int k = 0; k < 3; k++) {
            r.p[k] = p[3 * b + k];
            r.n[k] = n[3 * b + k];
        }
        r.a = a[b];
        r.d = d[b];
        r.e = e[b];
        r.g = g[b];
        r.ft = ft[b];
        r.fc = fc[b];
        r.fs = fs[b];
        return r;
    }
};

__host__ __device__ inline D3 gb_force(const GBond& b, D3 delta) {  // model.rs:115-119
    D3 n = d3(b.n[0], b.n[1], b.n[2]);
    double along = d_dot(delta, n);
    double k = b.a / b.d;
    return d_add(d_mul(n, b.e * k * along), d_mul(d_sub(delta, d_mul(n, along)), b.g * k));
}
__host__ __device__ inline double mat_used5(const double* m, double s1, double s3) {  // model.rs:66-68
    return fmax(fmax(s1 / m[2], -s3 / m[3]), (s1 - s3) / (2.0 * m[4]));
}
__host__ __device__ inline double gb_used(const GBond& b, D3 f) {  // model.rs:123-129
    D3 n = d3(b.n[0], b.n[1], b.n[2]);
    D3 t = d_mul(f, 1.0 / b.a);
    double sigma = d_dot(t, n);
    double tau2 = fmax(d_dot(t, t) - sigma * sigma, 0.0);
    double r = sqrt(sigma * sigma / 4.0 + tau2);
    const double m[5] = {b.e, b.g, b.ft, b.fc, b.fs};
    return mat_used5(m, sigma / 2.0 + r, sigma / 2.0 - r);
}
__host__ __device__ inline double gb_energy(const GBond& b, D3 f) {  // model.rs:132-136
    D3 n = d3(b.n[0], b.n[1], b.n[2]);
    double k = b.a / b.d;
    double along = d_dot(f, n);
    return 0.5 * (along * along / (b.e * k) + (d_dot(f, f) - along * along) / (b.g * k));
}

// One packed cell: nf free parts, nh handles, nb finer bonds (local ends in ij, the bond
// itself at bix in the finer lattice), the places' positions (free parts', then
// handles'), the cell's material (E, G, ft, fc, fs), the full cell's calibration (section
// and strength per class), its centre.
struct CellArgs {
    int nf, nh, nb, against_full;
    const uint8_t* ij;
    const int64_t* bix;
    BondsSoA fine;
    const double* place;
    const double* mat;
    const double* full;
    const double* middle;
    double s;
};

struct CellSmem {
    double a[GF_MAXN * GF_MAXW];
    double x[GF_MAXN * GF_MAXM];
    double k[GF_MAXM * GF_MAXM];
    double target[GF_MAXM * GF_MAXM];
    double f[GF_MAXN];
    double g[GF_MAXP * (GF_MAXP + 1)];
    double sol[GF_MAXP];
    double hold[GF_MAXB], work[GF_MAXB];
    double place[3 * (GF_MAXF + GF_MAXH)];
    double uval[GF_MAXP * 36];
    double fk[GF_MAXP];
    double scale;
    int32_t row[GF_MAXN];
    int32_t grow[GF_MAXP];
    int16_t uidx[GF_MAXP * 36];
    int32_t pa[GF_MAXP], pb[GF_MAXP], idx[GF_MAXP], fa[GF_MAXP], fb[GF_MAXP];
    int32_t parent[GF_MAXF + GF_MAXH], piece[GF_MAXH];
    int32_t npairs, mon, nfound, skip, more;
    uint8_t on[GF_MAXP];
    uint8_t ij[2 * GF_MAXB];
};

// gather.rs:164-184 on a small row-major n x (n + rhs) matrix, by one thread (the beams'
// normal equations): as eliminate above, with the row permutation in `row`.
__host__ __device__ inline void gf_eliminate_small(double* a, int n, int rhs, int32_t* row, double* x) {
    const int w = n + rhs;
    double scale = 0.0;
    for (int r = 0; r < n; r++) scale = fmax(scale, fabs(a[r * w + r]));
    for (int r = 0; r < n; r++) row[r] = r;
    for (int c = 0; c < n; c++) {
        int p = c;
        int64_t best = d_total_key(fabs(a[row[c] * w + c]));
        for (int q = c + 1; q < n; q++) {
            int64_t k = d_total_key(fabs(a[row[q] * w + c]));
            if (k >= best) {
                best = k;
                p = q;
            }
        }
        int32_t t = row[c];
        row[c] = row[p];
        row[p] = t;
        const double* piv = &a[row[c] * w];
        if (fabs(piv[c]) <= 1e-12 * scale) continue;
        for (int r = 0; r < n; r++) {
            if (r == c) continue;
            double* ar = &a[row[r] * w];
            double f = ar[c] / piv[c];
            if (f != 0.0)
                for (int k = c; k < w; k++) ar[k] -= f * piv[k];
        }
    }
    for (int r = 0; r < n; r++) {
        const double* ar = &a[row[r] * w];
        for (int k = 0; k < rhs; k++) x[r * rhs + k] = fabs(ar[r]) <= 1e-12 * scale ? 0.0 : ar[n + k] / ar[r];
    }
}

__host__ __device__ inline int32_t gf_find(int32_t* p, int32_t a) {  // bodies.rs:628-634
    while (p[a] != a) {
        p[a] = p[p[a]];
        a = p[a];
    }
    return a;
}

// The cell's beams into out_ab (a, b per beam), out_ks (stiffness along it, strength
// factor per beam) and *out_count. F: the finer bonds' forces, m x nb x 3 doubles.
__host__ __device__ void gf_measure_cell(const CellArgs& A, CellSmem& S, double* F, int32_t* out_ab, double* out_ks,
                                         int32_t* out_count) {
    const int tid = GF_TID, nt = GF_NT;
    const int nf = A.nf, nh = A.nh, nb = A.nb, n = 6 * nf, m = 3 * nh, w = n + m, np = nf + nh;
    for (int t = tid; t < 3 * np; t += nt) S.place[t] = A.place[t];
    for (int t = tid; t < 2 * nb; t += nt) S.ij[t] = A.ij[t];
    for (int t = tid; t < n * w; t += nt) S.a[t] = 0.0;
    GF_SYNC();
    auto pos = [&](int v) { return d3(S.place[3 * v], S.place[3 * v + 1], S.place[3 * v + 2]); };
    auto column = [&](int v, int d, D3 p) -> D3 {
        D3 e = d3(0.0, 0.0, 0.0);
        e.v[d % 3] = 1.0;
        return d < 3 ? e : d_cross(e, d_sub(p, pos(v)));
    };
    // gather.rs:84-101: the free parts' rows, a thread a row, each entry in bond order.
    for (int r = tid; r < n; r += nt) {
        const int v = r / 6, d = r % 6;
        double* ar = &S.a[r * w];
        for (int q = 0; q < nb; q++) {
            const int bi = S.ij[2 * q], bj = S.ij[2 * q + 1];
            if (bi != v && bj != v) continue;
            const GBond B = A.fine.at(A.bix[q]);
            const double k = B.a / B.d;
            D3 srow[3];
            for (int rr = 0; rr < 3; rr++)
                for (int cc = 0; cc < 3; cc++) {
                    double nn = B.n[rr] * B.n[cc];
                    srow[rr].v[cc] = B.e * k * nn + B.g * k * ((rr == cc ? 1.0 : 0.0) - nn);
                }
            const D3 p = d3(B.p[0], B.p[1], B.p[2]);
            const int ends[2] = {bi, bj};
            const double sgn[2] = {-1.0, 1.0};
            for (int s1 = 0; s1 < 2; s1++) {
                if (ends[s1] != v) continue;
                const double sv = sgn[s1];
                D3 cv = column(v, d, p);
                D3 scv = d3(d_dot(srow[0], cv), d_dot(srow[1], cv), d_dot(srow[2], cv));
                for (int s2 = 0; s2 < 2; s2++) {
                    const int u = ends[s2];
                    const double su = sgn[s2];
                    for (int e = 0; e < 6; e++) {
                        int c;
                        if (u < nf)
                            c = 6 * u + e;
                        else if (e < 3)
                            c = n + 3 * (u - nf) + e;
                        else
                            continue;
                        double sign = c < n ? 1.0 : -1.0;
                        ar[c] += sign * sv * su * d_dot(scv, column(u, e, p));
                    }
                }
            }
        }
    }
    GF_SYNC();
    // gather.rs:164-184: Gauss–Jordan over the free parts, every handle axis at once.
    if (tid == 0) {
        double sc = 0.0;
        for (int r = 0; r < n; r++) sc = fmax(sc, fabs(S.a[r * w + r]));
        S.scale = sc;
    }
    for (int r = tid; r < n; r += nt) S.row[r] = r;
    GF_SYNC();
    const double small = 1e-12 * S.scale;
    for (int c = 0; c < n; c++) {
        // the largest |a| at or below the diagonal, the last of equals: the largest
        // (key, position), by the first warp (one lane on the host)
        if (tid < GF_LANES) {
            int64_t bk = INT64_MIN;
            int32_t bp = -1;
            for (int q = c + tid; q < n; q += GF_LANES) {
                int64_t k = d_total_key(fabs(S.a[S.row[q] * w + c]));
                if (k > bk || (k == bk && q > bp)) {
                    bk = k;
                    bp = q;
                }
            }
#ifdef __CUDA_ARCH__
            for (int off = 16; off > 0; off >>= 1) {
                const int64_t ok = __shfl_down_sync(0xffffffffu, bk, off);
                const int32_t op = __shfl_down_sync(0xffffffffu, bp, off);
                if (op >= 0 && (ok > bk || (ok == bk && op > bp))) {
                    bk = ok;
                    bp = op;
                }
            }
#endif
            if (tid == 0) {
                int32_t t = S.row[c];
                S.row[c] = S.row[bp];
                S.row[bp] = t;
                S.skip = fabs(S.a[S.row[c] * w + c]) <= small ? 1 : 0;
            }
        }
        GF_SYNC();
        if (S.skip) continue;
        const double* piv = &S.a[S.row[c] * w];
        for (int r = tid; r < n; r += nt) S.f[r] = r == c ? 0.0 : S.a[S.row[r] * w + c] / piv[c];
        GF_SYNC();
        const int cols = w - c;
        for (int t = tid; t < n * cols; t += nt) {
            const int r = t / cols, k = c + t % cols;
            const double f = S.f[r];
            if (r == c || f == 0.0) continue;
            S.a[S.row[r] * w + k] -= f * piv[k];
        }
        GF_SYNC();
    }
    for (int t = tid; t < n * m; t += nt) {
        const int r = t / m, k = t % m;
        const double* ar = &S.a[S.row[r] * w];
        S.x[t] = fabs(ar[r]) <= small ? 0.0 : ar[n + k] / ar[r];
    }
    GF_SYNC();
    // Each handle axis moved alone: the finer bonds' forces (bodies.rs:420-423).
    for (int t = tid; t < m * nb; t += nt) {
        const int c = t / nb, q = t % nb;
        const GBond B = A.fine.at(A.bix[q]);
        const D3 p = d3(B.p[0], B.p[1], B.p[2]);
        auto motion_at = [&](int v) -> D3 {
            D3 tr = d3(0.0, 0.0, 0.0), ro = d3(0.0, 0.0, 0.0);
            if (v < nf) {
                for (int z = 0; z < 3; z++) {
                    tr.v[z] = S.x[(6 * v + z) * m + c];
                    ro.v[z] = S.x[(6 * v + 3 + z) * m + c];
                }
            } else if (v - nf == c / 3) {
                tr.v[c % 3] = 1.0;
            }
            return d_add(tr, d_cross(ro, d_sub(p, pos(v))));  // bodies.rs:44-47
        };
        D3 f = gb_force(B, d_sub(motion_at(S.ij[2 * q + 1]), motion_at(S.ij[2 * q])));
        for (int z = 0; z < 3; z++) F[(size_t)(c * nb + q) * 3 + z] = f.v[z];
    }
    GF_SYNC();
    // The stiffness between handles (gather.rs:322-333), each entry in bond order.
    for (int t = tid; t < m * m; t += nt) {
        const int r = t / m, c = t % m, h = r / 3, z = r % 3;
        double acc = 0.0;
        for (int q = 0; q < nb; q++) {
            const double fz = F[(size_t)(c * nb + q) * 3 + z];
            if (S.ij[2 * q + 1] == nf + h) acc += 1.0 * fz;
            if (S.ij[2 * q] == nf + h) acc += -1.0 * fz;
        }
        S.k[r * m + c] = acc;
    }
    GF_SYNC();
    // Which handles the matter joins (gather.rs:43-51); the pairs it joins (gather.rs:121-122).
    if (tid == 0) {
        for (int t = 0; t < np; t++) S.parent[t] = t;
        for (int q = 0; q < nb; q++) {
            int32_t a = gf_find(S.parent, S.ij[2 * q]), b = gf_find(S.parent, S.ij[2 * q + 1]);
            S.parent[a] = b;
        }
        for (int h = 0; h < nh; h++) S.piece[h] = gf_find(S.parent, nf + h);
        int np2 = 0;
        for (int a = 0; a < nh; a++)
            for (int b = a + 1; b < nh; b++)
                if (S.piece[a] == S.piece[b]) {
                    S.pa[np2] = a;
                    S.pb[np2] = b;
                    S.on[np2] = 1;
                    np2++;
                }
        S.npairs = np2;
    }
    GF_SYNC();
    auto at = [&](int h) { return pos(nf + h); };
    // A unit of each beam's stiffness (gather.rs:125-139): four 3x3 blocks, in flat order.
    for (int q = tid; q < S.npairs; q += nt) {
        const int a = S.pa[q], b = S.pb[q];
        D3 e = d_unit(d_sub(at(b), at(a)));
        int j = 0;
        for (int half = 0; half < 2; half++) {
            const int r0 = half == 0 ? 3 * a : 3 * b;
            for (int r = 0; r < 3; r++)
                for (int side = 0; side < 2; side++) {
                    const int c0 = side == 0 ? 3 * a : 3 * b;
                    for (int c = 0; c < 3; c++) {
                        double v = e.v[r] * e.v[c];
                        S.uidx[q * 36 + j] = (int16_t)((r0 + r) * m + c0 + c);
                        S.uval[q * 36 + j] = side == half ? 0.0 + v : 0.0 - v;
                        j++;
                    }
                }
        }
    }
    for (int t = tid; t < m * m; t += nt) S.target[t] = 0.5 * (S.k[(t / m) * m + t % m] + S.k[(t % m) * m + t / m]);
    GF_SYNC();
    // Least squares, dropping the most negative beam till none is (gather.rs:143-160).
    for (;;) {
        if (tid == 0) {
            int c = 0;
            for (int q = 0; q < S.npairs; q++)
                if (S.on[q]) S.idx[c++] = q;
            S.mon = c;
        }
        GF_SYNC();
        const int mo = S.mon;
        for (int t = tid; t < mo * (mo + 1); t += nt) {
            const int r = t / (mo + 1), c = t % (mo + 1);
            const double* pv = &S.uval[S.idx[r] * 36];
            const int16_t* pi = &S.uidx[S.idx[r] * 36];
            double acc = 0.0;
            if (c < mo) {
                const double* qv = &S.uval[S.idx[c] * 36];
                const int16_t* qi = &S.uidx[S.idx[c] * 36];
                int i = 0, j = 0;
                while (i < 36 && j < 36) {
                    if (pi[i] < qi[j])
                        i++;
                    else if (qi[j] < pi[i])
                        j++;
                    else {
                        acc += pv[i] * qv[j];
                        i++;
                        j++;
                    }
                }
            } else {
                for (int i = 0; i < 36; i++) acc += pv[i] * S.target[pi[i]];
            }
            S.g[r * (mo + 1) + c] = acc;
        }
        GF_SYNC();
        if (tid == 0) {
            gf_eliminate_small(S.g, mo, 1, S.grow, S.sol);
            int worst = -1;
            for (int r = 0; r < mo; r++)
                if (S.sol[r] < 0.0 && (worst < 0 || d_total_key(S.sol[r]) < d_total_key(S.sol[worst]))) worst = r;
            if (worst >= 0) {
                S.on[S.idx[worst]] = 0;
                S.more = 1;
            } else {
                int c = 0;
                for (int r = 0; r < mo; r++)
                    if (S.sol[r] > 0.0) {
                        S.fa[c] = S.pa[S.idx[r]];
                        S.fb[c] = S.pb[S.idx[r]];
                        S.fk[c] = S.sol[r];
                        c++;
                    }
                S.nfound = c;
                S.more = 0;
            }
        }
        GF_SYNC();
        if (!S.more) break;
    }
    // Each beam pulled alone, a unit apart (gather.rs:337-361).
    const int nfound = S.nfound;
    for (int bm = 0; bm < nfound; bm++) {
        const int a = S.fa[bm], b = S.fb[bm];
        const D3 e = d_unit(d_sub(at(b), at(a)));
        for (int q = tid; q < nb; q += nt) {
            D3 f = d3(0.0, 0.0, 0.0);
            for (int z = 0; z < 3; z++) {
                const double* fb_ = &F[(size_t)((3 * b + z) * nb + q) * 3];
                const double* fa_ = &F[(size_t)((3 * a + z) * nb + q) * 3];
                f = d_add(f, d_add(d_mul(d3(fb_[0], fb_[1], fb_[2]), e.v[z] / 2.0),
                                   d_mul(d3(fa_[0], fa_[1], fa_[2]), -e.v[z] / 2.0)));
            }
            const GBond B = A.fine.at(A.bix[q]);
            const double u = gb_used(B, f);
            const double wq = gb_energy(B, f);
            S.hold[q] = wq * u;
            S.work[q] = wq;
        }
        GF_SYNC();
        if (tid == 0) {
            double hold = 0.0, work = 0.0;
            for (int q = 0; q < nb; q++) {
                hold += S.hold[q];
                work += S.work[q];
            }
            const double fine_used = work > 0.0 ? hold / work : 0.0;
            const double length = d_norm(d_sub(at(b), at(a)));
            const double own = mat_used5(A.mat, A.mat[0] / length, 0.0);
            const double stronger = fine_used > 0.0 ? own / fine_used : 1.0;
            const D3 mid = d3(A.middle[0], A.middle[1], A.middle[2]);
            const D3 u1 = d_sub(at(a), mid), u2 = d_sub(at(b), mid);
            const int cls = (int)round(1.0 + d_dot(u1, u2) / (d_norm(u1) * d_norm(u2)));  // lattice.rs:29-32
            double section = S.fk[bm] * length / A.mat[0] / (A.s * A.s);
            if (A.against_full) section = section * 0.336 / A.full[2 * cls];  // SECTION, lattice.rs:25
            out_ab[2 * bm] = a;
            out_ab[2 * bm + 1] = b;
            out_ks[2 * bm] = section * A.s * A.s * A.mat[0] / length;
            out_ks[2 * bm + 1] = stronger / A.full[2 * cls + 1];
        }
        GF_SYNC();
    }
    if (tid == 0) *out_count = nfound;
}

// One CTA a cell at a time over the batch; F: each CTA's own forces scratch.
struct CellBatchView {
    int32_t ncells, against_full;
    double s;
    const int32_t *nf, *nh;
    const int64_t *bond_ptr, *place_ptr;
    const uint8_t* ij;
    const int64_t* bix;
    BondsSoA fine;
    const double *place, *mat, *full, *middle;
    int32_t *out_ab, *out_count;
    double* out_ks;
    __host__ __device__ CellArgs cell(int c) const {
        CellArgs A;
        A.nf = nf[c];
        A.nh = nh[c];
        A.nb = (int)(bond_ptr[c + 1] - bond_ptr[c]);
        A.against_full = against_full;
        A.ij = ij + 2 * bond_ptr[c];
        A.bix = bix + bond_ptr[c];
        A.fine = fine;
        A.place = place + 3 * place_ptr[c];
        A.mat = mat + 5 * (size_t)c;
        A.full = full + 4 * (size_t)c;
        A.middle = middle + 3 * (size_t)c;
        A.s = s;
        return A;
    }
};

__global__ void __launch_bounds__(GF_THREADS) k_gather_cells(CellBatchView B, double* scratch) {
    extern __shared__ __align__(16) unsigned char gf_smem[];
    CellSmem& S = *reinterpret_cast<CellSmem*>(gf_smem);
    double* F = scratch + (size_t)blockIdx.x * GF_MAXM * GF_MAXB * 3;
    for (int c = blockIdx.x; c < B.ncells; c += gridDim.x) {
        gf_measure_cell(B.cell(c), S, F, B.out_ab + 2 * GF_MAXP * (size_t)c, B.out_ks + 2 * GF_MAXP * (size_t)c,
                        B.out_count + c);
        __syncthreads();
    }
}

struct FineView {
    int level;
    int64_t nn, nb;
    const double *x, *m;
    const uint8_t* held;
    const int64_t* around;
    const int32_t* mat;
    const int64_t *bi, *bj;
    const double *p, *n, *a, *d, *e, *g, *ft, *fc, *fs;
    Site site(int64_t v, int s) const { return {around[6 * v + 3 * s], around[6 * v + 3 * s + 1], around[6 * v + 3 * s + 2]}; }
};

struct SiteHash {
    size_t operator()(const Site& s) const {
        uint64_t h = 1469598103934665603ull;
        for (int k = 0; k < 3; k++) h = (h ^ (uint64_t)s[k]) * 1099511628211ull;
        return (size_t)(h ^ (h >> 29));
    }
};

Full full_of(const Mat& mat);

// SC_TIMING=1: each phase's host milliseconds on stderr.
struct HostPhases {
    bool on = std::getenv("SC_TIMING") != nullptr;
    std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
    void mark(const char* phase) {
        if (!on) return;
        auto now = std::chrono::steady_clock::now();
        std::fprintf(stderr, "[gather] %-10s %8.2f ms\n", phase, std::chrono::duration<double, std::milli>(now - t).count());
        t = now;
    }
};

// f(lo, hi) over [0, n) in T contiguous ranges on T threads (f must not throw); one
// range below `least` items.
template <class Fn>
void split(size_t n, size_t T, Fn f, size_t least = 4096) {
    if (T <= 1 || n < least) {
        f(0, n);
        return;
    }
    std::vector<std::thread> pool;
    for (size_t t = 1; t < T; t++) pool.emplace_back(f, n * t / T, n * (t + 1) / T);
    f(0, n / T);
    for (auto& th : pool) th.join();
}

// The cells to measure, packed for gf_measure_cell: a cell's finer bonds and places
// contiguous, its material, calibration and centre beside them.
struct CellBatch {
    std::vector<int32_t> which, nf, nh;
    std::vector<int64_t> bond_ptr{0}, place_ptr{0};
    std::vector<uint8_t> ij;
    std::vector<int64_t> bix;
    BondsSoA fine{};
    std::vector<double> place, mat, full, middle;
    CellBatchView view(double s, bool against_full) {
        CellBatchView v{};
        v.ncells = (int32_t)which.size();
        v.against_full = against_full ? 1 : 0;
        v.s = s;
        v.nf = nf.data();
        v.nh = nh.data();
        v.bond_ptr = bond_ptr.data();
        v.place_ptr = place_ptr.data();
        v.ij = ij.data();
        v.bix = bix.data();
        v.fine = fine;
        v.place = place.data();
        v.mat = mat.data();
        v.full = full.data();
        v.middle = middle.data();
        return v;
    }
};

// gf_measure_cell over the batch on the device: one CTA a cell at a time, as many CTAs as
// fit on the GPU at once, each with its own forces scratch.
void measure_on_device(Context& ctx, CellBatch& cb, int64_t fine_bonds, double s, bool against_full,
                       std::vector<int32_t>& ab, std::vector<double>& ks, std::vector<int32_t>& count) {
    const int ncells = (int)cb.which.size();
    if (!ncells) return;
    cudaStream_t st = ctx.stream;
    auto up = [&](auto& buf, const auto& host) {
        buf.alloc(std::max<size_t>(host.size(), 1), st, &ctx.mem);
        buf.upload(host.data(), host.size());
    };
    DBuf<int32_t> nf, nh, oab, ocount;
    DBuf<int64_t> bptr, pptr, bix;
    DBuf<uint8_t> ij;
    DBuf<double> place, mat, full, middle, oks, scratch;
    up(nf, cb.nf);
    up(nh, cb.nh);
    up(bptr, cb.bond_ptr);
    up(pptr, cb.place_ptr);
    up(ij, cb.ij);
    up(bix, cb.bix);
    // the finer bonds straight from the caller's arrays
    DBuf<double> fb[9];
    const double* src[9] = {cb.fine.p, cb.fine.n, cb.fine.a, cb.fine.d, cb.fine.e,
                            cb.fine.g, cb.fine.ft, cb.fine.fc, cb.fine.fs};
    for (int k = 0; k < 9; k++) {
        const size_t count = (k < 2 ? 3 : 1) * (size_t)fine_bonds;
        fb[k].alloc(std::max<size_t>(count, 1), st, &ctx.mem);
        fb[k].upload(src[k], count);
    }
    up(place, cb.place);
    up(mat, cb.mat);
    up(full, cb.full);
    up(middle, cb.middle);
    oab.alloc((size_t)ncells * 2 * GF_MAXP, st, &ctx.mem);
    oks.alloc((size_t)ncells * 2 * GF_MAXP, st, &ctx.mem);
    ocount.alloc((size_t)ncells, st, &ctx.mem);
    const size_t smem = sizeof(CellSmem);
    SC_CK(cudaFuncSetAttribute(k_gather_cells, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int sms = 0, per = 0;
    SC_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device));
    SC_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_gather_cells, GF_THREADS, smem));
    require(per > 0, SC_CUDA, "the cell measurement does not fit on an SM");
    const int grid = std::min(ncells, sms * per);
    scratch.alloc((size_t)grid * GF_MAXM * GF_MAXB * 3, st, &ctx.mem);
    CellBatchView v{};
    v.ncells = ncells;
    v.against_full = against_full ? 1 : 0;
    v.s = s;
    v.nf = nf.get();
    v.nh = nh.get();
    v.bond_ptr = bptr.get();
    v.place_ptr = pptr.get();
    v.ij = ij.get();
    v.bix = bix.get();
    v.fine = BondsSoA{fb[0].get(), fb[1].get(), fb[2].get(), fb[3].get(), fb[4].get(),
                      fb[5].get(), fb[6].get(), fb[7].get(), fb[8].get()};
    v.place = place.get();
    v.mat = mat.get();
    v.full = full.get();
    v.middle = middle.get();
    v.out_ab = oab.get();
    v.out_ks = oks.get();
    v.out_count = ocount.get();
    const bool timing = std::getenv("SC_TIMING") != nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (timing) {
        SC_CK(cudaEventCreate(&e0));
        SC_CK(cudaEventCreate(&e1));
        SC_CK(cudaEventRecord(e0, st));
    }
    k_gather_cells<<<grid, GF_THREADS, smem, st>>>(v, scratch.get());
    SC_LAUNCH_CK();
    if (timing) {
        SC_CK(cudaEventRecord(e1, st));
        SC_CK(cudaEventSynchronize(e1));
        float ms = 0.0f;
        SC_CK(cudaEventElapsedTime(&ms, e0, e1));
        std::fprintf(stderr, "[gather] kernel     %8.3f ms (%d cells, %d blocks of %d threads, %zu B shared)\n", ms,
                     ncells, grid, GF_THREADS, smem);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    ab.resize((size_t)ncells * 2 * GF_MAXP);
    ks.resize((size_t)ncells * 2 * GF_MAXP);
    count.resize((size_t)ncells);
    oab.download(ab.data(), ab.size());
    oks.download(ks.data(), ks.size());
    ocount.download(count.data(), count.size());
    SC_CK(cudaStreamSynchronize(st));
}

// gf_measure_cell over the batch on the host's cores, one thread a cell (the kernel's
// code with one thread and no barriers).
void measure_emulated(CellBatch& cb, double s, bool against_full, size_t threads, std::vector<int32_t>& ab,
                      std::vector<double>& ks, std::vector<int32_t>& count) {
    const size_t ncells = cb.which.size();
    ab.assign(ncells * 2 * GF_MAXP, 0);
    ks.assign(ncells * 2 * GF_MAXP, 0.0);
    count.assign(ncells, 0);
    CellBatchView v = cb.view(s, against_full);
    v.out_ab = ab.data();
    v.out_ks = ks.data();
    v.out_count = count.data();
    std::atomic<size_t> next{0};
    auto work = [&] {
        auto S = std::make_unique<CellSmem>();
        std::vector<double> F((size_t)GF_MAXM * GF_MAXB * 3);
        for (size_t c; (c = next.fetch_add(1)) < ncells;)
            gf_measure_cell(v.cell((int)c), *S, F.data(), v.out_ab + 2 * GF_MAXP * c, v.out_ks + 2 * GF_MAXP * c,
                            v.out_count + c);
    };
    std::vector<std::thread> pool;
    for (size_t t = 1; t < threads; t++) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
}

// gather.rs:230-395. `dev`: measure the cells on that context's device; else on the
// host's cores (SC_GATHER_EMULATE set: with the device's code, one thread a cell).
void measured(const FineView& F, const std::vector<Mat>& table, bool against_full, int threads, Gathered& out,
              Context* dev = nullptr) {
    HostPhases ph;
    const int level = F.level + 1;
    std::unordered_map<Site, size_t, SiteHash> index;
    std::vector<Site> sites;
    auto cell_of = [&](const Site& s) {
        Site key = coarse_site(s, level);
        auto it = index.find(key);
        if (it != index.end()) return it->second;
        sites.push_back(key);
        index.emplace(key, sites.size() - 1);
        return sites.size() - 1;
    };
    std::vector<std::array<size_t, 2>> between((size_t)F.nn);
    for (int64_t v = 0; v < F.nn; v++) {
        size_t x = cell_of(F.site(v, 0));
        size_t y = cell_of(F.site(v, 1));
        between[(size_t)v] = {x, y};
    }
    ph.mark("cells");
    const size_t T = threads > 0 ? (size_t)threads : std::max<size_t>(1, std::thread::hardware_concurrency());
    // The site a bond's ends share is one of its first end's, whose coarse cell the node
    // pass above has numbered already: no bond adds a cell. Bond by bond, over the threads.
    std::vector<size_t> lies((size_t)F.nb);
    std::atomic<bool> apart{false};
    split((size_t)F.nb, T, [&](size_t lo, size_t hi) {
        for (size_t b = lo; b < hi; b++) {
            int64_t i = F.bi[b], j = F.bj[b];
            Site si[2] = {F.site(i, 0), F.site(i, 1)}, sj[2] = {F.site(j, 0), F.site(j, 1)};
            int k = (si[0] == sj[0] || si[0] == sj[1]) ? 0 : (si[1] == sj[0] || si[1] == sj[1]) ? 1 : -1;
            if (k < 0) {
                apart = true;
                return;
            }
            lies[b] = between[(size_t)i][k];
        }
    });
    require(!apart, SC_BAD_INPUT, "a bond whose ends share no cell");
    ph.mark("lies");
    const size_t n = sites.size();
    auto face = [&](size_t a, size_t b) { return sites[a] < sites[b] ? std::make_pair(a, b) : std::make_pair(b, a); };
    // Faces: every (cell, cell across) a node lies between or a bond reaches, in key order.
    std::vector<std::pair<size_t, size_t>> keys;
    for (int64_t v = 0; v < F.nn; v++)
        if (between[(size_t)v][0] != between[(size_t)v][1]) keys.push_back(face(between[(size_t)v][0], between[(size_t)v][1]));
    // Cells: free parts in node order, materials by first appearance, their weight summed
    // in node order (gather.rs:263-279).
    std::vector<std::vector<size_t>> free(n);
    std::vector<std::vector<std::pair<int32_t, double>>> mats(n);
    auto weigh = [](std::vector<std::pair<int32_t, double>>& list, int32_t mat, double w) {
        for (auto& e : list)
            if (e.first == mat) {
                e.second += w;
                return;
            }
        list.push_back({mat, w});
    };
    for (int64_t v = 0; v < F.nn; v++) {
        size_t x = between[(size_t)v][0], y = between[(size_t)v][1];
        weigh(mats[x], F.mat[v], F.m[v]);
        if (x != y) weigh(mats[y], F.mat[v], F.m[v]);
        if (x == y) free[x].push_back((size_t)v);
    }
    std::vector<size_t> place((size_t)F.nn, SIZE_MAX);
    for (size_t c = 0; c < n; c++)
        for (size_t k = 0; k < free[c].size(); k++) place[free[c][k]] = k;
    // Each bond into its cell's problem; handles numbered by first use (gather.rs:285-294).
    // The bonds grouped by cell in bond order (a stable counting sort), then each cell's
    // walked in that order on its own thread: the same handles as one pass over all bonds.
    // Each thread counts its own range of bonds; within a cell, a thread's bonds go after
    // the threads' before it, so the grouping keeps bond order.
    std::vector<int64_t> bptr(n + 1, 0), bord((size_t)F.nb);
    {
        const size_t nb = (size_t)F.nb, TT = nb < 65536 ? 1 : T;
        std::vector<std::vector<int64_t>> cnt(TT, std::vector<int64_t>(n, 0));
        auto range = [&](size_t t) { return std::make_pair(nb * t / TT, nb * (t + 1) / TT); };
        auto each_thread = [&](auto fn) {
            std::vector<std::thread> pool;
            for (size_t t = 1; t < TT; t++) pool.emplace_back(fn, t);
            fn(0);
            for (auto& th : pool) th.join();
        };
        each_thread([&](size_t t) {
            auto [lo, hi] = range(t);
            for (size_t b = lo; b < hi; b++) cnt[t][lies[b]]++;
        });
        int64_t at = 0;  // each (cell, thread)'s first slot, cells in order, threads in order
        for (size_t c = 0; c < n; c++) {
            bptr[c] = at;
            for (size_t t = 0; t < TT; t++) {
                int64_t k = cnt[t][c];
                cnt[t][c] = at;
                at += k;
            }
        }
        bptr[n] = at;
        each_thread([&](size_t t) {
            auto [lo, hi] = range(t);
            for (size_t b = lo; b < hi; b++) bord[(size_t)cnt[t][lies[b]]++] = (int64_t)b;
        });
    }
    ph.mark("group");
    std::vector<uint32_t> bli((size_t)F.nb), blj((size_t)F.nb);  // each grouped bond's local ends
    std::vector<std::vector<size_t>> across(n);
    split(n, T, [&](size_t lo, size_t hi) {
        for (size_t c = lo; c < hi; c++) {
            auto at = [&](int64_t v) {
                size_t x = between[(size_t)v][0], y = between[(size_t)v][1];
                if (x == c && y == c) return place[(size_t)v];
                size_t other = x == c ? y : x;
                auto& ac = across[c];
                size_t k = (size_t)(std::find(ac.begin(), ac.end(), other) - ac.begin());
                if (k == ac.size()) ac.push_back(other);
                return free[c].size() + k;
            };
            for (int64_t q = bptr[c]; q < bptr[c + 1]; q++) {
                const int64_t b = bord[(size_t)q];
                bli[(size_t)q] = (uint32_t)at(F.bi[b]);
                blj[(size_t)q] = (uint32_t)at(F.bj[b]);
            }
        }
    }, 64);
    ph.mark("handles");
    std::vector<uint8_t> held(n);
    for (size_t c = 0; c < n; c++) {
        bool all = !free[c].empty();
        for (size_t v : free[c]) all = all && F.held[v];
        held[c] = all;
    }
    for (size_t c = 0; c < n; c++)
        for (size_t o : across[c]) keys.push_back(face(c, o));
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    auto node_of = [&](size_t a, size_t b) {
        return (size_t)(std::lower_bound(keys.begin(), keys.end(), face(a, b)) - keys.begin());
    };
    const size_t nn = keys.size();
    std::vector<double> fmass(nn, 0.0);
    std::vector<uint8_t> fheld(nn, 0);
    for (int64_t v = 0; v < F.nn; v++) {
        size_t x = between[(size_t)v][0], y = between[(size_t)v][1];
        if (x == y) continue;
        size_t k = node_of(x, y);
        fmass[k] += F.m[v];
        fheld[k] = fheld[k] || F.held[v];
    }
    auto mat_of = [&](std::initializer_list<size_t> cs) -> int32_t {  // gather.rs:301-310
        std::vector<std::pair<int32_t, double>> all;
        for (size_t c : cs)
            for (const auto& [mt, wt] : mats[c]) weigh(all, mt, wt);
        if (all.empty()) return -1;  // STONE
        size_t best = 0;
        for (size_t k = 1; k < all.size(); k++)
            if (total_key(all[k].second) >= total_key(all[best].second)) best = k;
        return all[best].first;
    };
    out.level = level;
    out.x.resize(3 * nn);
    out.m.resize(nn);
    out.held.resize(nn);
    out.around.resize(6 * nn);
    out.mat.resize(nn);
    for (size_t k = 0; k < nn; k++) {
        auto [a, b] = keys[k];
        V3 x = mul(add(centre(sites[a], level), centre(sites[b], level)), 0.5);
        for (int t = 0; t < 3; t++) {
            out.x[3 * k + t] = x[t];
            out.around[6 * k + t] = sites[a][t];
            out.around[6 * k + 3 + t] = sites[b][t];
        }
        out.m[k] = fmass[k];
        out.mat[k] = mat_of({a, b});
        out.held[k] = fheld[k] || held[a] || held[b];
    }
    const double s = spacing(level);
    std::vector<std::vector<size_t>> ends(n);
    std::vector<std::vector<V3>> at(n);
    std::vector<int32_t> cmat(n);
    for (size_t c = 0; c < n; c++) {
        for (size_t o : across[c]) {
            size_t k = node_of(c, o);
            ends[c].push_back(k);
            at[c].push_back({out.x[3 * k], out.x[3 * k + 1], out.x[3 * k + 2]});
        }
        cmat[c] = mat_of({c});
    }
    // A cell without matter of a known material measures as stone (gather.rs:310); the
    // table's first entry stands for it only where such a cell has beams to measure.
    auto mat_value = [&](int32_t k) -> const Mat& { return table[(size_t)std::max<int32_t>(k, 0)]; };
    ph.mark("index");
    std::vector<Full> fulls(n, Full{std::make_pair(1.0, 1.0), std::make_pair(1.0, 1.0)});
    if (against_full)
        for (size_t c = 0; c < n; c++)
            if (!held[c] && !at[c].empty()) fulls[c] = full_of(mat_value(cmat[c]));
    // Every cell measured, over the host's threads (cells are independent).
    ph.mark("full");
    std::vector<std::vector<Beam>> found(n);
    auto work = [&](size_t lo, size_t hi) {
        Scratch scr;
        CellProblem cp;
        for (size_t c = lo; c < hi; c++) {
            if (held[c] || at[c].empty()) continue;
            cp.nf = free[c].size();
            cp.place.clear();
            for (size_t v : free[c]) cp.place.push_back({F.x[3 * v], F.x[3 * v + 1], F.x[3 * v + 2]});
            for (const V3& h : at[c]) cp.place.push_back(h);
            cp.bonds.clear();
            for (int64_t q = bptr[c]; q < bptr[c + 1]; q++) {
                const size_t b = (size_t)bord[(size_t)q];
                cp.bonds.push_back(LBond{bli[(size_t)q], blj[(size_t)q], {F.p[3 * b], F.p[3 * b + 1], F.p[3 * b + 2]},
                                         {F.n[3 * b], F.n[3 * b + 1], F.n[3 * b + 2]}, F.a[b], F.d[b], F.e[b], F.g[b],
                                         F.ft[b], F.fc[b], F.fs[b]});
            }
            found[c] = measure_cell(cp, at[c], mat_value(cmat[c]), fulls[c], centre(sites[c], level), s, against_full,
                                    scr);
        }
    };
    const bool emulate = !dev && std::getenv("SC_GATHER_EMULATE") != nullptr;
    if (dev || emulate) {
        CellBatch cb;
        cb.fine = BondsSoA{F.p, F.n, F.a, F.d, F.e, F.g, F.ft, F.fc, F.fs};
        cb.ij.reserve(2 * (size_t)F.nb);
        cb.bix.reserve((size_t)F.nb);
        for (size_t c = 0; c < n; c++) {
            if (held[c] || at[c].empty()) continue;
            const size_t nf = free[c].size(), nh = at[c].size(), nb = (size_t)(bptr[c + 1] - bptr[c]);
            require(nf <= GF_MAXF && nh <= GF_MAXH && nb <= GF_MAXB, SC_BAD_INPUT,
                    "a coarse cell holds more finer parts, faces or bonds than a built lattice's");
            cb.which.push_back((int32_t)c);
            cb.nf.push_back((int32_t)nf);
            cb.nh.push_back((int32_t)nh);
            for (size_t v : free[c])
                for (int t = 0; t < 3; t++) cb.place.push_back(F.x[3 * v + t]);
            for (const V3& h : at[c])
                for (int t = 0; t < 3; t++) cb.place.push_back(h[t]);
            cb.place_ptr.push_back(cb.place_ptr.back() + (int64_t)(nf + nh));
            for (int64_t q = bptr[c]; q < bptr[c + 1]; q++) {
                cb.ij.push_back((uint8_t)bli[(size_t)q]);
                cb.ij.push_back((uint8_t)blj[(size_t)q]);
                cb.bix.push_back(bord[(size_t)q]);
            }
            cb.bond_ptr.push_back(cb.bond_ptr.back() + (int64_t)nb);
            const Mat& mt = mat_value(cmat[c]);
            for (double v : {mt.e, mt.g, mt.ft, mt.fc, mt.fs}) cb.mat.push_back(v);
            for (int k = 0; k < 2; k++) {
                cb.full.push_back(fulls[c][k].first);
                cb.full.push_back(fulls[c][k].second);
            }
            V3 mid = centre(sites[c], level);
            for (int t = 0; t < 3; t++) cb.middle.push_back(mid[t]);
        }
        ph.mark("pack");
        std::vector<int32_t> ab, count;
        std::vector<double> ks;
        if (dev)
            measure_on_device(*dev, cb, F.nb, s, against_full, ab, ks, count);
        else
            measure_emulated(cb, s, against_full, T, ab, ks, count);
        for (size_t i = 0; i < cb.which.size(); i++) {
            auto& fc = found[(size_t)cb.which[i]];
            for (int bm = 0; bm < count[i]; bm++)
                fc.push_back(Beam{(size_t)ab[2 * GF_MAXP * i + 2 * bm], (size_t)ab[2 * GF_MAXP * i + 2 * bm + 1],
                                  ks[2 * GF_MAXP * i + 2 * bm], ks[2 * GF_MAXP * i + 2 * bm + 1]});
        }
    } else if (n < 64 || T == 1) {
        work(0, n);
    } else {
        // Interleaved blocks of cells: a level's cells with matter cluster by first
        // appearance, so contiguous halves would leave threads idle.
        std::vector<std::thread> pool;
        const size_t chunk = 16;
        std::atomic<size_t> next{0};
        for (size_t t = 0; t < T; t++)
            pool.emplace_back([&] {
                for (;;) {
                    size_t lo = next.fetch_add(chunk);
                    if (lo >= n) return;
                    work(lo, std::min(n, lo + chunk));
                }
            });
        for (auto& th : pool) th.join();
    }
    ph.mark("measure");
    // Each cell's weight on its faces, as much as each is joined (gather.rs:370-381): a
    // face takes from its two cells in cell order, so this stays one pass.
    std::vector<int64_t> first(n + 1, 0);  // each cell's first bond of the level
    for (size_t c = 0; c < n; c++) {
        double mass = 0.0;
        for (size_t v : free[c]) mass += F.m[v];
        const size_t nh = at[c].size();
        std::vector<double> joined(nh, 0.0);
        for (const Beam& bm : found[c]) {
            joined[bm.a] += bm.k;
            joined[bm.b] += bm.k;
        }
        double total = 0.0;
        for (double j : joined) total += j;
        for (size_t h = 0; h < nh; h++) out.m[ends[c][h]] += mass * (total > 0.0 ? joined[h] / total : 1.0 / (double)nh);
        int64_t kept = 0;
        for (const Beam& bm : found[c]) kept += (out.held[ends[c][bm.a]] && out.held[ends[c][bm.b]]) ? 0 : 4;
        first[c + 1] = first[c] + kept;
    }
    // Its beams (gather.rs:382-391), every cell's into its own slots, over the threads.
    const size_t nbo = (size_t)first[n];
    out.bi.resize(nbo);
    out.bj.resize(nbo);
    out.bmat.resize(nbo);
    out.p.resize(3 * nbo);
    out.n.resize(3 * nbo);
    for (auto* v : {&out.a, &out.d, &out.e, &out.g, &out.ft, &out.fc, &out.fs}) v->resize(nbo);
    split(n, T, [&](size_t lo, size_t hi) {
        for (size_t c = lo; c < hi; c++) {
            size_t q = (size_t)first[c];
            const Mat& mt = mat_value(cmat[c]);
            for (const Beam& bm : found[c]) {
                size_t ia = ends[c][bm.a], ib = ends[c][bm.b];
                if (out.held[ia] && out.held[ib]) continue;
                V3 pa = at[c][bm.a], pb = at[c][bm.b];
                double length = norm(sub(pb, pa));
                double area = bm.k * length / mt.e;
                // lattice.rs:76-84: four bonds at radius sqrt(A / 2 pi) about the middle
                V3 nrm = unit(sub(pb, pa));
                V3 e1 = unit(cross(nrm, std::fabs(nrm[0]) < 0.9 ? V3{1.0, 0.0, 0.0} : V3{0.0, 1.0, 0.0}));
                V3 e2 = cross(nrm, e1);
                double r = std::sqrt(area / (2.0 * PI));
                V3 middle = mul(add(pa, pb), 0.5);
                double d = norm(sub(pb, pa));
                const V3 offs[4] = {mul(e1, r), mul(e1, -r), mul(e2, r), mul(e2, -r)};
                for (const V3& o : offs) {
                    V3 p = add(middle, o);
                    out.bi[q] = (int64_t)ia;
                    out.bj[q] = (int64_t)ib;
                    out.bmat[q] = std::max<int32_t>(cmat[c], 0);
                    for (int t = 0; t < 3; t++) {
                        out.p[3 * q + t] = p[t];
                        out.n[3 * q + t] = nrm[t];
                    }
                    out.a[q] = area / 4.0;
                    out.d[q] = d;
                    out.e[q] = mt.e;
                    out.g[q] = mt.g;
                    out.ft[q] = mt.ft * bm.stronger;  // Mat::stronger, model.rs:71-73
                    out.fc[q] = mt.fc * bm.stronger;
                    out.fs[q] = mt.fs * bm.stronger;
                    q++;
                }
            }
        }
    }, 64);
    ph.mark("assemble");
}

// A full block of `mat` at level 0, 6 cells a side about the origin, all free, as
// lattice.rs:87-163 builds it (sites x-major, then y, then z; nodes by first touch; the
// 15 beams of a cell in face-pair order).
struct Block {
    std::vector<double> x, m, p, n, a, d, e, g, ft, fc, fs;
    std::vector<uint8_t> held;
    std::vector<int64_t> around, bi, bj;
    std::vector<int32_t> mat;
};

Block full_block(const Mat& mt) {
    static const int FACES[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    Block B;
    const double s = spacing(0);
    std::unordered_map<uint64_t, size_t> index;
    auto pack = [](const Site& a, const Site& b) {
        uint64_t h = 0;
        for (int k = 0; k < 3; k++) h = h * 64 + (uint64_t)(a[k] + 16);
        for (int k = 0; k < 3; k++) h = h * 64 + (uint64_t)(b[k] + 16);
        return h;
    };
    for (int64_t i = -3; i < 3; i++)
        for (int64_t j = -3; j < 3; j++)
            for (int64_t k = -3; k < 3; k++) {
                Site site{i, j, k};
                size_t ends[6];
                for (int f = 0; f < 6; f++) {
                    Site other{i + FACES[f][0], j + FACES[f][1], k + FACES[f][2]};
                    Site lo = site < other ? site : other, hi = site < other ? other : site;
                    uint64_t key = pack(lo, hi);
                    auto it = index.find(key);
                    if (it == index.end()) {
                        V3 x = mul(add(centre(site, 0), centre(other, 0)), 0.5);
                        for (int t = 0; t < 3; t++) {
                            B.x.push_back(x[t]);
                            B.around.push_back(lo[t]);
                        }
                        for (int t = 0; t < 3; t++) B.around.push_back(hi[t]);
                        B.m.push_back(0.0);
                        B.held.push_back(0);
                        B.mat.push_back(0);
                        it = index.emplace(key, B.m.size() - 1).first;
                    }
                    B.m[it->second] += 1.0 / 6.0;
                    ends[f] = it->second;
                }
                V3 middle = centre(site, 0);
                for (int fa = 0; fa < 6; fa++)
                    for (int fb = fa + 1; fb < 6; fb++) {
                        size_t ia = ends[fa], ib = ends[fb];
                        V3 pa{B.x[3 * ia], B.x[3 * ia + 1], B.x[3 * ia + 2]};
                        V3 pb{B.x[3 * ib], B.x[3 * ib + 1], B.x[3 * ib + 2]};
                        double area = SECTION[beam_class(pa, pb, middle)] * s * s;
                        V3 nrm = unit(sub(pb, pa));
                        V3 e1 = unit(cross(nrm, std::fabs(nrm[0]) < 0.9 ? V3{1.0, 0.0, 0.0} : V3{0.0, 1.0, 0.0}));
                        V3 e2 = cross(nrm, e1);
                        double r = std::sqrt(area / (2.0 * PI));
                        V3 mid = mul(add(pa, pb), 0.5);
                        double d = norm(sub(pb, pa));
                        const V3 offs[4] = {mul(e1, r), mul(e1, -r), mul(e2, r), mul(e2, -r)};
                        for (const V3& o : offs) {
                            V3 p = add(mid, o);
                            B.bi.push_back((int64_t)ia);
                            B.bj.push_back((int64_t)ib);
                            for (int t = 0; t < 3; t++) {
                                B.p.push_back(p[t]);
                                B.n.push_back(nrm[t]);
                            }
                            B.a.push_back(area / 4.0);
                            B.d.push_back(d);
                            B.e.push_back(mt.e);
                            B.g.push_back(mt.g);
                            B.ft.push_back(mt.ft);
                            B.fc.push_back(mt.fc);
                            B.fs.push_back(mt.fs);
                        }
                    }
            }
    return B;
}

// gather.rs:203-226: a full cell of `mat` measured a level up, by class: its beams'
// section over the spacing squared and strength over the material's, kept per material.
Full full_of(const Mat& mt) {
    static std::mutex lock;
    static std::vector<std::pair<Mat, Full>> known;
    {
        std::lock_guard<std::mutex> g(lock);
        for (const auto& [k, f] : known)
            if (std::memcmp(&k, &mt, sizeof(Mat)) == 0) return f;
    }
    Block B = full_block(mt);
    FineView F{0, (int64_t)B.m.size(), (int64_t)B.bi.size(), B.x.data(), B.m.data(), B.held.data(), B.around.data(),
               B.mat.data(), B.bi.data(), B.bj.data(), B.p.data(), B.n.data(), B.a.data(), B.d.data(), B.e.data(),
               B.g.data(), B.ft.data(), B.fc.data(), B.fs.data()};
    Gathered coarse;
    measured(F, std::vector<Mat>{mt}, false, 1, coarse);
    const double s = spacing(1);
    double sum[2][3] = {{0, 0, 0}, {0, 0, 0}};
    auto touches = [&](size_t v) {
        const int64_t* a = &coarse.around[6 * v];
        return (a[0] == 0 && a[1] == 0 && a[2] == 0) || (a[3] == 0 && a[4] == 0 && a[5] == 0);
    };
    for (size_t q = 0; q + 4 <= coarse.bi.size(); q += 4) {
        size_t i = (size_t)coarse.bi[q], j = (size_t)coarse.bj[q];
        if (touches(i) && touches(j)) {
            V3 xi{coarse.x[3 * i], coarse.x[3 * i + 1], coarse.x[3 * i + 2]};
            V3 xj{coarse.x[3 * j], coarse.x[3 * j + 1], coarse.x[3 * j + 2]};
            size_t k = beam_class(xi, xj, centre(Site{0, 0, 0}, 1));
            sum[k][0] += 4.0 * coarse.a[q] / (s * s);
            sum[k][1] += coarse.ft[q] / mt.ft;
            sum[k][2] += 1.0;
        }
    }
    Full f;
    for (int k = 0; k < 2; k++)
        f[k] = sum[k][2] > 0.0 ? std::make_pair(sum[k][0] / sum[k][2], sum[k][1] / sum[k][2]) : std::make_pair(1.0, 1.0);
    std::lock_guard<std::mutex> g(lock);
    known.push_back({mt, f});
    return f;
}

}  // namespace gth

void gather_level(Context* dev, const sc_lattice& L, const sc_strength& S, const int32_t* node_mat,
                  const sc_material* materials, int32_t n_materials, bool against_full, int32_t threads,
                  Gathered& out) {
    std::vector<gth::Mat> table((size_t)n_materials);
    for (int32_t k = 0; k < n_materials; k++)
        table[(size_t)k] = gth::Mat{materials[k].e, materials[k].g, materials[k].ft, materials[k].fc, materials[k].fs};
    gth::FineView F{L.level,  L.n_nodes,  L.n_bonds,  L.x,        S.m,        L.held,     L.around,
                    node_mat, L.bond_i,   L.bond_j,   L.bond_p,   L.bond_n,   L.bond_a,   L.bond_d,
                    L.bond_e, L.bond_g,   S.ft,       S.fc,       S.fs};
    gth::measured(F, table, against_full, threads, out, dev);
}

void gather_full(const sc_material& m, double* out) {
    auto f = gth::full_of(gth::Mat{m.e, m.g, m.ft, m.fc, m.fs});
    for (int k = 0; k < 2; k++) {
        out[2 * k] = f[k].first;
        out[2 * k + 1] = f[k].second;
    }
}

}  // namespace sc
