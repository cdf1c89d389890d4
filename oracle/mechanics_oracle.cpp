// ORACLE -- test infrastructure only: a CPU restatement of the engine's solver,
// mechanics::solve::Solver (mechanics/src/solve.rs:1-538), and of the unit cell element
// it is assembled from (mechanics/src/element.rs:15-69), for parity checks of a GPU port.
// Loops and sums keep the Rust source's order (built without FMA contraction). One
// difference: the coarse levels' pairs are kept in (a, c) order, where the reference
// collects them from a hash map (solve.rs:249-262) in the map's iteration order; the
// products over pairs then add in another order, equal up to rounding.
//
// Also a synthetic system of a voxel piece at rest, restating Matter::system
// (mechanics/src/lib.rs:638-676) and its node numbering and pair pattern
// (lib.rs:375-423): every free cell is an 8-node element welded to its free neighbours
// (corners at one lattice point are one node), corners touching a held cell are held.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <map>
#include <tuple>
#include <unordered_map>
#include <vector>

namespace mech {

typedef std::array<double, 3> V3;
typedef std::array<V3, 3> M3;
typedef std::array<double, 6> V6;
typedef std::array<V6, 6> M6;

constexpr int ROUNDS = 300;     // solve.rs:21
constexpr size_t DIRECT = 24;   // solve.rs:23
constexpr double NU = 0.3;      // element.rs:15
constexpr double GRAVITY = 9.81;  // lib.rs:23
constexpr double DAMPING = 0.3;   // lib.rs:63

static V3 add(V3 a, V3 b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
static V3 sub(V3 a, V3 b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
static V3 scale(V3 a, double s) { return {a[0] * s, a[1] * s, a[2] * s}; }
static double dot(V3 a, V3 b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static V3 cross(V3 a, V3 b) {
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
static V3 times(const M3& m, V3 v) { return {dot(m[0], v), dot(m[1], v), dot(m[2], v)}; }
static V3 times_t(const M3& m, V3 v) {
    V3 o;
    for (int c = 0; c < 3; c++) {
        double s = 0.0;
        for (int r = 0; r < 3; r++) s += m[r][c] * v[r];
        o[c] = s;
    }
    return o;
}

struct Pair {
    uint32_t i, j;
    M3 b;
};

// solve.rs:50-74
struct System {
    std::vector<std::array<int64_t, 3>> sites;
    std::vector<V3> at;
    std::vector<M3> diag;
    std::vector<Pair> pairs;
    void times(const std::vector<V3>& x, std::vector<V3>& y) const {
        for (size_t i = 0; i < diag.size(); i++) y[i] = mech::times(diag[i], x[i]);
        for (const Pair& p : pairs) {
            y[p.i] = add(y[p.i], mech::times(p.b, x[p.j]));
            y[p.j] = add(y[p.j], times_t(p.b, x[p.i]));
        }
    }
};

// solve.rs:77-94: T(r)' M T(s)
static M6 lift(const M6& m, V3 r, V3 s) {
    auto X = [](V3 v) -> M3 { return M3{V3{0.0, v[2], -v[1]}, V3{-v[2], 0.0, v[0]}, V3{v[1], -v[0], 0.0}}; };
    const M3 xr = X(r), xs = X(s);
    M6 t = m;
    for (int row = 0; row < 6; row++)
        for (int c = 0; c < 3; c++) {
            double acc = 0.0;
            for (int k = 0; k < 3; k++) acc += m[row][k] * xs[k][c];
            t[row][3 + c] += acc;
        }
    M6 out = t;
    for (int r3 = 0; r3 < 3; r3++)
        for (int col = 0; col < 6; col++) {
            double acc = 0.0;
            for (int k = 0; k < 3; k++) acc += xr[k][r3] * t[k][col];
            out[3 + r3][col] += acc;
        }
    return out;
}

static M6 embed(const M3& b) {
    M6 m{};
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) m[r][c] = b[r][c];
    return m;
}
static M6 transpose6(const M6& m) {
    M6 t;
    for (int r = 0; r < 6; r++)
        for (int c = 0; c < 6; c++) t[r][c] = m[c][r];
    return t;
}
static void plus6(M6& a, const M6& b) {
    for (int r = 0; r < 6; r++)
        for (int c = 0; c < 6; c++) a[r][c] += b[r][c];
}
static V6 times6(const M6& m, const V6& v) {
    V6 o;
    for (int r = 0; r < 6; r++) {
        double s = 0.0;
        for (int c = 0; c < 6; c++) s += m[r][c] * v[c];
        o[r] = s;
    }
    return o;
}
static V6 times6t(const M6& m, const V6& v) {
    V6 o;
    for (int r = 0; r < 6; r++) {
        double s = 0.0;
        for (int c = 0; c < 6; c++) s += m[c][r] * v[c];
        o[r] = s;
    }
    return o;
}

// solve.rs:138-165: L L' in place; which pivots were dropped
static std::vector<bool> cholesky(std::vector<double>& a, size_t n) {
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

// solve.rs:167-186
static void solve_cholesky(const std::vector<double>& a, const std::vector<bool>& dropped, size_t n, double* b) {
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

// solve.rs:123-135: out[c] = the solve for unit column c
template <size_t N>
static std::array<std::array<double, N>, N> inverse(const std::array<std::array<double, N>, N>& m) {
    std::vector<double> a(N * N);
    for (size_t r = 0; r < N; r++)
        for (size_t c = 0; c < N; c++) a[r * N + c] = m[r][c];
    std::vector<bool> l = cholesky(a, N);
    std::array<std::array<double, N>, N> out;
    for (size_t c = 0; c < N; c++) {
        std::vector<double> e(N, 0.0);
        e[c] = 1.0;
        solve_cholesky(a, l, N, e.data());
        for (size_t r = 0; r < N; r++) out[c][r] = e[r];
    }
    return out;
}

// solve.rs:211-238: union-find, ids by first appearance
static size_t find(std::vector<size_t>& up, size_t i) {
    while (up[i] != i) {
        up[i] = up[up[i]];
        i = up[i];
    }
    return i;
}
static void unite(std::vector<size_t>& up, size_t i, size_t j) {
    size_t r = find(up, i), s = find(up, j);
    up[std::max(r, s)] = std::min(r, s);
}
static std::vector<uint32_t> sets(size_t n, const std::vector<std::pair<size_t, size_t>>& joined, size_t& count) {
    std::vector<size_t> up(n);
    for (size_t i = 0; i < n; i++) up[i] = i;
    for (auto& p : joined) unite(up, p.first, p.second);
    std::vector<uint32_t> index(n, UINT32_MAX), of(n);
    count = 0;
    for (size_t i = 0; i < n; i++) {
        size_t root = find(up, i);
        if (index[root] == UINT32_MAX) index[root] = (uint32_t)count++;
        of[i] = index[root];
    }
    return of;
}

static int64_t div_euclid2(int64_t v) { return v >= 0 ? v / 2 : -((-v + 1) / 2); }
static std::array<int64_t, 3> parent(const std::array<int64_t, 3>& k) {
    return {div_euclid2(k[0]), div_euclid2(k[1]), div_euclid2(k[2])};
}

struct Pair6 {
    uint32_t p, q;
    M6 m;
};

// solve.rs:188-203
struct Coarse {
    std::vector<uint32_t> of;
    std::vector<V3> r;
    std::vector<std::array<int64_t, 3>> keys;
    std::vector<V3> centre;
    std::vector<M6> diag;
    std::vector<Pair6> pairs;
    std::vector<M6> inv;
    bool direct = false;
    std::vector<double> a;
    std::vector<bool> dropped;
    double size = 0.0, step = 1.0;

    void apply(const std::vector<V6>& x, std::vector<V6>& y) const {  // solve.rs:306-317
        for (size_t p = 0; p < diag.size(); p++) y[p] = times6(diag[p], x[p]);
        for (const Pair6& e : pairs) {
            V6 av = times6(e.m, x[e.q]), cv = times6t(e.m, x[e.p]);
            for (int k = 0; k < 6; k++) y[e.p][k] = y[e.p][k] + av[k];
            for (int k = 0; k < 6; k++) y[e.q][k] = y[e.q][k] + cv[k];
        }
    }
    void factor() {  // solve.rs:320-347
        size_t n = centre.size(), m = 6 * n;
        a.assign(36 * n * n, 0.0);
        for (size_t p = 0; p < n; p++) {
            const M6& d = diag[p];
            for (int r = 0; r < 6; r++)
                for (int c = 0; c < 6; c++) a[(6 * p + r) * m + 6 * p + c] += d[r][c];
            double t = (d[0][0] + d[1][1] + d[2][2]) / 3.0;
            for (int k = 3; k < 6; k++) a[(6 * p + k) * m + 6 * p + k] += 1e-6 * t * size * size;
        }
        for (const Pair6& e : pairs)
            for (int r = 0; r < 6; r++)
                for (int c = 0; c < 6; c++) {
                    a[(6 * e.p + r) * m + 6 * e.q + c] += e.m[r][c];
                    a[(6 * e.q + c) * m + 6 * e.p + r] += e.m[r][c];
                }
        dropped = cholesky(a, m);
        direct = true;
    }
};

// solve.rs:274-296: 4/3 over the largest eigenvalue of over(apply), by ten power steps
template <size_t N, class Apply, class Over>
static double step_of(size_t n, Apply apply, Over over) {
    typedef std::array<double, N> VN;
    auto norm = [](const std::vector<VN>& v) {
        double s = 0.0;
        for (const VN& e : v)
            for (double x : e) s += x * x;
        return std::sqrt(s);
    };
    std::vector<VN> v(n), a(n), w(n);
    for (size_t k = 0; k < n; k++)
        for (size_t s = 0; s < N; s++) v[k][s] = 1.0 + (double)((7 * k + 3 * s) % 11) / 11.0;
    for (size_t k = 0; k < n; k++) a[k].fill(0.0), w[k].fill(0.0);
    double most = 1.0;
    for (int it = 0; it < 10; it++) {
        apply(v, a);
        over(a, w);
        double nw = norm(w), nv = norm(v);
        if (nw == 0.0) break;
        most = nw / nv;
        for (size_t k = 0; k < n; k++)
            for (size_t s = 0; s < N; s++) v[k][s] = w[k][s] / nw;
    }
    return 4.0 / 3.0 / most;
}

// solve.rs:241-271
static Coarse coarsen(const std::vector<std::array<int64_t, 3>>& keys, const std::vector<V3>& at,
                      const std::vector<M6>& diag, const std::vector<Pair6>& pairs, double size) {
    std::vector<std::pair<size_t, size_t>> joined;
    for (const Pair6& e : pairs)
        if (parent(keys[e.p]) == parent(keys[e.q])) joined.push_back({e.p, e.q});
    size_t n = 0;
    Coarse c;
    c.of = sets(keys.size(), joined, n);
    c.centre.assign(n, V3{0.0, 0.0, 0.0});
    std::vector<double> count(n, 0.0);
    c.keys.assign(n, std::array<int64_t, 3>{0, 0, 0});
    for (size_t i = 0; i < c.of.size(); i++) {
        uint32_t a = c.of[i];
        c.centre[a] = add(c.centre[a], at[i]);
        count[a] += 1.0;
        c.keys[a] = parent(keys[i]);
    }
    for (size_t a = 0; a < n; a++) c.centre[a] = scale(c.centre[a], 1.0 / count[a]);
    c.r.resize(c.of.size());
    for (size_t i = 0; i < c.of.size(); i++) c.r[i] = sub(at[i], c.centre[c.of[i]]);
    c.diag.assign(n, M6{});
    for (size_t i = 0; i < diag.size(); i++) plus6(c.diag[c.of[i]], lift(diag[i], c.r[i], c.r[i]));
    std::map<std::pair<uint32_t, uint32_t>, M6> map;
    for (const Pair6& e : pairs) {
        uint32_t a = c.of[e.p], cc = c.of[e.q];
        M6 m = lift(e.m, c.r[e.p], c.r[e.q]);
        if (a == cc) {
            plus6(c.diag[a], m);
            plus6(c.diag[a], transpose6(m));
        } else if (a < cc) {
            auto it = map.emplace(std::make_pair(a, cc), M6{}).first;
            plus6(it->second, m);
        } else {
            auto it = map.emplace(std::make_pair(cc, a), M6{}).first;
            plus6(it->second, transpose6(m));
        }
    }
    for (auto& kv : map) c.pairs.push_back(Pair6{kv.first.first, kv.first.second, kv.second});
    c.inv.resize(n);
    for (size_t p = 0; p < n; p++) {
        M6 d = c.diag[p];
        double t = (d[0][0] + d[1][1] + d[2][2]) / 3.0;
        for (int k = 3; k < 6; k++) d[k][k] += 1e-6 * t * size * size;
        c.inv[p] = inverse<6>(d);
    }
    c.size = size;
    c.step = step_of<6>(
        n, [&](const std::vector<V6>& x, std::vector<V6>& y) { c.apply(x, y); },
        [&](const std::vector<V6>& x, std::vector<V6>& y) {
            for (size_t p = 0; p < n; p++) y[p] = times6(c.inv[p], x[p]);
        });
    if (n <= DIRECT) c.factor();
    return c;
}

// solve.rs:356-538
struct Solver {
    std::vector<M3> inv;
    double step = 1.0;
    std::vector<Coarse> levels;

    Solver(const System& s, double size) {
        inv.resize(s.diag.size());
        for (size_t i = 0; i < s.diag.size(); i++) inv[i] = inverse<3>(s.diag[i]);
        step = step_of<3>(
            s.sites.size(), [&](const std::vector<V3>& x, std::vector<V3>& y) { s.times(x, y); },
            [&](const std::vector<V3>& x, std::vector<V3>& y) {
                for (size_t i = 0; i < x.size(); i++) y[i] = mech::times(inv[i], x[i]);
            });
        std::vector<M6> diag(s.diag.size());
        for (size_t i = 0; i < s.diag.size(); i++) diag[i] = embed(s.diag[i]);
        std::vector<Pair6> pairs;
        for (const Pair& p : s.pairs) pairs.push_back(Pair6{p.i, p.j, embed(p.b)});
        Coarse next = coarsen(s.sites, s.at, diag, pairs, size * 2.0);
        for (;;) {
            size *= 2.0;
            size_t n = next.centre.size(), before = levels.empty() ? s.sites.size() : levels.back().centre.size();
            if (next.direct) {
                levels.push_back(std::move(next));
                break;
            }
            if (n == before) {
                next.factor();
                levels.push_back(std::move(next));
                break;
            }
            levels.push_back(std::move(next));
            const Coarse& l = levels.back();
            next = coarsen(l.keys, l.centre, l.diag, l.pairs, size * 2.0);
        }
    }

    std::vector<V6> cycle(size_t l, const std::vector<V6>& b) const {
        const Coarse& level = levels[l];
        size_t n = level.centre.size();
        if (level.direct) {
            std::vector<double> x(6 * n);
            for (size_t p = 0; p < n; p++)
                for (int k = 0; k < 6; k++) x[6 * p + k] = b[p][k];
            solve_cholesky(level.a, level.dropped, 6 * n, x.data());
            std::vector<V6> out(n);
            for (size_t p = 0; p < n; p++)
                for (int k = 0; k < 6; k++) out[p][k] = x[6 * p + k];
            return out;
        }
        auto apply = [&](const std::vector<V6>& x) {
            std::vector<V6> y(n, V6{});
            level.apply(x, y);
            return y;
        };
        auto smooth = [&](std::vector<V6>& x, const std::vector<V6>& r) {
            for (size_t p = 0; p < n; p++) {
                V6 d = times6(level.inv[p], r[p]);
                for (int k = 0; k < 6; k++) x[p][k] = x[p][k] + level.step * d[k];
            }
        };
        auto residual = [&](const std::vector<V6>& x) {
            std::vector<V6> y = apply(x);
            for (size_t p = 0; p < n; p++)
                for (int k = 0; k < 6; k++) y[p][k] = b[p][k] - y[p][k];
            return y;
        };
        std::vector<V6> x(n, V6{});
        smooth(x, b);
        std::vector<V6> r = residual(x);
        const Coarse& up = levels[l + 1];
        std::vector<V6> rb(up.centre.size(), V6{});
        for (size_t p = 0; p < n; p++) {
            size_t a = up.of[p];
            V3 rp = up.r[p];
            V3 t = cross(rp, V3{r[p][0], r[p][1], r[p][2]});
            for (int k = 0; k < 3; k++) {
                rb[a][k] += r[p][k];
                rb[a][3 + k] += r[p][3 + k] + t[k];
            }
        }
        std::vector<V6> e = cycle(l + 1, rb);
        for (size_t p = 0; p < n; p++) {
            size_t a = up.of[p];
            V3 u = cross(V3{e[a][3], e[a][4], e[a][5]}, up.r[p]);
            for (int k = 0; k < 3; k++) {
                x[p][k] += e[a][k] + u[k];
                x[p][3 + k] += e[a][3 + k];
            }
        }
        r = residual(x);
        smooth(x, r);
        return x;
    }

    void precondition(const System& s, const std::vector<V3>& b, std::vector<V3>& out, std::vector<V3>& scratch) const {
        size_t n = b.size();
        for (size_t i = 0; i < n; i++) out[i] = scale(mech::times(inv[i], b[i]), step);
        s.times(out, scratch);
        const Coarse& up = levels[0];
        std::vector<V6> rb(up.centre.size(), V6{});
        for (size_t i = 0; i < n; i++) {
            V3 r = sub(b[i], scratch[i]);
            size_t a = up.of[i];
            V3 t = cross(up.r[i], r);
            for (int k = 0; k < 3; k++) {
                rb[a][k] += r[k];
                rb[a][3 + k] += t[k];
            }
        }
        std::vector<V6> e = cycle(0, rb);
        for (size_t i = 0; i < n; i++) {
            size_t a = up.of[i];
            out[i] = add(out[i], add(V3{e[a][0], e[a][1], e[a][2]}, cross(V3{e[a][3], e[a][4], e[a][5]}, up.r[i])));
        }
        s.times(out, scratch);
        for (size_t i = 0; i < n; i++) out[i] = add(out[i], scale(mech::times(inv[i], sub(b[i], scratch[i])), step));
    }

    // rounds, or -1 where the levels do not fit s (not positive)
    int solve(const System& s, const std::vector<V3>& b, std::vector<V3>& x, double tolerance) const {
        size_t n = b.size();
        if (n == 0) return 0;
        auto measure = [](const std::vector<V3>& r, const std::vector<V3>& z) {
            double acc = 0.0;
            for (size_t i = 0; i < r.size(); i++) acc += dot(r[i], z[i]);
            return acc;
        };
        std::vector<V3> z(n, V3{0, 0, 0}), scratch(n, V3{0, 0, 0});
        precondition(s, b, z, scratch);
        double target = tolerance * tolerance * measure(b, z);
        if (std::isnan(target) || target < 0.0) return -1;
        std::vector<V3> ax(n, V3{0, 0, 0});
        s.times(x, ax);
        std::vector<V3> r(n);
        for (size_t i = 0; i < n; i++) r[i] = sub(b[i], ax[i]);
        precondition(s, r, z, scratch);
        std::vector<V3> p = z, ap(n, V3{0, 0, 0});
        double rz = measure(r, z);
        for (int round = 0; round < ROUNDS; round++) {
            if (rz < 0.0) return -1;
            if (rz <= target) return round;
            s.times(p, ap);
            double pap = 0.0;
            for (size_t i = 0; i < n; i++) pap += dot(p[i], ap[i]);
            if (pap <= 0.0) return round;
            double alpha = rz / pap;
            for (size_t i = 0; i < n; i++) {
                x[i] = add(x[i], scale(p[i], alpha));
                r[i] = sub(r[i], scale(ap[i], alpha));
            }
            precondition(s, r, z, scratch);
            double next = measure(r, z);
            double beta = next / rz;
            rz = next;
            for (size_t i = 0; i < n; i++) p[i] = add(z[i], scale(p[i], beta));
        }
        return ROUNDS;
    }
};

// ---- the unit cell element (element.rs:15-69) --------------------------------------
static const int CORNERS[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {1, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
static V3 sign_of(int c) {
    return {(double)(2 * CORNERS[c][0] - 1), (double)(2 * CORNERS[c][1] - 1), (double)(2 * CORNERS[c][2] - 1)};
}
// strain rows (xx, yy, zz, 2yz, 2xz, 2xy) of node a's motion at `at`
static std::array<V3, 6> strain(int a, V3 at) {
    V3 s = sign_of(a), g;
    for (int k = 0; k < 3; k++) {
        double prod = 1.0;
        for (int j = 0; j < 3; j++)
            if (j != k) prod *= 1.0 + s[j] * at[j];
        g[k] = s[k] / 4.0 * prod;
    }
    return {V3{g[0], 0.0, 0.0}, V3{0.0, g[1], 0.0}, V3{0.0, 0.0, g[2]},
            V3{0.0, g[2], g[1]}, V3{g[2], 0.0, g[0]}, V3{g[1], g[0], 0.0}};
}
static std::array<double, 6> stress_of(const std::array<double, 6>& e) {
    const double l = NU / ((1.0 + NU) * (1.0 - 2.0 * NU)), m = 1.0 / (2.0 * (1.0 + NU));
    const double tr = e[0] + e[1] + e[2];
    return {l * tr + 2.0 * m * e[0], l * tr + 2.0 * m * e[1], l * tr + 2.0 * m * e[2], m * e[3], m * e[4], m * e[5]};
}
typedef std::array<std::array<M3, 8>, 8> Unit;
static const Unit& unit() {
    static Unit k = [] {
        Unit k{};
        const double g = 1.0 / std::sqrt(3.0);
        for (int p = 0; p < 8; p++) {
            V3 s = sign_of(p), at = {s[0] * g, s[1] * g, s[2] * g};
            std::array<std::array<V3, 6>, 8> b;
            for (int a = 0; a < 8; a++) b[a] = strain(a, at);
            for (int a = 0; a < 8; a++)
                for (int c = 0; c < 8; c++)
                    for (int j = 0; j < 3; j++) {
                        std::array<double, 6> e;
                        for (int r = 0; r < 6; r++) e[r] = b[c][r][j];
                        std::array<double, 6> st = stress_of(e);
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

// ---- a voxel piece at rest as a system (lib.rs:375-423, 638-676) ---------------------
// state: 0 empty, 1 free, 2 held, x-major then y then z; e: per cell stiffness (E).
struct Built {
    System s;
    std::vector<V3> b;
};
static Built build(const uint8_t* state, const float* e, int nx, int ny, int nz, double h, double dt, double mass) {
    auto idx = [&](int x, int y, int z) { return ((int64_t)x * ny + y) * nz + z; };
    auto st = [&](int x, int y, int z) -> int {
        if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) return 0;
        return state[idx(x, y, z)];
    };
    // free cells in flat order; nodes by the first (cell, corner) that reaches them
    std::vector<std::array<int, 3>> cells;
    std::vector<float> ke;
    for (int x = 0; x < nx; x++)
        for (int y = 0; y < ny; y++)
            for (int z = 0; z < nz; z++)
                if (st(x, y, z) == 1) {
                    cells.push_back({x, y, z});
                    ke.push_back(e[idx(x, y, z)]);
                }
    const int64_t NX = nx + 1, NY = ny + 1, NZ = nz + 1;
    std::vector<int64_t> node_of((size_t)(NX * NY * NZ), -1);
    std::vector<std::array<int64_t, 3>> node_site;
    std::vector<double> node_mass;
    std::vector<bool> node_held;
    std::vector<std::array<uint32_t, 8>> corners(cells.size());
    for (size_t i = 0; i < cells.size(); i++)
        for (int c = 0; c < 8; c++) {
            int px = cells[i][0] + CORNERS[c][0], py = cells[i][1] + CORNERS[c][1], pz = cells[i][2] + CORNERS[c][2];
            int64_t g = (px * NY + py) * NZ + pz;
            if (node_of[g] < 0) {
                node_of[g] = (int64_t)node_site.size();
                node_site.push_back({px, py, pz});
                node_mass.push_back(0.0);
                // held where a held cell has this corner
                bool held = false;
                for (int dx = -1; dx <= 0; dx++)
                    for (int dy = -1; dy <= 0; dy++)
                        for (int dz = -1; dz <= 0; dz++) held = held || st(px + dx, py + dy, pz + dz) == 2;
                node_held.push_back(held);
            }
            corners[i][c] = (uint32_t)node_of[g];
            node_mass[node_of[g]] += mass / 8.0;
        }
    const uint32_t NONE = UINT32_MAX;
    std::vector<uint32_t> fr(node_site.size());
    uint32_t count = 0;
    for (size_t k = 0; k < node_site.size(); k++) fr[k] = node_held[k] ? NONE : count++;
    Built out;
    System& s = out.s;
    for (size_t k = 0; k < node_site.size(); k++) {
        if (fr[k] == NONE) continue;
        s.sites.push_back(node_site[k]);
        s.at.push_back(V3{node_site[k][0] * h, node_site[k][1] * h, node_site[k][2] * h});
        const double m = node_mass[k];
        s.diag.push_back(M3{V3{m, 0.0, 0.0}, V3{0.0, m, 0.0}, V3{0.0, 0.0, m}});  // block([1,0,0], m, m)
        out.b.push_back(scale(V3{0.0, -GRAVITY * dt, 0.0}, m));                 // v = 0
    }
    std::unordered_map<uint64_t, uint32_t> index;
    std::vector<std::array<uint32_t, 64>> slots(cells.size());
    const uint32_t TURNED = 1u << 31;
    for (size_t i = 0; i < cells.size(); i++) {
        slots[i].fill(NONE);
        for (int a = 0; a < 8; a++)
            for (int c = a + 1; c < 8; c++) {
                uint32_t p = fr[corners[i][a]], q = fr[corners[i][c]];
                if (p == NONE || q == NONE) continue;
                uint64_t key = ((uint64_t)std::min(p, q) << 32) | std::max(p, q);
                auto it = index.find(key);
                uint32_t k;
                if (it == index.end()) {
                    k = (uint32_t)s.pairs.size();
                    index.emplace(key, k);
                    s.pairs.push_back(Pair{std::min(p, q), std::max(p, q), M3{}});
                } else {
                    k = it->second;
                }
                slots[i][8 * a + c] = k | (p > q ? TURNED : 0u);
            }
    }
    const double stiff = dt * dt + DAMPING * dt;
    const Unit& K = unit();
    for (size_t i = 0; i < cells.size(); i++) {
        const double k = (double)ke[i] * h;
        for (int a = 0; a < 8; a++) {
            uint32_t p = fr[corners[i][a]];
            if (p != NONE)
                for (int r = 0; r < 3; r++)
                    for (int c = 0; c < 3; c++) s.diag[p][r][c] += K[a][a][r][c] * k * stiff;
            for (int c = a + 1; c < 8; c++) {
                uint32_t slot = slots[i][8 * a + c];
                if (slot == NONE) continue;
                M3& into = s.pairs[slot & ~TURNED].b;
                const bool turned = (slot & TURNED) != 0;
                for (int r = 0; r < 3; r++)
                    for (int cc = 0; cc < 3; cc++)
                        into[r][cc] += (turned ? K[a][c][cc][r] : K[a][c][r][cc]) * k * stiff;
            }
        }
    }
    return out;
}

}  // namespace mech

// ---- C entry points for the tests ---------------------------------------------------
extern "C" {

// K[a][c][i][j] of the unit cube (8 * 8 * 9 values)
void mo_unit_stiffness(double* k) {
    const mech::Unit& u = mech::unit();
    for (int a = 0; a < 8; a++)
        for (int c = 0; c < 8; c++)
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) k[((a * 8 + c) * 3 + i) * 3 + j] = u[a][c][i][j];
}

// the system of a voxel piece at rest: counts first (out arrays null), then the arrays
int mo_system(const uint8_t* state, const float* e, int nx, int ny, int nz, double h, double dt, double mass,
              int64_t* n, int64_t* npairs, int64_t* sites, double* at, double* diag, uint32_t* pi, uint32_t* pj,
              double* pb, double* b) {
    mech::Built B = mech::build(state, e, nx, ny, nz, h, dt, mass);
    *n = (int64_t)B.s.sites.size();
    *npairs = (int64_t)B.s.pairs.size();
    if (!sites) return 0;
    for (size_t i = 0; i < B.s.sites.size(); i++) {
        for (int k = 0; k < 3; k++) {
            sites[3 * i + k] = B.s.sites[i][k];
            at[3 * i + k] = B.s.at[i][k];
            b[3 * i + k] = B.b[i][k];
        }
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) diag[9 * i + 3 * r + c] = B.s.diag[i][r][c];
    }
    for (size_t p = 0; p < B.s.pairs.size(); p++) {
        pi[p] = B.s.pairs[p].i;
        pj[p] = B.s.pairs[p].j;
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) pb[9 * p + 3 * r + c] = B.s.pairs[p].b[r][c];
    }
    return 0;
}

static mech::System make(int64_t n, const int64_t* sites, const double* at, const double* diag, int64_t npairs,
                         const uint32_t* pi, const uint32_t* pj, const double* pb) {
    mech::System s;
    s.sites.resize(n);
    s.at.resize(n);
    s.diag.resize(n);
    for (int64_t i = 0; i < n; i++) {
        for (int k = 0; k < 3; k++) {
            s.sites[i][k] = sites[3 * i + k];
            s.at[i][k] = at[3 * i + k];
        }
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) s.diag[i][r][c] = diag[9 * i + 3 * r + c];
    }
    s.pairs.resize(npairs);
    for (int64_t p = 0; p < npairs; p++) {
        s.pairs[p].i = pi[p];
        s.pairs[p].j = pj[p];
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) s.pairs[p].b[r][c] = pb[9 * p + 3 * r + c];
    }
    return s;
}

// y = S x
void mo_times(int64_t n, const int64_t* sites, const double* at, const double* diag, int64_t npairs,
              const uint32_t* pi, const uint32_t* pj, const double* pb, const double* x, double* y) {
    mech::System s = make(n, sites, at, diag, npairs, pi, pj, pb);
    std::vector<mech::V3> xv(n), yv(n);
    for (int64_t i = 0; i < n; i++) xv[i] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
    s.times(xv, yv);
    for (int64_t i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) y[3 * i + k] = yv[i][k];
}

// Solver::new only: the coarse levels' sizes and the steps (the nodes', then each level's,
// 0 at a direct top)
int mo_levels(int64_t n, const int64_t* sites, const double* at, const double* diag, int64_t npairs,
              const uint32_t* pi, const uint32_t* pj, const double* pb, double size, int max_levels,
              int64_t* level_sizes, double* steps) {
    mech::System s = make(n, sites, at, diag, npairs, pi, pj, pb);
    mech::Solver solver(s, size);
    steps[0] = solver.step;
    int l = 0;
    for (; l < (int)solver.levels.size() && l < max_levels; l++) {
        level_sizes[l] = (int64_t)solver.levels[l].centre.size();
        steps[l + 1] = solver.levels[l].direct ? 0.0 : solver.levels[l].step;
    }
    return (int)solver.levels.size();
}

// Solver::new then solve from x (in/out): rounds, or -1 (the levels do not fit); the
// level sizes (parts per coarse level, up to max_levels) and the fine smoothing step
int mo_solve(int64_t n, const int64_t* sites, const double* at, const double* diag, int64_t npairs,
             const uint32_t* pi, const uint32_t* pj, const double* pb, const double* b, double* x, double tol,
             double size, int max_levels, int64_t* level_sizes, int* nlevels, double* step) {
    mech::System s = make(n, sites, at, diag, npairs, pi, pj, pb);
    mech::Solver solver(s, size);
    *nlevels = (int)solver.levels.size();
    for (int l = 0; l < (int)solver.levels.size() && l < max_levels; l++)
        level_sizes[l] = (int64_t)solver.levels[l].centre.size();
    *step = solver.step;
    std::vector<mech::V3> bv(n), xv(n);
    for (int64_t i = 0; i < n; i++) {
        bv[i] = {b[3 * i], b[3 * i + 1], b[3 * i + 2]};
        xv[i] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
    }
    int rounds = solver.solve(s, bv, xv, tol);
    for (int64_t i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) x[3 * i + k] = xv[i][k];
    return rounds;
}

}  // extern "C"
