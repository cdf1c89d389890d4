// ORACLE — test infrastructure only (see statics_oracle.hpp). A line-by-line CPU
// restatement of statics/src/{model,lattice,bodies}.rs; every function cites the
// reference lines it follows. Compiled without FMA contraction or fast-math so the
// FP64 operation order is the Rust source's.
#include "statics_oracle.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <set>
#include <thread>
#include <unordered_map>
#include <unordered_set>

namespace oracle {

// ---------------------------------------------------------------- model.rs:16-36
V3 add(V3 a, V3 b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
V3 sub(V3 a, V3 b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
V3 mul(V3 a, double s) { return {a[0] * s, a[1] * s, a[2] * s}; }
double dot(V3 a, V3 b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
V3 cross(V3 a, V3 b) {
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
double norm(V3 a) { return std::sqrt(dot(a, a)); }
V3 unit(V3 a) { return mul(a, 1.0 / norm(a)); }

// model.rs:53-58
const Mat STONE{"stone", 2500.0, 30e9, 12e9, 5e6, 100e6, 10e6};
const Mat WOOD{"wood", 600.0, 10e9, 4e9, 40e6, 30e6, 6e6};
const Mat MASONRY{"masonry", 2000.0, 5e9, 2e9, 0.2e6, 10e6, 0.4e6};
const Mat SOIL{"soil", 1800.0, 50e6, 20e6, 5e3, 0.3e6, 20e3};
const Mat STEEL{"steel", 7850.0, 200e9, 80e9, 250e6, 250e6, 145e6};
const Mat LEAVES{"leaves", 60.0, 0.2e9, 0.08e9, 5e6, 5e6, 1e6};

// Rust's f64::max: the non-NaN one if one is NaN (same as fmax).
static double fmax_r(double a, double b) { return std::fmax(a, b); }

double Mat::used(double s1, double s3) const {  // model.rs:66-68
    return fmax_r(fmax_r(s1 / ft, -s3 / fc), (s1 - s3) / (2.0 * fs));
}
Mat Mat::stronger(double by) const {  // model.rs:71-73
    Mat m = *this;
    m.ft = ft * by;
    m.fc = fc * by;
    m.fs = fs * by;
    return m;
}

V3 Bond::force(V3 delta) const {  // model.rs:115-119
    double along = dot(delta, n);
    double k = a / d;
    return add(mul(n, mat.e * k * along), mul(sub(delta, mul(n, along)), mat.g * k));
}
double Bond::used(V3 force) const {  // model.rs:123-129
    V3 t = mul(force, 1.0 / a);
    double sigma = dot(t, n);
    double tau2 = fmax_r(dot(t, t) - sigma * sigma, 0.0);
    double r = std::sqrt(sigma * sigma / 4.0 + tau2);
    return mat.used(sigma / 2.0 + r, sigma / 2.0 - r);
}
double Bond::energy(V3 force) const {  // model.rs:132-136
    double k = a / d;
    double along = dot(force, n);
    return 0.5 * (along * along / (mat.e * k) + (dot(force, force) - along * along) / (mat.g * k));
}
M3 Bond::stiffness() const {  // model.rs:139-149
    double k = a / d;
    M3 s{};
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) {
            double nn = n[r] * n[c];
            s[r][c] = mat.e * k * nn + mat.g * k * ((r == c ? 1.0 : 0.0) - nn);
        }
    return s;
}

// ---------------------------------------------------------------- lattice.rs
const int VOXEL_FACES[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};

size_t beam_class(V3 a, V3 b, V3 c) {  // lattice.rs:29-32
    V3 u = sub(a, c), v = sub(b, c);
    return (size_t)std::round(1.0 + dot(u, v) / (norm(u) * norm(v)));
}
double spacing(uint32_t level) { return UNIT * (double)(uint64_t(1) << level); }  // lattice.rs:34-36
V3 centre(Site site, uint32_t level) {  // lattice.rs:39-41
    V3 c;
    for (int k = 0; k < 3; k++) c[k] = ((double)site[k] + 0.5 * (double)(uint64_t(1) << level)) * UNIT;
    return c;
}
Site coarse_site(Site p, uint32_t l) {  // lattice.rs:45-47: v >> l << l, an arithmetic floor
    Site q;
    for (int k = 0; k < 3; k++) q[k] = p[k] & ~((int64_t(1) << l) - 1);
    return q;
}

std::array<Bond, 4> beam(size_t i, size_t j, V3 a, V3 b, double area, Mat mat) {  // lattice.rs:76-84
    V3 n = unit(sub(b, a));
    V3 e1 = unit(cross(n, std::fabs(n[0]) < 0.9 ? V3{1.0, 0.0, 0.0} : V3{0.0, 1.0, 0.0}));
    V3 e2 = cross(n, e1);
    double r = std::sqrt(area / (2.0 * M_PI));
    V3 middle = mul(add(a, b), 0.5);
    double d = norm(sub(b, a));
    V3 offs[4] = {mul(e1, r), mul(e1, -r), mul(e2, r), mul(e2, -r)};
    std::array<Bond, 4> out;
    for (int q = 0; q < 4; q++) out[q] = Bond{i, j, add(middle, offs[q]), n, area / 4.0, d, mat};
    return out;
}

std::vector<Solid> solids(uint32_t level, V3 lo, V3 hi, const Fill& fill) {  // lattice.rs:87-102
    double s = spacing(level);
    int64_t lo_k[3], hi_k[3];
    for (int k = 0; k < 3; k++) {
        lo_k[k] = (int64_t)std::floor(lo[k] / s);
        hi_k[k] = (int64_t)std::ceil(hi[k] / s);
    }
    std::vector<Solid> found;
    for (int64_t a = lo_k[0]; a < hi_k[0]; a++)
        for (int64_t b = lo_k[1]; b < hi_k[1]; b++)
            for (int64_t c = lo_k[2]; c < hi_k[2]; c++) {
                Site site{a * (int64_t(1) << level), b * (int64_t(1) << level), c * (int64_t(1) << level)};
                Mat mat;
                bool held;
                if (fill(centre(site, level), mat, held)) found.push_back(Solid{site, mat, held});
            }
    return found;
}

struct SiteHash {
    size_t operator()(const Site& s) const {
        uint64_t h = (uint64_t)s[0] * 0x9E3779B97F4A7C15ull;
        h ^= (uint64_t)s[1] * 0xC2B2AE3D27D4EB4Full + (h << 6) + (h >> 2);
        h ^= (uint64_t)s[2] * 0x165667B19E3779F9ull + (h << 6) + (h >> 2);
        return (size_t)h;
    }
};
struct KeyHash {
    size_t operator()(const std::array<Site, 2>& k) const {
        SiteHash h;
        return h(k[0]) * 31 + h(k[1]);
    }
};

void hold_bulk(uint32_t level, std::vector<Solid>& cells, double radius) {  // lattice.rs:107-119
    int64_t r = (int64_t)std::ceil(radius / spacing(level));
    std::vector<Site> near;
    for (int64_t a = -r; a <= r; a++)
        for (int64_t b = -r; b <= r; b++)
            for (int64_t c = -r; c <= r; c++)
                if (std::sqrt((double)(a * a + b * b + c * c)) * spacing(level) <= radius)
                    near.push_back({a << level, b << level, c << level});
    std::unordered_set<Site, SiteHash> filled;
    for (auto& c : cells) filled.insert(c.site);
    std::vector<bool> held(cells.size());
    for (size_t i = 0; i < cells.size(); i++) {
        bool all = true;
        for (auto& o : near) {
            Site q{cells[i].site[0] + o[0], cells[i].site[1] + o[1], cells[i].site[2] + o[2]};
            if (!filled.count(q)) {
                all = false;
                break;
            }
        }
        held[i] = all;
    }
    for (size_t i = 0; i < cells.size(); i++) cells[i].held = held[i];
}

// lattice.rs:124-163. `cell_of_bond` (an oracle extension) records each bond's cell.
static Lattice build_impl(uint32_t level, const std::vector<Solid>& cells, std::vector<int64_t>* cell_of_bond) {
    double s = spacing(level);
    std::unordered_set<Site, SiteHash> held;
    for (auto& c : cells)
        if (c.held) held.insert(c.site);
    std::unordered_map<std::array<Site, 2>, size_t, KeyHash> index;
    Lattice lat;
    lat.level = level;
    for (size_t ci = 0; ci < cells.size(); ci++) {
        const Solid& cell = cells[ci];
        if (cell.held) continue;
        double m = cell.mat.rho * s * s * s / 6.0;
        size_t ends[6];
        for (int f = 0; f < 6; f++) {
            Site other;
            for (int k = 0; k < 3; k++) other[k] = cell.site[k] + ((int64_t)VOXEL_FACES[f][k] << level);
            std::array<Site, 2> key = cell.site < other ? std::array<Site, 2>{cell.site, other}
                                                        : std::array<Site, 2>{other, cell.site};
            auto it = index.find(key);
            size_t k;
            if (it == index.end()) {
                V3 x = mul(add(centre(cell.site, level), centre(other, level)), 0.5);
                lat.nodes.push_back(Node{x, 0.0, cell.mat, held.count(other) > 0});
                lat.around.push_back(key);
                k = lat.nodes.size() - 1;
                index.emplace(key, k);
            } else {
                k = it->second;
            }
            Node& node = lat.nodes[k];
            node.m += m;
            if (cell.mat.rho > node.mat.rho) node.mat = cell.mat;
            ends[f] = k;
        }
        V3 middle = centre(cell.site, level);
        for (int a = 0; a < 6; a++)
            for (int b = a + 1; b < 6; b++) {
                if (!(lat.nodes[ends[a]].held && lat.nodes[ends[b]].held)) {
                    V3 x = lat.nodes[ends[a]].x, y = lat.nodes[ends[b]].x;
                    double area = SECTION[beam_class(x, y, middle)] * s * s;
                    auto bs = beam(ends[a], ends[b], x, y, area, cell.mat);
                    for (auto& bd : bs) {
                        lat.bonds.push_back(bd);
                        if (cell_of_bond) cell_of_bond->push_back((int64_t)ci);
                    }
                }
            }
    }
    return lat;
}
Lattice build(uint32_t level, const std::vector<Solid>& cells) { return build_impl(level, cells, nullptr); }

// ---------------------------------------------------------------- bodies.rs
using Pair = std::tuple<size_t, size_t, M6>;
struct RowRef {
    size_t o, p;
    bool transposed;
};
using BRow = std::vector<std::pair<size_t, M6>>;

Six shift(Six x, V3 r) {  // bodies.rs:44-47
    V3 u = add({x[0], x[1], x[2]}, cross({x[3], x[4], x[5]}, r));
    return {u[0], u[1], u[2], x[3], x[4], x[5]};
}

static int g_threads = 0;
void set_threads(int n) { g_threads = n; }
int threads() {
    if (g_threads > 0) return g_threads;
    unsigned h = std::thread::hardware_concurrency();
    return h ? (int)h : 1;
}


// Rust's `(0..6).map(..).sum()`: a left fold (from -0.0; 0.0 here, which differs
// only in the sign of an all-zero sum).
static Six times(const M6& a, const Six& x) {  // bodies.rs:71-73
    Six y;
    for (int s = 0; s < 6; s++) {
        double acc = 0.0;
        for (int t = 0; t < 6; t++) acc += a[s][t] * x[t];
        y[s] = acc;
    }
    return y;
}
static Six times_transposed(const M6& a, const Six& x) {  // bodies.rs:75-77
    Six y;
    for (int s = 0; s < 6; s++) {
        double acc = 0.0;
        for (int t = 0; t < 6; t++) acc += a[t][s] * x[t];
        y[s] = acc;
    }
    return y;
}
static Six add6v(const Six& a, const Six& b) {  // bodies.rs:79-81
    Six y;
    for (int s = 0; s < 6; s++) y[s] = a[s] + b[s];
    return y;
}
static M6 product(const M6& a, const M6& b) {  // bodies.rs:83-85
    M6 m;
    for (int r = 0; r < 6; r++)
        for (int c = 0; c < 6; c++) {
            double acc = 0.0;
            for (int k = 0; k < 6; k++) acc += a[r][k] * b[k][c];
            m[r][c] = acc;
        }
    return m;
}
static M6 transpose(const M6& a) {  // bodies.rs:87-89
    M6 m;
    for (int r = 0; r < 6; r++)
        for (int c = 0; c < 6; c++) m[r][c] = a[c][r];
    return m;
}
static void add6(M6& to, const M6& a, double by) {  // bodies.rs:91-97
    for (int r = 0; r < 6; r++)
        for (int c = 0; c < 6; c++) to[r][c] += by * a[r][c];
}
template <class F>
static M6 matrix(const F& f) {  // bodies.rs:100-109
    M6 a{};
    for (int c = 0; c < 6; c++) {
        Six e{};
        e[c] = 1.0;
        Six col = f(e);
        for (int r = 0; r < 6; r++) a[r][c] = col[r];
    }
    return a;
}
static void merge(BRow& row, size_t c, const M6& m, double by) {  // bodies.rs:112-121
    for (auto& e : row)
        if (e.first == c) {
            add6(e.second, m, by);
            return;
        }
    M6 to{};
    add6(to, m, by);
    row.emplace_back(c, to);
}

static double dot6(const std::vector<Six>& a, const std::vector<Six>& b) {  // bodies.rs:333-335
    double acc = 0.0;
    for (size_t k = 0; k < a.size(); k++) {
        double in = 0.0;
        for (int s = 0; s < 6; s++) in += a[k][s] * b[k][s];
        acc += in;
    }
    return acc;
}

M6 invert(const M6& m) {  // bodies.rs:576-602
    M6 a = m, inv{};
    for (int k = 0; k < 6; k++) inv[k][k] = 1.0;
    for (int col = 0; col < 6; col++) {
        // max_by over total_cmp of |a[x][col]|, the last of equal maxima. For the
        // non-negative values abs() yields, total order is the order of the raw bits.
        int piv = col;
        uint64_t best;
        {
            double v = std::fabs(a[col][col]);
            std::memcpy(&best, &v, 8);
        }
        for (int x = col + 1; x < 6; x++) {
            double v = std::fabs(a[x][col]);
            uint64_t bits;
            std::memcpy(&bits, &v, 8);
            if (bits >= best) {
                best = bits;
                piv = x;
            }
        }
        std::swap(a[col], a[piv]);
        std::swap(inv[col], inv[piv]);
        double d = a[col][col];
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
    return inv;
}

struct Cholesky {  // bodies.rs:286-328
    size_t n = 0;
    std::vector<double> l;
    std::vector<Six> solve(const std::vector<Six>& r) const;
};

struct Level {  // bodies.rs:25-40
    std::vector<V3> centre;
    std::vector<M6> own;
    std::vector<Pair> pairs;
    std::vector<std::vector<RowRef>> rows;
    std::vector<M6> inverse;
    double step = 1.0;
    std::vector<BRow> down;
    std::vector<std::vector<std::pair<size_t, size_t>>> from;
    std::optional<Cholesky> direct;

    static Level make(const Lattice& lattice, const std::vector<std::optional<size_t>>& part, size_t parts,
                      const std::vector<size_t>& live);                            // bodies.rs:126-164
    static Level of(std::vector<V3> centre, std::vector<M6> own, std::vector<Pair> pairs);  // :166-176
    double most_asked() const;                                                     // :180-190
    std::vector<Six> apply(const std::vector<Six>& x, Work& work) const;           // :193-206
    std::vector<Six> jacobi(const std::vector<Six>& r) const;                      // :208-210
    template <class F>
    BRow ask(size_t k, const F& m) const;                                          // :213-225
    Level coarser(const std::vector<size_t>& up, size_t count);                    // :228-282
};

Level Level::make(const Lattice& lattice, const std::vector<std::optional<size_t>>& part, size_t parts,
                  const std::vector<size_t>& live) {
    const auto& nodes = lattice.nodes;
    const auto& bonds = lattice.bonds;
    std::vector<V3> centre(parts, V3{0, 0, 0});
    for (size_t v = 0; v < part.size(); v++)
        if (part[v]) centre[*part[v]] = nodes[v].x;
    std::vector<M6> own(parts, M6{});
    std::vector<Pair> pairs;
    std::unordered_map<uint64_t, size_t> pair;
    using T3 = std::array<std::array<double, 6>, 3>;
    for (size_t b : live) {
        const Bond& bond = bonds[b];
        M3 s = bond.stiffness();
        auto seen = [&](size_t v) -> T3 {  // T = [1 | -r x], bodies.rs:141-144
            V3 r = sub(bond.p, nodes[v].x);
            return T3{std::array<double, 6>{1.0, 0.0, 0.0, 0.0, r[2], -r[1]},
                      std::array<double, 6>{0.0, 1.0, 0.0, -r[2], 0.0, r[0]},
                      std::array<double, 6>{0.0, 0.0, 1.0, r[1], -r[0], 0.0}};
        };
        auto through = [&](const T3& a, const T3& bb) -> M6 {  // bodies.rs:146-149
            T3 sb;
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 6; c++) {
                    double acc = 0.0;
                    for (int k = 0; k < 3; k++) acc += s[r][k] * bb[k][c];
                    sb[r][c] = acc;
                }
            M6 out;
            for (int r = 0; r < 6; r++)
                for (int c = 0; c < 6; c++) {
                    double acc = 0.0;
                    for (int k = 0; k < 3; k++) acc += a[k][r] * sb[k][c];
                    out[r][c] = acc;
                }
            return out;
        };
        std::optional<std::pair<size_t, T3>> side[2];
        size_t ends[2] = {bond.i, bond.j};
        for (int q = 0; q < 2; q++)
            if (part[ends[q]]) side[q] = std::make_pair(*part[ends[q]], seen(ends[q]));
        for (int q = 0; q < 2; q++)
            if (side[q]) add6(own[side[q]->first], through(side[q]->second, side[q]->second), 1.0);
        if (side[0] && side[1]) {
            size_t i = side[0]->first, j = side[1]->first;
            const T3* a = &side[0]->second;
            const T3* bb = &side[1]->second;
            if (!(i < j)) {
                std::swap(i, j);
                std::swap(a, bb);
            }
            uint64_t key = (uint64_t)i * (uint64_t)parts + (uint64_t)j;
            auto it = pair.find(key);
            size_t k;
            if (it == pair.end()) {
                pairs.emplace_back(i, j, M6{});
                k = pairs.size() - 1;
                pair.emplace(key, k);
            } else {
                k = it->second;
            }
            add6(std::get<2>(pairs[k]), through(*a, *bb), -1.0);
        }
    }
    return Level::of(std::move(centre), std::move(own), std::move(pairs));
}

Level Level::of(std::vector<V3> centre, std::vector<M6> own, std::vector<Pair> pairs) {
    Level level;
    level.rows.assign(own.size(), {});
    for (size_t p = 0; p < pairs.size(); p++) {
        size_t i = std::get<0>(pairs[p]), j = std::get<1>(pairs[p]);
        level.rows[i].push_back(RowRef{j, p, false});
        level.rows[j].push_back(RowRef{i, p, true});
    }
    level.inverse.resize(own.size());
    for (size_t k = 0; k < own.size(); k++) level.inverse[k] = invert(own[k]);
    level.centre = std::move(centre);
    level.own = std::move(own);
    level.pairs = std::move(pairs);
    level.step = 1.0;
    level.step = 4.0 / 3.0 / level.most_asked();
    return level;
}

double Level::most_asked() const {
    std::vector<Six> v(own.size());
    for (size_t k = 0; k < own.size(); k++)
        for (int s = 0; s < 6; s++) v[k][s] = 1.0 + (double)((7 * k + 3 * s) % 11) / 11.0;
    double most = 1.0;
    for (int it = 0; it < 12; it++) {
        Work w;
        std::vector<Six> wv = jacobi(apply(v, w));
        most = std::sqrt(dot6(wv, wv)) / std::sqrt(dot6(v, v));
        double scale = 1.0 / std::sqrt(dot6(wv, wv));
        for (auto& x : wv)
            for (auto& a : x) a = a * scale;
        v = std::move(wv);
    }
    return most;
}

std::vector<Six> Level::apply(const std::vector<Six>& x, Work& work) const {
    work.v += (double)(x.size() + pairs.size());
    return each<Six>(x.size(), [&](size_t i) {
        Six y = times(own[i], x[i]);
        for (const RowRef& rr : rows[i]) {
            const M6& m = std::get<2>(pairs[rr.p]);
            Six a = rr.transposed ? times_transposed(m, x[rr.o]) : times(m, x[rr.o]);
            for (int s = 0; s < 6; s++) y[s] += a[s];
        }
        return y;
    });
}

std::vector<Six> Level::jacobi(const std::vector<Six>& r) const {
    return each<Six>(r.size(), [&](size_t i) { return times(inverse[i], r[i]); });
}

template <class F>
BRow Level::ask(size_t k, const F& m) const {
    BRow row;
    for (const auto& cb : m(k)) merge(row, cb.first, product(own[k], cb.second), 1.0);
    for (const RowRef& rr : rows[k]) {
        M6 a = rr.transposed ? transpose(std::get<2>(pairs[rr.p])) : std::get<2>(pairs[rr.p]);
        for (const auto& cb : m(rr.o)) merge(row, cb.first, product(a, cb.second), 1.0);
    }
    return row;
}

Level Level::coarser(const std::vector<size_t>& up, size_t count) {
    std::vector<V3> cen(count, V3{0, 0, 0});
    std::vector<double> n(count, 0.0);
    for (size_t k = 0; k < up.size(); k++) {
        size_t c = up[k];
        cen[c] = add(cen[c], centre[k]);
        n[c] += 1.0;
    }
    for (size_t c = 0; c < count; c++) cen[c] = mul(cen[c], 1.0 / n[c]);
    std::vector<M6> rigid(up.size());
    for (size_t k = 0; k < up.size(); k++) {
        V3 r = sub(centre[k], cen[up[k]]);
        rigid[k] = matrix([&](Six y) { return shift(y, r); });
    }
    auto rigid_row = [&](size_t k) { return BRow{{up[k], rigid[k]}}; };
    down = each<BRow>(up.size(), [&](size_t k) {
        BRow row = rigid_row(k);
        for (const auto& cm : ask(k, rigid_row)) merge(row, cm.first, product(inverse[k], cm.second), -step);
        return row;
    });
    from.assign(count, {});
    for (size_t k = 0; k < down.size(); k++)
        for (size_t q = 0; q < down[k].size(); q++) from[down[k][q].first].emplace_back(k, q);
    const Level& fine = *this;
    auto kp = each<BRow>(up.size(), [&](size_t k) { return fine.ask(k, [&](size_t o) -> const BRow& { return fine.down[o]; }); });
    auto rows_c = each<BRow>(count, [&](size_t c) {
        BRow row;
        for (const auto& kq : fine.from[c]) {
            M6 pt = transpose(fine.down[kq.first][kq.second].second);
            for (const auto& dm : kp[kq.first])
                if (dm.first >= c) merge(row, dm.first, product(pt, dm.second), 1.0);
        }
        return row;
    });
    std::vector<M6> own_c(count, M6{});
    std::vector<Pair> pairs_c;
    for (size_t c = 0; c < count; c++)
        for (auto& dm : rows_c[c]) {
            if (dm.first == c)
                own_c[c] = dm.second;
            else
                pairs_c.emplace_back(c, dm.first, dm.second);
        }
    return Level::of(std::move(cen), std::move(own_c), std::move(pairs_c));
}

static Cholesky cholesky_of(const Level& level) {  // bodies.rs:293-315
    size_t parts = level.centre.size();
    size_t n = 6 * parts;
    std::vector<double> a(n * n, 0.0);
    Work w;
    for (size_t c = 0; c < n; c++) {
        std::vector<Six> e(parts, Six{});
        e[c / 6][c % 6] = 1.0;
        auto v = level.apply(e, w);
        for (size_t k = 0; k < v.size(); k++)
            for (int s = 0; s < 6; s++) a[(6 * k + s) * n + c] = v[k][s];
    }
    for (size_t j = 0; j < n; j++) {
        double sum = 0.0;
        for (size_t k = 0; k < j; k++) sum += a[j * n + k] * a[j * n + k];
        double d = std::sqrt(a[j * n + j] - sum);
        a[j * n + j] = d;
        for (size_t i = j + 1; i < n; i++) {
            double s2 = 0.0;
            for (size_t k = 0; k < j; k++) s2 += a[i * n + k] * a[j * n + k];
            a[i * n + j] = (a[i * n + j] - s2) / d;
        }
    }
    Cholesky ch;
    ch.n = n;
    ch.l = std::move(a);
    return ch;
}

std::vector<Six> Cholesky::solve(const std::vector<Six>& r) const {  // bodies.rs:317-327
    std::vector<double> y;
    y.reserve(n);
    for (auto& v : r)
        for (double a : v) y.push_back(a);
    for (size_t i = 0; i < n; i++) {
        double s = 0.0;
        for (size_t k = 0; k < i; k++) s += l[i * n + k] * y[k];
        y[i] = (y[i] - s) / l[i * n + i];
    }
    for (size_t i = n; i-- > 0;) {
        double s = 0.0;
        for (size_t k = i + 1; k < n; k++) s += l[k * n + i] * y[k];
        y[i] = (y[i] - s) / l[i * n + i];
    }
    std::vector<Six> out(n / 6);
    for (size_t c = 0; c < n / 6; c++)
        for (int s = 0; s < 6; s++) out[c][s] = y[6 * c + s];
    return out;
}

// bodies.rs:338-373; `iterations` (an oracle extension) counts the loop's passes.
template <class P>
static std::vector<Six> conjugate_gradients(const Level& level, const std::vector<Six>& loads, P& precondition,
                                            double tol, size_t max_iter, Work& work, size_t* iterations) {
    std::vector<Six> x(loads.size(), Six{});
    std::vector<Six> r = loads;
    std::vector<Six> z = precondition(r);
    std::vector<Six> p = z;
    double rz = dot6(r, z);
    double goal = tol * std::sqrt(dot6(loads, loads));
    size_t it = 0;
    for (; it < max_iter; it++) {
        if (std::sqrt(dot6(r, r)) <= goal) break;
        auto ap = level.apply(p, work);
        double alpha = rz / dot6(p, ap);
        for (size_t k = 0; k < x.size(); k++)
            for (int s = 0; s < 6; s++) {
                x[k][s] += alpha * p[k][s];
                r[k][s] -= alpha * ap[k][s];
            }
        z = precondition(r);
        double next = dot6(r, z);
        for (size_t k = 0; k < x.size(); k++)
            for (int s = 0; s < 6; s++) p[k][s] = z[k][s] + next / rz * p[k][s];
        rz = next;
    }
    if (iterations) *iterations = it;
    return x;
}

static std::vector<Six> cycle(const std::vector<Level>& levels, size_t l, const std::vector<Six>& r,
                              Work& work) {  // bodies.rs:377-403
    const Level& level = levels[l];
    if (l + 1 == levels.size()) return level.direct->solve(r);
    auto rest = [&](const std::vector<Six>& x) {
        auto ax = level.apply(x, work);
        std::vector<Six> out(r.size());
        for (size_t k = 0; k < r.size(); k++)
            for (int s = 0; s < 6; s++) out[k][s] = r[k][s] - ax[k][s];
        return out;
    };
    std::vector<Six> x = level.jacobi(r);
    for (auto& v : x)
        for (auto& a : v) a = a * level.step;
    auto left = rest(x);
    auto coarse = each<Six>(level.from.size(), [&](size_t c) {
        Six a{};
        for (const auto& kq : level.from[c])
            a = add6v(a, times_transposed(level.down[kq.first][kq.second].second, left[kq.first]));
        return a;
    });
    auto y = cycle(levels, l + 1, coarse, work);
    auto mv = each<Six>(x.size(), [&](size_t k) {
        Six a{};
        for (const auto& cp : level.down[k]) a = add6v(a, times(cp.second, y[cp.first]));
        return a;
    });
    for (size_t k = 0; k < x.size(); k++) x[k] = add6v(x[k], mv[k]);
    left = rest(x);
    auto d = level.jacobi(left);
    for (size_t k = 0; k < x.size(); k++)
        for (int s = 0; s < 6; s++) x[k][s] += level.step * d[k][s];
    return x;
}

size_t find(std::vector<size_t>& p, size_t a) {  // bodies.rs:628-634
    while (p[a] != a) {
        p[a] = p[p[a]];
        a = p[a];
    }
    return a;
}

// bodies.rs:472-496
static size_t bodies_of(const Level& level, const std::vector<std::optional<size_t>>& part,
                        const std::vector<Site>& key, std::vector<size_t>& up,
                        std::vector<std::optional<size_t>>& next) {
    size_t parts = level.centre.size();
    std::vector<Site> their(parts, Site{0, 0, 0});
    for (size_t v = 0; v < part.size(); v++)
        if (part[v]) their[*part[v]] = key[v];
    std::vector<size_t> parent(parts);
    for (size_t k = 0; k < parts; k++) parent[k] = k;
    for (const auto& pr : level.pairs) {
        size_t i = std::get<0>(pr), j = std::get<1>(pr);
        if (their[i] == their[j]) {
            size_t a = find(parent, i), c = find(parent, j);
            parent[a] = c;
        }
    }
    std::unordered_map<size_t, size_t> id;
    up.assign(parts, 0);
    for (size_t k = 0; k < parts; k++) {
        size_t n = id.size();
        size_t root = find(parent, k);
        auto it = id.find(root);
        if (it == id.end()) {
            id.emplace(root, n);
            up[k] = n;
        } else {
            up[k] = it->second;
        }
    }
    next.assign(part.size(), std::nullopt);
    for (size_t v = 0; v < part.size(); v++)
        if (part[v]) next[v] = up[*part[v]];
    return id.size();
}

std::vector<Six> motions(const Lattice& lattice, const std::vector<bool>& alive, const std::vector<bool>& gone,
                         const std::function<Six(size_t)>& loads, Work& work, const MotionsOptions& opt,
                         Hierarchy* hier) {  // bodies.rs:429-468
    auto t0 = std::chrono::steady_clock::now();
    const auto& nodes = lattice.nodes;
    const auto& bonds = lattice.bonds;
    std::vector<size_t> live;
    for (size_t b = 0; b < bonds.size(); b++)
        if (alive[b] && !gone[bonds[b].i] && !gone[bonds[b].j]) live.push_back(b);
    std::vector<std::optional<size_t>> part(nodes.size());
    size_t count = 0;
    for (size_t v = 0; v < nodes.size(); v++)
        if (!nodes[v].held && !gone[v]) part[v] = count++;
    auto node = part;
    std::vector<Level> levels;
    levels.push_back(Level::make(lattice, part, count, live));
    if (hier) {
        *hier = Hierarchy{};
        hier->counts.push_back(count);
        hier->pairs.push_back(levels.back().pairs.size());
        hier->steps.push_back(levels.back().step);
    }
    std::vector<Site> key(lattice.around.size());
    for (size_t v = 0; v < key.size(); v++) key[v] = lattice.around[v][0];
    uint32_t l = lattice.level;
    while (count > opt.few) {
        l += 1;
        for (auto& k : key) k = coarse_site(k, l);
        std::vector<size_t> up;
        std::vector<std::optional<size_t>> next;
        size_t bodies = bodies_of(levels.back(), part, key, up, next);
        if (bodies == count) break;
        Level up_level = levels.back().coarser(up, bodies);
        levels.push_back(std::move(up_level));
        if (hier) {
            hier->up.push_back(up);
            hier->counts.push_back(bodies);
            hier->pairs.push_back(levels.back().pairs.size());
            hier->steps.push_back(levels.back().step);
        }
        part = std::move(next);
        count = bodies;
    }
    levels.back().direct = cholesky_of(levels.back());
    auto t1 = std::chrono::steady_clock::now();
    std::vector<Six> lv;
    for (size_t v = 0; v < nodes.size(); v++)
        if (node[v]) lv.push_back(loads(v));
    Work inner;
    auto v_cycle = [&](const std::vector<Six>& r) { return cycle(levels, 0, r, inner); };
    size_t iters = 0;
    auto x = conjugate_gradients(levels[0], lv, v_cycle, opt.tol, opt.max_iter, work, &iters);
    work.v += inner.v;
    auto t2 = std::chrono::steady_clock::now();
    if (hier) {
        hier->iterations = iters;
        hier->setup_seconds = std::chrono::duration<double>(t1 - t0).count();
        hier->solve_seconds = std::chrono::duration<double>(t2 - t1).count();
    }
    std::vector<Six> out(nodes.size(), Six{});
    for (size_t v = 0; v < nodes.size(); v++)
        if (node[v]) out[v] = x[*node[v]];
    return out;
}

std::vector<V3> moved(const Lattice& lattice, const std::vector<Six>& x) {  // bodies.rs:420-423
    auto at = [&](size_t v, V3 p) -> V3 {
        Six s = shift(x[v], sub(p, lattice.nodes[v].x));
        return {s[0], s[1], s[2]};
    };
    std::vector<V3> f(lattice.bonds.size());
    for (size_t b = 0; b < lattice.bonds.size(); b++) {
        const Bond& bd = lattice.bonds[b];
        f[b] = bd.force(sub(at(bd.j, bd.p), at(bd.i, bd.p)));
    }
    return f;
}

std::vector<V3> forces(const Lattice& lattice, const std::vector<bool>& alive, const std::vector<bool>& gone,
                       Work& work) {  // bodies.rs:407-417
    auto weight = [&](size_t v) { return Six{0.0, -lattice.nodes[v].m * GRAVITY, 0.0, 0.0, 0.0, 0.0}; };
    auto x = motions(lattice, alive, gone, weight, work);
    auto f = moved(lattice, x);
    for (size_t b = 0; b < lattice.bonds.size(); b++) {
        const Bond& bd = lattice.bonds[b];
        if (!alive[b] || gone[bd.i] || gone[bd.j]) f[b] = V3{0, 0, 0};
    }
    return f;
}

std::vector<double> used(const Lattice& lattice, const std::vector<V3>& force) {  // bodies.rs:544-546
    std::vector<double> u(lattice.bonds.size());
    for (size_t b = 0; b < u.size(); b++) u[b] = lattice.bonds[b].used(force[b]);
    return u;
}

std::vector<bool> joined_to_held(const std::vector<Node>& nodes, const std::vector<Bond>& bonds,
                                 const std::vector<bool>& alive) {  // bodies.rs:557-574
    std::vector<std::vector<size_t>> next(nodes.size());
    for (size_t b = 0; b < bonds.size(); b++)
        if (alive[b]) {
            next[bonds[b].i].push_back(bonds[b].j);
            next[bonds[b].j].push_back(bonds[b].i);
        }
    std::vector<bool> held(nodes.size());
    std::vector<size_t> stack;
    for (size_t v = 0; v < nodes.size(); v++) {
        held[v] = nodes[v].held;
        if (held[v]) stack.push_back(v);
    }
    while (!stack.empty()) {
        size_t v = stack.back();
        stack.pop_back();
        for (size_t w : next[v])
            if (!held[w]) {
                held[w] = true;
                stack.push_back(w);
            }
    }
    return held;
}

std::vector<double> used_standing(const Lattice& lattice) {  // bodies.rs:550-554
    std::vector<bool> alive(lattice.bonds.size(), true);
    auto h = joined_to_held(lattice.nodes, lattice.bonds, alive);
    std::vector<bool> gone(h.size());
    for (size_t v = 0; v < h.size(); v++) gone[v] = !h[v];
    Work w;
    return used(lattice, forces(lattice, alive, gone, w));
}

Outcome settle(const Lattice& lattice) {  // bodies.rs:511-541
    const auto& nodes = lattice.nodes;
    const auto& bonds = lattice.bonds;
    std::vector<bool> alive(bonds.size(), true);
    std::vector<bool> gone(nodes.size(), false);
    Work work;
    size_t rounds = 0;
    for (;;) {
        rounds += 1;
        auto held = joined_to_held(nodes, bonds, alive);
        for (size_t v = 0; v < nodes.size(); v++) gone[v] = gone[v] || !held[v];
        auto f = forces(lattice, alive, gone, work);
        auto u = used(lattice, f);
        std::vector<bool> over(bonds.size());
        for (size_t b = 0; b < bonds.size(); b++)
            over[b] = alive[b] && !gone[bonds[b].i] && !gone[bonds[b].j] && u[b] > 1.0;
        bool broke = false;
        for (size_t beam0 = 0; beam0 + PER_BEAM <= over.size(); beam0 += PER_BEAM) {
            bool any = false;
            for (size_t q = 0; q < PER_BEAM; q++) any = any || over[beam0 + q];
            if (any) {
                for (size_t q = 0; q < PER_BEAM; q++) alive[beam0 + q] = false;
                broke = true;
            }
        }
        if (!broke) break;
    }
    double free = 0.0, fell = 0.0;
    for (size_t v = 0; v < nodes.size(); v++) {
        if (!nodes[v].held) free += nodes[v].m;
        if (gone[v]) fell += nodes[v].m;
    }
    return Outcome{free > 0.0 ? fell / free : 0.0, gone, rounds, work.v};
}

void as_generated(Lattice& lattice, const Lattice& generated) {  // bodies.rs:611-625
    using BK = std::array<std::array<Site, 2>, 2>;
    auto beam_key = [](const Lattice& l, const Bond& b) -> BK {
        auto i = l.around[b.i], j = l.around[b.j];
        return i < j ? BK{i, j} : BK{j, i};
    };
    std::map<BK, double> need;
    auto u = used_standing(generated);
    for (size_t b = 0; b < generated.bonds.size(); b++) {
        auto it = need.emplace(beam_key(generated, generated.bonds[b]), 0.0).first;
        it->second = fmax_r(it->second, u[b]);
    }
    std::vector<double> by(lattice.bonds.size());
    for (size_t b = 0; b < lattice.bonds.size(); b++) {
        auto it = need.find(beam_key(lattice, lattice.bonds[b]));
        by[b] = it == need.end() ? 1.0 : fmax_r(it->second * MARGIN, 1.0);
    }
    for (size_t b = 0; b < lattice.bonds.size(); b++) lattice.bonds[b].mat = lattice.bonds[b].mat.stronger(by[b]);
}

// Level 0's operator alone (Level::new + Level::apply, bodies.rs:126-206), every bond
// alive and no node gone: the parity reference for the GPU stencil.
std::vector<Six> level0_apply(const Lattice& lattice, const std::vector<Six>& x_parts) {
    std::vector<size_t> live(lattice.bonds.size());
    for (size_t b = 0; b < live.size(); b++) live[b] = b;
    std::vector<std::optional<size_t>> part(lattice.nodes.size());
    size_t count = 0;
    for (size_t v = 0; v < lattice.nodes.size(); v++)
        if (!lattice.nodes[v].held) part[v] = count++;
    Level level = Level::make(lattice, part, count, live);
    Work w;
    return level.apply(x_parts, w);
}

// ---------------------------------------------------------------- synthetic pieces
Lattice grid_lattice(int nx, int ny, int nz, const uint8_t* state, const float* k, double g_over_e, double rho,
                     std::vector<int64_t>* cell_of_bond) {
    std::vector<Solid> cells;
    std::vector<int64_t> flat;
    for (int x = 0; x < nx; x++)
        for (int y = 0; y < ny; y++)
            for (int z = 0; z < nz; z++) {
                size_t c = ((size_t)x * ny + y) * nz + z;
                if (!state[c]) continue;
                double e = (double)k[c];
                Mat m{"piece", rho, e, g_over_e * e, 1.0, 1.0, 1.0};
                cells.push_back(Solid{Site{x, y, z}, m, state[c] == 2});
                flat.push_back((int64_t)c);
            }
    std::vector<int64_t> cob;
    Lattice lat = build_impl(0, cells, cell_of_bond ? &cob : nullptr);
    if (cell_of_bond) {
        cell_of_bond->resize(cob.size());
        for (size_t b = 0; b < cob.size(); b++) (*cell_of_bond)[b] = flat[cob[b]];
    }
    return lat;
}

}  // namespace oracle
