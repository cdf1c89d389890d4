// ORACLE — test infrastructure only, never part of the product.
//
// A CPU restatement of statics/src/gather.rs: a coarser level measured from a finer
// one. Each coarse cell's matter is condensed onto its faces (each face a rigid handle
// moved alone along each axis, one Gauss–Jordan elimination of the free parts), the
// handles' reactions fitted by non-negative least squares with beams between faces,
// and each beam's strength taken from the finer bonds' use when it is pulled alone.
// Loop orders, map orders (a BTreeMap of face keys) and floating-point operation
// orders follow the Rust source, so node and bond numbering are the reference's.
//
// Pinned by the reference's own test `a_bar_weighs_as_much` (gather.rs:401-412) and by
// the full-cell figures its docs publish (docs/statics.md:166-175); both in tests/.
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <stdexcept>
#include <unordered_map>

#include "statics_oracle.hpp"

namespace oracle {

namespace {

// Rust's f64::total_cmp as a key: a signed integer order over every bit pattern.
int64_t total_key(double v) {
    int64_t i;
    std::memcpy(&i, &v, 8);
    return i ^ (int64_t)(((uint64_t)(i >> 63)) >> 1);
}

bool same_mat(const Mat& a, const Mat& b) { return std::strcmp(a.name, b.name) == 0; }

// gather.rs:24-31: a cell's free parts (finer nodes inside it), the cells across its
// faces, and its finer bonds between places (free parts first, then one handle a face).
struct Cell {
    std::vector<size_t> free;
    std::vector<size_t> across;
    std::vector<std::array<size_t, 3>> bonds;

    size_t handle(size_t other) {  // gather.rs:34-40
        size_t k = 0;
        while (k < across.size() && across[k] != other) k++;
        if (k == across.size()) across.push_back(other);
        return free.size() + k;
    }

    std::vector<size_t> pieces() const {  // gather.rs:43-51
        size_t nf = free.size();
        std::vector<size_t> parent(nf + across.size());
        for (size_t k = 0; k < parent.size(); k++) parent[k] = k;
        for (const auto& b : bonds) {
            size_t a = find(parent, b[0]), c = find(parent, b[1]);
            parent[a] = c;
        }
        std::vector<size_t> out(across.size());
        for (size_t h = 0; h < across.size(); h++) out[h] = find(parent, nf + h);
        return out;
    }
};

// gather.rs:58-114: the cell's matter as a lattice of its own (handles held, at `at`),
// and per handle axis the finer bonds' forces with the free parts at rest.
std::pair<Lattice, std::vector<std::vector<V3>>> responses(const Lattice& fine, const Cell& cell,
                                                           const std::vector<V3>& at) {
    size_t nf = cell.free.size(), nh = cell.across.size();
    Lattice lat;
    lat.level = fine.level;
    for (size_t v : cell.free) {
        Node n = fine.nodes[v];
        n.held = false;
        lat.nodes.push_back(n);
    }
    for (const V3& x : at) lat.nodes.push_back(Node{x, 0.0, STONE, true});
    for (const auto& t : cell.bonds) {
        Bond b = fine.bonds[t[2]];
        b.i = t[0];
        b.j = t[1];
        lat.bonds.push_back(b);
    }
    lat.around.assign(nf + nh, std::array<Site, 2>{});
    size_t n = 6 * nf, m = 3 * nh;
    auto column = [&](size_t v, size_t d, V3 p) -> V3 {
        V3 e{0.0, 0.0, 0.0};
        e[d % 3] = 1.0;
        return d < 3 ? e : cross(e, sub(p, lat.nodes[v].x));
    };
    // -1: no unknown (a handle's turn)
    auto dof = [&](size_t v, size_t d) -> int64_t {
        if (v < nf) return (int64_t)(6 * v + d);
        if (d < 3) return (int64_t)(n + 3 * (v - nf) + d);
        return -1;
    };
    std::vector<std::vector<double>> a(n, std::vector<double>(n + m, 0.0));
    for (const Bond& b : lat.bonds) {
        M3 s = b.stiffness();
        const std::pair<size_t, double> ends[2] = {{b.i, -1.0}, {b.j, 1.0}};
        for (const auto& [v, sv] : ends)
            for (size_t d = 0; d < 6; d++) {
                int64_t r = dof(v, d);
                if (r < 0 || (size_t)r >= n) continue;
                V3 cv = column(v, d, b.p);
                V3 scv{dot(s[0], cv), dot(s[1], cv), dot(s[2], cv)};
                for (const auto& [w, sw] : ends)
                    for (size_t e = 0; e < 6; e++) {
                        int64_t c = dof(w, e);
                        if (c < 0) continue;
                        double sign = (size_t)c < n ? 1.0 : -1.0;
                        a[r][c] += sign * sv * sw * dot(scv, column(w, e, b.p));
                    }
            }
    }
    auto x = gather_solve(std::move(a), m);
    std::vector<std::vector<V3>> cases(m);
    for (size_t c = 0; c < m; c++) {
        std::vector<Six> motion(nf + nh, Six{});
        for (size_t v = 0; v < nf; v++)
            for (size_t d = 0; d < 6; d++) motion[v][d] = x[6 * v + d][c];
        motion[nf + c / 3][c % 3] = 1.0;
        cases[c] = moved(lat, motion);
    }
    return {std::move(lat), std::move(cases)};
}

}  // namespace

std::vector<std::vector<double>> gather_solve(std::vector<std::vector<double>> a, size_t rhs) {  // gather.rs:164-184
    size_t n = a.size();
    double scale = 0.0;
    for (size_t r = 0; r < n; r++) scale = std::fmax(scale, std::fabs(a[r][r]));
    auto small = [&](double v) { return std::fabs(v) <= 1e-12 * scale; };
    for (size_t c = 0; c < n; c++) {
        size_t p = c;  // max_by: the last of equal maxima
        for (size_t x = c + 1; x < n; x++)
            if (total_key(std::fabs(a[x][c])) >= total_key(std::fabs(a[p][c]))) p = x;
        std::swap(a[c], a[p]);
        if (small(a[c][c])) continue;
        std::vector<double> pivot = a[c];
        for (size_t r = 0; r < n; r++) {
            std::vector<double>& row = a[r];
            double f = row[c] / pivot[c];
            if (r != c && f != 0.0)
                for (size_t k = c; k < n + rhs; k++) row[k] -= f * pivot[k];
        }
    }
    std::vector<std::vector<double>> out(n, std::vector<double>(rhs));
    for (size_t r = 0; r < n; r++)
        for (size_t k = 0; k < rhs; k++) out[r][k] = small(a[r][r]) ? 0.0 : a[r][n + k] / a[r][r];
    return out;
}

std::vector<std::tuple<size_t, size_t, double>> gather_beams(const std::vector<std::vector<double>>& k,
                                                             const std::vector<V3>& at,
                                                             const std::function<bool(size_t, size_t)>& joined) {
    // gather.rs:119-161
    size_t n = 3 * at.size();
    std::vector<std::pair<size_t, size_t>> pairs;
    for (size_t a = 0; a < at.size(); a++)
        for (size_t b = a + 1; b < at.size(); b++)
            if (joined(a, b)) pairs.push_back({a, b});
    std::vector<std::vector<double>> units;
    for (const auto& [a, b] : pairs) {
        V3 e = unit(sub(at[b], at[a]));
        std::vector<double> d(n * n, 0.0);
        for (size_t r = 0; r < 3; r++)
            for (size_t c = 0; c < 3; c++) {
                double v = e[r] * e[c];
                d[(3 * a + r) * n + 3 * a + c] += v;
                d[(3 * b + r) * n + 3 * b + c] += v;
                d[(3 * a + r) * n + 3 * b + c] -= v;
                d[(3 * b + r) * n + 3 * a + c] -= v;
            }
        units.push_back(std::move(d));
    }
    std::vector<double> target(n * n);
    for (size_t i = 0; i < n * n; i++) target[i] = 0.5 * (k[i / n][i % n] + k[i % n][i / n]);
    auto vdot = [](const std::vector<double>& a, const std::vector<double>& b) {
        double s = 0.0;
        for (size_t i = 0; i < a.size(); i++) s += a[i] * b[i];
        return s;
    };
    // Least squares, dropping the most negative beam till none is.
    std::vector<bool> on(pairs.size(), true);
    for (;;) {
        std::vector<size_t> idx;
        for (size_t p = 0; p < pairs.size(); p++)
            if (on[p]) idx.push_back(p);
        size_t m = idx.size();
        std::vector<std::vector<double>> g(m, std::vector<double>(m + 1, 0.0));
        for (size_t r = 0; r < m; r++) {
            for (size_t c = 0; c < m; c++) g[r][c] = vdot(units[idx[r]], units[idx[c]]);
            g[r][m] = vdot(units[idx[r]], target);
        }
        auto sol = gather_solve(std::move(g), 1);
        int64_t worst = -1;  // min_by: the first of equal minima
        for (size_t r = 0; r < m; r++)
            if (sol[r][0] < 0.0 && (worst < 0 || total_key(sol[r][0]) < total_key(sol[(size_t)worst][0])))
                worst = (int64_t)r;
        if (worst >= 0) {
            on[idx[(size_t)worst]] = false;
            continue;
        }
        std::vector<std::tuple<size_t, size_t, double>> out;
        for (size_t r = 0; r < m; r++)
            if (sol[r][0] > 0.0) out.emplace_back(pairs[idx[r]].first, pairs[idx[r]].second, sol[r][0]);
        return out;
    }
}

Lattice gathered(const Lattice& fine) { return measured(fine, true); }  // gather.rs:193-195

Full full(const Mat& mat) {  // gather.rs:203-226
    static std::mutex lock;
    static std::vector<std::pair<std::string, Full>> known;
    {
        std::lock_guard<std::mutex> g(lock);
        for (const auto& [name, f] : known)
            if (name == mat.name) return f;
    }
    double s = spacing(1);
    Fill fill = [&](V3, Mat& m, bool& held) {
        m = mat;
        held = false;
        return true;
    };
    Lattice coarse = measured(build(0, solids(0, {-1.5 * s, -1.5 * s, -1.5 * s}, {1.5 * s, 1.5 * s, 1.5 * s}, fill)),
                              false);
    double sum[2][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    const Site zero{0, 0, 0};
    for (size_t q = 0; q + PER_BEAM <= coarse.bonds.size(); q += PER_BEAM) {
        const Bond& b = coarse.bonds[q];
        size_t i = b.i, j = b.j;
        auto touches = [&](size_t v) { return coarse.around[v][0] == zero || coarse.around[v][1] == zero; };
        if (touches(i) && touches(j)) {
            size_t k = beam_class(coarse.nodes[i].x, coarse.nodes[j].x, centre(zero, 1));
            sum[k][0] += 4.0 * b.a / (s * s);
            sum[k][1] += b.mat.ft / mat.ft;
            sum[k][2] += 1.0;
        }
    }
    Full f;
    for (int k = 0; k < 2; k++)
        f[k] = sum[k][2] > 0.0 ? std::make_pair(sum[k][0] / sum[k][2], sum[k][1] / sum[k][2]) : std::make_pair(1.0, 1.0);
    std::lock_guard<std::mutex> g(lock);
    known.push_back({mat.name, f});
    return f;
}

Lattice measured(const Lattice& fine, bool against_full) {  // gather.rs:230-395
    uint32_t level = fine.level + 1;
    std::map<Site, size_t> index;
    std::vector<Site> sites;
    auto cell_of = [&](Site site) {
        Site key = coarse_site(site, level);
        auto it = index.find(key);
        if (it != index.end()) return it->second;
        sites.push_back(key);
        index.emplace(key, sites.size() - 1);
        return sites.size() - 1;
    };
    // Each fine node: the coarse cells it lies between; each fine bond: the one its
    // finer cell is in.
    std::vector<std::array<size_t, 2>> between(fine.nodes.size());
    for (size_t v = 0; v < fine.nodes.size(); v++) {
        size_t x = cell_of(fine.around[v][0]);
        size_t y = cell_of(fine.around[v][1]);
        between[v] = {x, y};
    }
    std::vector<size_t> lies(fine.bonds.size());
    for (size_t b = 0; b < fine.bonds.size(); b++) {
        const auto& ai = fine.around[fine.bonds[b].i];
        const auto& aj = fine.around[fine.bonds[b].j];
        const Site* shared = nullptr;
        for (const Site& s : ai)
            if (s == aj[0] || s == aj[1]) {
                shared = &s;
                break;
            }
        if (!shared) throw std::runtime_error("a beam is inside a cell");
        lies[b] = cell_of(*shared);
    }
    size_t n = sites.size();
    auto face = [&](size_t a, size_t b) { return sites[a] < sites[b] ? std::make_pair(a, b) : std::make_pair(b, a); };
    std::vector<Cell> cells(n);
    std::vector<std::vector<std::pair<Mat, double>>> mats(n);
    // On each face: what weighs on it, and whether anything on it is held.
    std::map<std::pair<size_t, size_t>, std::pair<double, bool>> faces;
    for (size_t v = 0; v < between.size(); v++) {
        size_t x = between[v][0], y = between[v][1];
        const Node& part = fine.nodes[v];
        size_t cs[2] = {x, y};
        for (size_t t = 0; t < (x == y ? 1u : 2u); t++) {
            auto& list = mats[cs[t]];
            auto it = std::find_if(list.begin(), list.end(), [&](const auto& e) { return same_mat(e.first, part.mat); });
            if (it != list.end())
                it->second += part.m;
            else
                list.push_back({part.mat, part.m});
        }
        if (x == y) {
            cells[x].free.push_back(v);
        } else {
            auto& f = faces[face(x, y)];
            f.first += part.m;
            f.second = f.second || part.held;
        }
    }
    // A fine node in a cell is itself there; on its face, that face.
    std::vector<size_t> place(fine.nodes.size(), SIZE_MAX);
    for (const Cell& cell : cells)
        for (size_t k = 0; k < cell.free.size(); k++) place[cell.free[k]] = k;
    for (size_t b = 0; b < fine.bonds.size(); b++) {
        size_t c = lies[b];
        auto at = [&](size_t v) {
            size_t x = between[v][0], y = between[v][1];
            if (x == c && y == c) return place[v];
            return cells[c].handle(x == c ? y : x);
        };
        size_t i = at(fine.bonds[b].i);
        size_t j = at(fine.bonds[b].j);
        cells[c].bonds.push_back({i, j, b});
    }
    // A cell is held if all in it is; a face, if anything on it is, or either cell.
    std::vector<bool> held(n);
    for (size_t c = 0; c < n; c++) {
        bool all = !cells[c].free.empty();
        for (size_t v : cells[c].free) all = all && fine.nodes[v].held;
        held[c] = all;
    }
    for (size_t c = 0; c < n; c++)
        for (size_t o : cells[c].across) faces[face(c, o)];
    auto mat_of = [&](std::initializer_list<size_t> cs) {
        std::vector<std::pair<Mat, double>> all;
        for (size_t c : cs)
            for (const auto& [m, w] : mats[c]) {
                auto it = std::find_if(all.begin(), all.end(), [&](const auto& e) { return same_mat(e.first, m); });
                if (it != all.end())
                    it->second += w;
                else
                    all.push_back({m, w});
            }
        if (all.empty()) return STONE;
        size_t best = 0;  // max_by: the last of equal maxima
        for (size_t k = 1; k < all.size(); k++)
            if (total_key(all[k].second) >= total_key(all[best].second)) best = k;
        return all[best].first;
    };
    auto centre_of = [&](size_t c) { return centre(sites[c], level); };
    std::map<std::pair<size_t, size_t>, size_t> node;
    std::vector<Node> nodes;
    for (const auto& [key, val] : faces) {
        node.emplace(key, nodes.size());
        auto [a, b] = key;
        nodes.push_back(Node{mul(add(centre_of(a), centre_of(b)), 0.5), val.first, mat_of({a, b}),
                             val.second || held[a] || held[b]});
    }
    double s = spacing(level);
    std::vector<std::vector<size_t>> ends(n);
    std::vector<std::vector<V3>> at(n);
    std::vector<Mat> mat(n);
    std::vector<Full> fulls(n);
    for (size_t c = 0; c < n; c++) {
        for (size_t o : cells[c].across) ends[c].push_back(node.at(face(c, o)));
        for (size_t k : ends[c]) at[c].push_back(nodes[k].x);
        mat[c] = mat_of({c});
    }
    for (size_t c = 0; c < n; c++)
        fulls[c] = against_full ? full(mat[c]) : Full{std::make_pair(1.0, 1.0), std::make_pair(1.0, 1.0)};
    using Found = std::vector<std::tuple<size_t, size_t, double, double>>;
    // Each cell's beams, all cells at once: its faces a and b, its stiffness along
    // it, how much stronger than its material.
    auto found = each<Found>(n, [&](size_t c) {
        const Cell& cell = cells[c];
        const std::vector<V3>& atc = at[c];
        const Mat& m = mat[c];
        const Full& fl = fulls[c];
        Found out;
        if (held[c] || atc.empty()) return out;
        auto [lat, cases] = responses(fine, cell, atc);
        // The stiffness between handles: what holds each, each case.
        size_t nf = cell.free.size();
        std::vector<std::vector<double>> k(cases.size(), std::vector<double>(cases.size(), 0.0));
        for (size_t cs = 0; cs < cases.size(); cs++)
            for (size_t b = 0; b < lat.bonds.size(); b++) {
                const V3& f = cases[cs][b];
                const std::pair<size_t, double> sides[2] = {{lat.bonds[b].j, 1.0}, {lat.bonds[b].i, -1.0}};
                for (const auto& [v, sign] : sides)
                    if (v >= nf)
                        for (size_t q = 0; q < 3; q++) k[3 * (v - nf) + q][cs] += sign * f[q];
            }
        auto piece = cell.pieces();
        for (const auto& [a, b, stiff] :
             gather_beams(k, atc, [&](size_t p, size_t q) { return piece[p] == piece[q]; })) {
            // The beam pulled alone, a unit apart: the finer matter's forces, and how
            // much of its strength it uses.
            V3 e = unit(sub(atc[b], atc[a]));
            std::vector<V3> pulled(lat.bonds.size());
            for (size_t q = 0; q < lat.bonds.size(); q++) {
                V3 f{0.0, 0.0, 0.0};
                for (size_t sx = 0; sx < 3; sx++)
                    f = add(f, add(mul(cases[3 * b + sx][q], e[sx] / 2.0), mul(cases[3 * a + sx][q], -e[sx] / 2.0)));
                pulled[q] = f;
            }
            // Each finer bond as much as it holds of the work done.
            auto u = used(lat, pulled);
            double hold = 0.0, work = 0.0;
            for (size_t q = 0; q < lat.bonds.size(); q++) {
                double w = lat.bonds[q].energy(pulled[q]);
                hold += w * u[q];
                work += w;
            }
            double fine_used = work > 0.0 ? hold / work : 0.0;
            double length = norm(sub(atc[b], atc[a]));
            double own = m.used(m.e / length, 0.0);
            double stronger = fine_used > 0.0 ? own / fine_used : 1.0;
            size_t cls = beam_class(atc[a], atc[b], centre_of(c));
            double section = stiff * length / m.e / (s * s);
            if (against_full) section = section * SECTION[cls] / fl[cls].first;
            out.emplace_back(a, b, section * s * s * m.e / length, stronger / fl[cls].second);
        }
        return out;
    });
    std::vector<Bond> bonds;
    for (size_t c = 0; c < n; c++) {
        const Cell& cell = cells[c];
        // The cell's weight on its faces, as much as each is joined.
        double mass = 0.0;
        for (size_t v : cell.free) mass += fine.nodes[v].m;
        std::vector<double> joined(at[c].size(), 0.0);
        for (const auto& [a, b, k, st] : found[c]) {
            joined[a] += k;
            joined[b] += k;
        }
        double total = 0.0;
        for (double j : joined) total += j;
        for (size_t h = 0; h < ends[c].size(); h++)
            nodes[ends[c][h]].m += mass * (total > 0.0 ? joined[h] / total : 1.0 / (double)at[c].size());
        for (const auto& [a, b, k, st] : found[c]) {
            if (nodes[ends[c][a]].held && nodes[ends[c][b]].held) continue;
            double length = norm(sub(at[c][b], at[c][a]));
            auto bs = beam(ends[c][a], ends[c][b], at[c][a], at[c][b], k * length / mat[c].e, mat[c].stronger(st));
            bonds.insert(bonds.end(), bs.begin(), bs.end());
        }
    }
    Lattice out;
    out.level = level;
    out.nodes = std::move(nodes);
    out.bonds = std::move(bonds);
    for (const auto& [key, val] : faces) out.around.push_back({sites[key.first], sites[key.second]});
    return out;
}

}  // namespace oracle
