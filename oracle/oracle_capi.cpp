// ORACLE — test infrastructure only. A flat C interface over the restatement so that
// tests/ and bench.py's CPU-baseline leg can drive it through ctypes.
#include <chrono>
#include <cmath>
#include <cstring>
#include <exception>
#include <memory>

#include "statics_oracle.hpp"

using namespace oracle;

namespace {
struct Handle {
    Lattice lat;
    std::vector<int64_t> cell_of_bond;  // grid pieces only
};
const Mat* mat_of(int i) {
    static const Mat* all[6] = {&STONE, &WOOD, &MASONRY, &SOIL, &STEEL, &LEAVES};
    return (i >= 0 && i < 6) ? all[i] : &STONE;
}
}  // namespace

extern "C" {

void or_set_threads(int n) { set_threads(n); }
int or_threads() { return threads(); }

// kind: 0 cantilever(mat, h=a, l=b); 1 tree(lean=a, side=b, depth=c); 2 portico(cut=a, slab=b);
// 3 rock(w=a, over=b); 4 tower(mat, cut=a); 5 pendant(apart=a!=0).
void* or_scene(int kind, int mat, double a, double b, double c, int level) {
    Scene s;
    switch (kind) {
        case 0: s = cantilever(*mat_of(mat), a, b); break;
        case 1: s = tree(a, b, c); break;
        case 2: s = portico((size_t)a, b); break;
        case 3: s = rock(a, b); break;
        case 4: s = tower(*mat_of(mat), (size_t)a); break;
        case 5: s = pendant(a != 0.0); break;
        default: return nullptr;
    }
    auto* h = new Handle;
    h->lat = s.build_at((uint32_t)level);
    return h;
}

// build(level, solids(level, lo, hi, fill)) (lattice.rs:87-163) with the fill taking
// every site whose centre x has |x_k| < half[k] on each axis, of material `mat`, free:
// the steel bar of gather.rs:403-405 and the full block of statics.rs:352.
void* or_block(int mat, const double* lo, const double* hi, const double* half, int level) {
    const Mat m = *mat_of(mat);
    V3 h{half[0], half[1], half[2]};
    Fill fill = [m, h](V3 x, Mat& out, bool& held) {
        if (!(std::fabs(x[0]) < h[0] && std::fabs(x[1]) < h[1] && std::fabs(x[2]) < h[2])) return false;
        out = m;
        held = false;
        return true;
    };
    auto* hd = new Handle;
    hd->lat = build((uint32_t)level, solids((uint32_t)level, V3{lo[0], lo[1], lo[2]}, V3{hi[0], hi[1], hi[2]}, fill));
    return hd;
}

void* or_grid(int nx, int ny, int nz, const uint8_t* state, const float* k, double g_over_e, double rho) {
    auto* h = new Handle;
    h->lat = grid_lattice(nx, ny, nz, state, k, g_over_e, rho, &h->cell_of_bond);
    return h;
}

void or_free(void* p) { delete static_cast<Handle*>(p); }

void or_sizes(void* p, int64_t* n_nodes, int64_t* n_bonds) {
    auto* h = static_cast<Handle*>(p);
    *n_nodes = (int64_t)h->lat.nodes.size();
    *n_bonds = (int64_t)h->lat.bonds.size();
}

// Flat structure-of-arrays copy of the lattice; any pointer may be null.
void or_export(void* p, double* x, double* m, uint8_t* held, int64_t* around, int64_t* bi, int64_t* bj, double* bp,
               double* bn, double* ba, double* bd, double* be, double* bg, int64_t* cell_of_bond) {
    auto* h = static_cast<Handle*>(p);
    const Lattice& L = h->lat;
    for (size_t v = 0; v < L.nodes.size(); v++) {
        if (x)
            for (int k = 0; k < 3; k++) x[3 * v + k] = L.nodes[v].x[k];
        if (m) m[v] = L.nodes[v].m;
        if (held) held[v] = L.nodes[v].held ? 1 : 0;
        if (around)
            for (int s = 0; s < 2; s++)
                for (int k = 0; k < 3; k++) around[6 * v + 3 * s + k] = L.around[v][s][k];
    }
    for (size_t b = 0; b < L.bonds.size(); b++) {
        const Bond& B = L.bonds[b];
        if (bi) bi[b] = (int64_t)B.i;
        if (bj) bj[b] = (int64_t)B.j;
        for (int k = 0; k < 3; k++) {
            if (bp) bp[3 * b + k] = B.p[k];
            if (bn) bn[3 * b + k] = B.n[k];
        }
        if (ba) ba[b] = B.a;
        if (bd) bd[b] = B.d;
        if (be) be[b] = B.mat.e;
        if (bg) bg[b] = B.mat.g;
        if (cell_of_bond) cell_of_bond[b] = b < h->cell_of_bond.size() ? h->cell_of_bond[b] : -1;
    }
}

// Each bond's strengths (Mat::ft, fc, fs of its material, statics/src/model.rs:43-51).
void or_strengths(void* p, double* ft, double* fc, double* fs) {
    auto* h = static_cast<Handle*>(p);
    const Lattice& L = h->lat;
    for (size_t b = 0; b < L.bonds.size(); b++) {
        ft[b] = L.bonds[b].mat.ft;
        fc[b] = L.bonds[b].mat.fc;
        fs[b] = L.bonds[b].mat.fs;
    }
}

// motions (bodies.rs:429-468) with explicit loads (6 per node). Hierarchy outputs
// (any may be null): counts/pairs/steps per level (capacity max_levels), n_levels,
// and the concatenated `up` arrays of every coarsening (capacity up_cap).
int or_motions(void* p, const uint8_t* alive, const uint8_t* gone, const double* loads, double tol, int64_t few,
               int64_t max_iter, double* out, double* work, int64_t* iterations, double* seconds,
               int64_t* counts, int64_t* pairs, double* steps, int64_t max_levels, int64_t* n_levels,
               int32_t* up_concat, int64_t up_cap) {
    auto* h = static_cast<Handle*>(p);
    const Lattice& L = h->lat;
    std::vector<bool> al(L.bonds.size(), true), gn(L.nodes.size(), false);
    if (alive)
        for (size_t b = 0; b < al.size(); b++) al[b] = alive[b] != 0;
    if (gone)
        for (size_t v = 0; v < gn.size(); v++) gn[v] = gone[v] != 0;
    MotionsOptions opt;
    opt.tol = tol;
    opt.few = (size_t)few;
    opt.max_iter = (size_t)max_iter;
    Hierarchy hier;
    Work w;
    auto t0 = std::chrono::steady_clock::now();
    auto x = motions(
        L, al, gn,
        [&](size_t v) {
            Six s;
            for (int k = 0; k < 6; k++) s[k] = loads[6 * v + k];
            return s;
        },
        w, opt, &hier);
    auto t1 = std::chrono::steady_clock::now();
    for (size_t v = 0; v < x.size(); v++)
        for (int k = 0; k < 6; k++) out[6 * v + k] = x[v][k];
    if (work) *work = w.v;
    if (iterations) *iterations = (int64_t)hier.iterations;
    if (seconds) {
        seconds[0] = std::chrono::duration<double>(t1 - t0).count();
        seconds[1] = hier.setup_seconds;
        seconds[2] = hier.solve_seconds;
    }
    int64_t nl = (int64_t)hier.counts.size();
    if (n_levels) *n_levels = nl;
    for (int64_t l = 0; l < nl && l < max_levels; l++) {
        if (counts) counts[l] = (int64_t)hier.counts[l];
        if (pairs) pairs[l] = (int64_t)hier.pairs[l];
        if (steps) steps[l] = hier.steps[l];
    }
    if (up_concat) {
        int64_t pos = 0;
        for (auto& u : hier.up)
            for (size_t k = 0; k < u.size() && pos < up_cap; k++) up_concat[pos++] = (int32_t)u[k];
    }
    return 0;
}

void or_moved(void* p, const double* x, double* f) {
    auto* h = static_cast<Handle*>(p);
    std::vector<Six> xs(h->lat.nodes.size());
    for (size_t v = 0; v < xs.size(); v++)
        for (int k = 0; k < 6; k++) xs[v][k] = x[6 * v + k];
    auto fs = moved(h->lat, xs);
    for (size_t b = 0; b < fs.size(); b++)
        for (int k = 0; k < 3; k++) f[3 * b + k] = fs[b][k];
}

// Strain energy per grid cell, sum over its bonds of Bond::energy(moved force)
// (model.rs:132-136): with K linear in the cell's stiffness k, the compliance
// gradient is dC/dk = -2 U / k.
void or_cell_energy(void* p, const double* x, int64_t n_cells, double* energy) {
    auto* h = static_cast<Handle*>(p);
    std::vector<Six> xs(h->lat.nodes.size());
    for (size_t v = 0; v < xs.size(); v++)
        for (int k = 0; k < 6; k++) xs[v][k] = x[6 * v + k];
    auto fs = moved(h->lat, xs);
    for (int64_t c = 0; c < n_cells; c++) energy[c] = 0.0;
    for (size_t b = 0; b < fs.size(); b++) {
        int64_t c = h->cell_of_bond[b];
        if (c >= 0 && c < n_cells) energy[c] += h->lat.bonds[b].energy(fs[b]);
    }
}

void or_used_standing(void* p, double* used_out) {
    auto* h = static_cast<Handle*>(p);
    auto u = used_standing(h->lat);
    for (size_t b = 0; b < u.size(); b++) used_out[b] = u[b];
}

void or_settle(void* p, double* fallen, int64_t* rounds, uint8_t* gone) {
    auto* h = static_cast<Handle*>(p);
    auto o = settle(h->lat);
    if (fallen) *fallen = o.fallen;
    if (rounds) *rounds = (int64_t)o.rounds;
    if (gone)
        for (size_t v = 0; v < o.gone.size(); v++) gone[v] = o.gone[v] ? 1 : 0;
}

// A copy of a lattice (Lattice::clone), as a new handle.
void* or_clone(void* p) {
    auto* h = new Handle;
    *h = *static_cast<Handle*>(p);
    return h;
}

void or_as_generated(void* lattice, void* generated) {
    as_generated(static_cast<Handle*>(lattice)->lat, static_cast<Handle*>(generated)->lat);
}

void or_level0_apply(void* p, int64_t n_parts, const double* x, double* y) {
    auto* h = static_cast<Handle*>(p);
    std::vector<Six> xs((size_t)n_parts);
    for (int64_t k = 0; k < n_parts; k++)
        for (int s = 0; s < 6; s++) xs[k][s] = x[6 * k + s];
    auto ys = level0_apply(h->lat, xs);
    for (size_t k = 0; k < ys.size(); k++)
        for (int s = 0; s < 6; s++) y[6 * k + s] = ys[k][s];
}

void or_invert(const double* m, double* out) {
    M6 a;
    for (int r = 0; r < 6; r++)
        for (int c = 0; c < 6; c++) a[r][c] = m[6 * r + c];
    M6 inv = invert(a);
    for (int r = 0; r < 6; r++)
        for (int c = 0; c < 6; c++) out[6 * r + c] = inv[r][c];
}

// gather.rs:193-195 (against_full != 0) or measured(fine, false), gather.rs:230-395:
// the next level up, as a new lattice handle (NULL where the restatement throws).
void* or_gather(void* p, int against_full) {
    try {
        auto* h = new Handle;
        h->lat = measured(static_cast<Handle*>(p)->lat, against_full != 0);
        return h;
    } catch (const std::exception&) {
        return nullptr;
    }
}

// gather.rs:203-226 for material `mat`: per class (180°, 90°) the section over the
// spacing squared and the strength over the material's; out holds 4 values.
void or_full(int mat, double* out) {
    Full f = full(*mat_of(mat));
    for (int k = 0; k < 2; k++) {
        out[2 * k] = f[k].first;
        out[2 * k + 1] = f[k].second;
    }
}

// Each node's material as an index into (stone, wood, masonry, soil, steel, leaves),
// -1 for another; each bond's tensile strength over its material's own (Mat::stronger).
void or_materials(void* p, int32_t* node_mat, int32_t* bond_mat, double* bond_stronger) {
    static const Mat* all[6] = {&STONE, &WOOD, &MASONRY, &SOIL, &STEEL, &LEAVES};
    auto index = [&](const Mat& m) {
        for (int k = 0; k < 6; k++)
            if (std::strcmp(all[k]->name, m.name) == 0) return k;
        return -1;
    };
    const Lattice& L = static_cast<Handle*>(p)->lat;
    for (size_t v = 0; v < L.nodes.size(); v++)
        if (node_mat) node_mat[v] = index(L.nodes[v].mat);
    for (size_t b = 0; b < L.bonds.size(); b++) {
        int k = index(L.bonds[b].mat);
        if (bond_mat) bond_mat[b] = k;
        if (bond_stronger) bond_stronger[b] = k >= 0 ? L.bonds[b].mat.ft / all[k]->ft : 0.0;
    }
}

int64_t or_coarse_site(const int64_t* p, uint32_t l, int64_t* out) {
    Site s = coarse_site(Site{p[0], p[1], p[2]}, l);
    for (int k = 0; k < 3; k++) out[k] = s[k];
    return 0;
}
}
