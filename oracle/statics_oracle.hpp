// ORACLE — test infrastructure only, never part of the product.
//
// A CPU restatement of the reference's `statics` crate (SupraSummus/parallax-world,
// Rust): statics/src/model.rs, statics/src/lattice.rs and statics/src/bodies.rs,
// plus the face order of lattice/src/lib.rs:64 (VOXEL_FACES), and statics/src/gather.rs
// (gather_oracle.cpp). Loop orders, merge
// orders and floating-point operation orders follow the Rust source line by line so
// that node numbering, part numbering and body ids are bit-exact, and FP64 values are
// the reference's up to the sign of zero (Rust's float `sum()` folds from -0.0).
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load this.
// Parity status: the reference ships no test that pins `motions`; the oracle is pinned
// by the reference's `cells_nest` test (statics/src/lattice.rs:170-181) and by the
// known answers its docs publish (docs/statics.md:236-247), reproduced in tests/.
#pragma once
#include <algorithm>
#include <array>
#include <cstdint>
#include <functional>
#include <memory>
#include <optional>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

namespace oracle {

using V3 = std::array<double, 3>;
using Six = std::array<double, 6>;
using M3 = std::array<std::array<double, 3>, 3>;
using M6 = std::array<std::array<double, 6>, 6>;
using Site = std::array<int64_t, 3>;

// ---- statics/src/model.rs ------------------------------------------------------
V3 add(V3 a, V3 b);
V3 sub(V3 a, V3 b);
V3 mul(V3 a, double s);
double dot(V3 a, V3 b);
V3 cross(V3 a, V3 b);
double norm(V3 a);
V3 unit(V3 a);

constexpr double GRAVITY = 9.81;  // model.rs:38

struct Mat {  // model.rs:43-51
    const char* name;
    double rho, e, g, ft, fc, fs;
    double used(double s1, double s3) const;  // model.rs:66-68
    Mat stronger(double by) const;            // model.rs:71-73
};

extern const Mat STONE, WOOD, MASONRY, SOIL, STEEL, LEAVES;  // model.rs:53-58

struct Node {  // model.rs:92-98
    V3 x;
    double m;
    Mat mat;
    bool held;
};

struct Bond {  // model.rs:101-111
    size_t i, j;
    V3 p, n;
    double a, d;
    Mat mat;
    V3 force(V3 delta) const;    // model.rs:115-119
    double used(V3 force) const; // model.rs:123-129
    double energy(V3 force) const;  // model.rs:132-136
    M3 stiffness() const;        // model.rs:139-149
};

// ---- statics/src/lattice.rs ----------------------------------------------------
constexpr double UNIT = 0.125;          // lattice.rs:16
constexpr size_t PER_BEAM = 4;          // lattice.rs:19
constexpr double SECTION[2] = {0.336, 0.336};  // lattice.rs:25
extern const int VOXEL_FACES[6][3];     // lattice/src/lib.rs:64

size_t beam_class(V3 a, V3 b, V3 c);    // lattice.rs:29-32
double spacing(uint32_t level);         // lattice.rs:34-36
V3 centre(Site site, uint32_t level);   // lattice.rs:39-41
Site coarse_site(Site p, uint32_t l);   // lattice.rs:45-47

struct Solid {  // lattice.rs:54-58
    Site site;
    Mat mat;
    bool held;
};

struct Lattice {  // lattice.rs:61-71
    uint32_t level = 0;
    std::vector<Node> nodes;
    std::vector<Bond> bonds;
    std::vector<std::array<Site, 2>> around;
};

using Fill = std::function<bool(V3, Mat&, bool&)>;

std::array<Bond, 4> beam(size_t i, size_t j, V3 a, V3 b, double area, Mat mat);  // lattice.rs:76-84
std::vector<Solid> solids(uint32_t level, V3 lo, V3 hi, const Fill& fill);      // lattice.rs:87-102
void hold_bulk(uint32_t level, std::vector<Solid>& solids, double radius);     // lattice.rs:107-119
Lattice build(uint32_t level, const std::vector<Solid>& solids);               // lattice.rs:124-163

// ---- statics/src/bodies.rs -----------------------------------------------------
struct Work {  // bodies.rs:331
    double v = 0.0;
};

Six shift(Six x, V3 r);  // bodies.rs:44-47

/// Threads used by `each` (bodies.rs:51-69); 0 = all hardware threads.
void set_threads(int n);
int threads();

// bodies.rs:51-69: contiguous chunks over the threads, sequential below 256.
template <class T, class F>
std::vector<T> each(size_t n, const F& f) {
    size_t th = (size_t)threads();
    std::vector<T> out(n);
    if (n < 256 || th == 1) {
        for (size_t i = 0; i < n; i++) out[i] = f(i);
        return out;
    }
    size_t size = (n + th - 1) / th;
    std::vector<std::thread> pool;
    for (size_t start = 0; start < n; start += size) {
        size_t end = std::min(n, start + size);
        pool.emplace_back([&, start, end] {
            for (size_t i = start; i < end; i++) out[i] = f(i);
        });
    }
    for (auto& t : pool) t.join();
    return out;
}

size_t find(std::vector<size_t>& p, size_t a);  // bodies.rs:628-634

/// What one `motions` call built and did, for parity checks against the GPU path.
struct Hierarchy {
    std::vector<size_t> counts;             // parts per level
    std::vector<size_t> pairs;              // pairs (i<j blocks) per level
    std::vector<double> steps;              // smoother step per level
    std::vector<std::vector<size_t>> up;    // body of each part, level l -> l+1
    size_t iterations = 0;                  // CG iterations taken
    double setup_seconds = 0, solve_seconds = 0;
};

struct MotionsOptions {
    double tol = 1e-6;   // bodies.rs:432
    size_t few = 64;     // bodies.rs:430
    size_t max_iter = 100000;  // bodies.rs:351
};

/// bodies.rs:429-468, with the tolerance and FEW made parameters.
std::vector<Six> motions(const Lattice& lattice, const std::vector<bool>& alive, const std::vector<bool>& gone,
                         const std::function<Six(size_t)>& loads, Work& work, const MotionsOptions& opt = {},
                         Hierarchy* hier = nullptr);

std::vector<V3> forces(const Lattice& lattice, const std::vector<bool>& alive, const std::vector<bool>& gone,
                       Work& work);                                                  // bodies.rs:407-417
std::vector<V3> moved(const Lattice& lattice, const std::vector<Six>& x);           // bodies.rs:420-423
std::vector<double> used(const Lattice& lattice, const std::vector<V3>& force);     // bodies.rs:544-546
std::vector<double> used_standing(const Lattice& lattice);                          // bodies.rs:550-554
std::vector<bool> joined_to_held(const std::vector<Node>& nodes, const std::vector<Bond>& bonds,
                                 const std::vector<bool>& alive);                   // bodies.rs:557-574
struct Outcome {  // bodies.rs:498-507
    double fallen;
    std::vector<bool> gone;
    size_t rounds;
    double work;
};
Outcome settle(const Lattice& lattice);  // bodies.rs:511-541
constexpr double MARGIN = 2.0;           // bodies.rs:605
void as_generated(Lattice& lattice, const Lattice& generated);  // bodies.rs:611-625
M6 invert(const M6& m);                  // bodies.rs:576-602
/// Level 0's operator alone (Level::new + apply), all bonds alive, no node gone.
std::vector<Six> level0_apply(const Lattice& lattice, const std::vector<Six>& x_parts);

// ---- statics/src/gather.rs -----------------------------------------------------
/// A full cell's beams by class (180°, 90°): section over the spacing squared, and
/// how much stronger than the material (gather.rs:199-226).
using Full = std::array<std::pair<double, double>, 2>;
Full full(const Mat& mat);                                 // gather.rs:203-226
Lattice measured(const Lattice& fine, bool against_full);  // gather.rs:230-395
Lattice gathered(const Lattice& fine);                     // gather.rs:193-195
/// gather.rs:164-184: Gauss–Jordan with `rhs` right-hand columns; rows of the answer.
std::vector<std::vector<double>> gather_solve(std::vector<std::vector<double>> a, size_t rhs);
/// gather.rs:119-161: (a, b, stiffness) of the beams nearest the handles' stiffness k.
std::vector<std::tuple<size_t, size_t, double>> gather_beams(const std::vector<std::vector<double>>& k,
                                                             const std::vector<V3>& at,
                                                             const std::function<bool(size_t, size_t)>& joined);

// ---- restated example scenes (statics/examples/statics.rs) ---------------------
struct Scene {
    std::string name;
    V3 lo, hi;
    Fill fill;
    std::optional<double> bulk;
    Lattice build_at(uint32_t level) const;  // statics.rs:32-38
};
Scene cantilever(Mat mat, double h, double l);          // statics.rs:42-58
Scene tree(double lean, double side, double depth);     // statics.rs:63-85
Scene portico(size_t cut, double slab);                 // statics.rs:88-111
Scene rock(double w, double over);                      // statics.rs:114-133
Scene tower(Mat mat, size_t cut);                       // statics.rs:221-256
Scene pendant(bool apart);                              // statics.rs:285-303

// ---- synthetic voxel pieces (the workload's structures) -------------------------
/// A grid of cells, x slowest, z fastest (the order `solids` visits sites):
/// state 0 empty, 1 free, 2 held; k is each cell's stiffness (E = k, G = g_over_e*k).
/// Density `rho` (512 gives each level-0 cell a weight of 1). `cell_of_bond`, if
/// given, receives the flat cell index each bond belongs to.
Lattice grid_lattice(int nx, int ny, int nz, const uint8_t* state, const float* k, double g_over_e, double rho,
                     std::vector<int64_t>* cell_of_bond = nullptr);

}  // namespace oracle
