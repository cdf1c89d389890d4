// ORACLE — test infrastructure only. The reference's example scenes, restated from
// statics/examples/statics.rs: they carry the only published known answers for the
// solve (docs/statics.md:236-247, "Used at 0").
#include <algorithm>
#include <cmath>
#include <string>

#include "statics_oracle.hpp"

namespace oracle {

static bool inside(double v, double lo, double hi) { return v >= lo - 1e-9 && v < hi - 1e-9; }  // statics.rs:18-20
static double to_radians(double d) { return d * (M_PI / 180.0); }
static double clampd(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

Lattice Scene::build_at(uint32_t level) const {  // statics.rs:32-38
    auto cells = solids(level, lo, hi, fill);
    if (bulk) hold_bulk(level, cells, *bulk);
    return build(level, cells);
}

Scene cantilever(Mat mat, double h, double l) {  // statics.rs:42-58
    Scene s;
    s.name = std::string("cantilever ") + mat.name;
    s.lo = {-0.6, -0.6, -0.6};
    s.hi = {l + 0.2, h + 0.6, h + 0.6};
    s.fill = [mat, h, l](V3 x, Mat& out, bool& held) {
        if (inside(x[0], -0.5, 0.0) && inside(x[1], -0.5, h + 0.5) && inside(x[2], -0.5, h + 0.5)) {
            out = STONE;
            held = true;
            return true;
        }
        if (inside(x[0], 0.0, l) && inside(x[1], 0.0, h) && inside(x[2], 0.0, h)) {
            out = mat;
            held = false;
            return true;
        }
        return false;
    };
    return s;
}

Scene tree(double lean, double side, double depth) {  // statics.rs:63-85
    double r = 0.3, h = 8.0, crown = 2.0;
    V3 axis{std::sin(to_radians(lean)), std::cos(to_radians(lean)), 0.0};
    V3 middle = mul(axis, h + crown * 0.8);
    Scene s;
    s.name = "tree";
    s.lo = {-4.0, -0.5, -3.0};
    s.hi = {6.0, h + 2.0 * crown + 0.5, 3.0};
    s.fill = [=](V3 x, Mat& out, bool& held) {
        if (x[1] < 0.0) {
            if (std::fabs(x[0]) < 1.0 && std::fabs(x[2]) < 1.0 && x[1] >= -0.4) {
                out = STONE;
                held = true;
                return true;
            }
            return false;
        }
        double along = dot(x, axis);
        V3 off = sub(x, mul(axis, clampd(along, 0.0, h)));
        if (norm(off) < r && along <= h) {
            bool cut = inside(x[1], 0.5, 0.5 + UNIT) && side * off[0] > r - 2.0 * r * depth;
            if (cut) return false;
            out = WOOD;
            held = false;
            return true;
        }
        if (norm(sub(x, middle)) < crown) {
            out = LEAVES;
            held = false;
            return true;
        }
        return false;
    };
    return s;
}

Scene portico(size_t cut, double slab) {  // statics.rs:88-111
    double w = 6.0, high = 3.0, c = 0.5;
    double columns[4][2] = {{0.0, 0.0}, {0.0, w - c}, {w - c, 0.0}, {w - c, w - c}};
    Scene s;
    s.name = "portico";
    s.lo = {-0.5, -0.5, -0.5};
    s.hi = {w + 0.5, high + slab + 0.5, w + 0.5};
    s.fill = [=](V3 x, Mat& out, bool& held) {
        if (inside(x[1], -0.25, 0.0) && inside(x[0], -0.5, w + 0.5) && inside(x[2], -0.5, w + 0.5)) {
            out = STONE;
            held = true;
            return true;
        }
        if (inside(x[1], high, high + slab) && inside(x[0], 0.0, w) && inside(x[2], 0.0, w)) {
            out = STONE;
            held = false;
            return true;
        }
        for (size_t k = 0; k < 4; k++) {
            const double* col = columns[k];
            if (inside(x[1], 0.0, high) && inside(x[0], col[0], col[0] + c) && inside(x[2], col[1], col[1] + c)) {
                if (k < 4 - cut || !inside(x[1], 1.0, 1.0 + UNIT)) {
                    out = STONE;
                    held = false;
                    return true;
                }
                return false;
            }
        }
        return false;
    };
    return s;
}

Scene rock(double w, double over) {  // statics.rs:114-133
    double h = w / 2.0;
    Scene s;
    s.name = "rock";
    s.lo = {-0.5, -0.5, -0.5};
    s.hi = {w + over + 0.5, h + 1.5, w + 0.5};
    s.fill = [=](V3 x, Mat& out, bool& held) {
        held = false;
        if (inside(x[1], -0.25, 0.0) && inside(x[0], -0.5, w + over + 0.5) && inside(x[2], -0.5, w + 0.5)) {
            out = STONE;
            held = true;
            return true;
        }
        if (inside(x[1], 0.0, h) && inside(x[0], 0.0, w) && inside(x[2], 0.0, w)) {
            out = STONE;
            return true;
        }
        if (inside(x[1], h, h + 1.0) && inside(x[0], 0.0, w + over) && inside(x[2], 0.0, w)) {
            out = SOIL;
            return true;
        }
        return false;
    };
    return s;
}

static double to_segment(V3 x, V3 a, V3 b) {  // statics.rs:211-215
    V3 ab = sub(b, a);
    double t = clampd(dot(sub(x, a), ab) / dot(ab, ab), 0.0, 1.0);
    return norm(sub(x, add(a, mul(ab, t))));
}

Scene tower(Mat mat, size_t cut) {  // statics.rs:221-256
    double base = 10.0, top = 2.0, high = 30.0, panel = 3.0, thick = 0.3;
    auto leg = [=](size_t k, double y) -> V3 {
        double w = (base + (top - base) * y / high) / 2.0;
        static const double sgn[4][2] = {{1.0, 1.0}, {-1.0, 1.0}, {-1.0, -1.0}, {1.0, -1.0}};
        return {sgn[k][0] * w, y, sgn[k][1] * w};
    };
    std::vector<std::pair<V3, V3>> members;
    for (size_t k = 0; k < 4; k++) {
        members.emplace_back(leg(k, -1.0), leg(k, high));
        double y = 0.0;
        while (y < high - 1e-9) {
            double next = y + panel;
            members.emplace_back(leg(k, next), leg((k + 1) % 4, next));
            members.emplace_back(leg(k, y), leg((k + 1) % 4, next));
            members.emplace_back(leg((k + 1) % 4, y), leg(k, next));
            y = next;
        }
    }
    Scene s;
    s.name = "tower";
    s.lo = {-base / 2.0 - 2.0, -2.5, -base / 2.0 - 2.0};
    s.hi = {base / 2.0 + 2.0, high + 0.5, base / 2.0 + 2.0};
    s.fill = [=](V3 x, Mat& out, bool& held) {
        held = false;
        for (size_t k = 0; k < 4; k++) {
            V3 foot = leg(k, 0.0);
            if (inside(x[1], -2.5, 0.0) && std::fabs(x[0] - foot[0]) < 1.5 && std::fabs(x[2] - foot[2]) < 1.5) {
                out = STEEL;
                return true;
            }
        }
        bool gone = false;
        for (size_t k = 0; k < cut && !gone; k++)
            gone = inside(x[1], 1.0, 2.5) && to_segment(x, leg(k, -1.0), leg(k, high)) < thick;
        if (gone) return false;
        for (auto& ab : members)
            if (to_segment(x, ab.first, ab.second) < thick / 2.0) {
                out = mat;
                return true;
            }
        return false;
    };
    s.bulk = 0.75;
    return s;
}

Scene pendant(bool apart) {  // statics.rs:285-303
    Scene s;
    s.name = "pendant";
    s.lo = {-0.6, -0.6, -0.6};
    s.hi = {1.2, 1.1, 1.1};
    s.fill = [=](V3 x, Mat& out, bool& held) {
        if (inside(x[0], -0.5, 0.0) && inside(x[1], -0.5, 1.0) && inside(x[2], -0.5, 1.0)) {
            out = STONE;
            held = true;
            return true;
        }
        if ((inside(x[0], 0.0, 1.0) && inside(x[1], 0.0, 0.5) && inside(x[2], 0.0, 0.5)) ||
            (inside(x[0], 0.5, 0.75) && inside(x[1], -0.375, apart ? -0.125 : 0.0) && inside(x[2], 0.0, 0.25))) {
            out = STONE;
            held = false;
            return true;
        }
        return false;
    };
    return s;
}

}  // namespace oracle
