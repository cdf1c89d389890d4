// The engine solver's levels (mechanics::solve::Solver, mechanics/src/solve.rs:188-203,
// 356-386) as they sit on the device: made there by mech_levels.cu, read by mech.cu's
// V-cycles and conjugate gradients.
#pragma once
#include <cstdint>
#include <vector>

#include "kernels.cuh"

namespace sc {

constexpr size_t MECH_DIRECT = 24;  // solve.rs:23: a level this small is solved directly

// One coarse level: its parts (rigid aggregates of the finer level's), their blocks as
// full 6x6 block rows, block inverses and smoother step, or the direct top's inverse.
struct MechLevel {
    int64_t n = 0;         // parts
    DBuf<int32_t> of;      // finer part -> its part here
    DBuf<double> r;        // 3 per finer part: its offset from its part's centre
    DBuf<int64_t> mptr;    // n + 1
    DBuf<int32_t> mem;     // each part's finer parts, in order
    DBuf<int64_t> rowptr;  // n + 1
    DBuf<int32_t> col;
    DBuf<double> val, inv, step;  // 36 a block; 36 a part; 1
    int64_t nnzb = 0;
    double step_h = 0.0;  // the step, on the host too (0 at the direct top)
    bool direct = false;
    DBuf<double> top_inv;  // (6 n)^2 at the direct top
    DBuf<double> b, x, res, t;
};

// The nodes' 3x3 block rows, inverses and step, and the coarse levels.
struct MechLevels {
    int64_t n0 = 0;
    DBuf<int64_t> rowptr0;
    DBuf<int32_t> col0;
    DBuf<double> val0, inv0;
    double step0 = 1.0;
    std::vector<MechLevel> lv;
};

// Solver::new on the context's device, from the system's host arrays (the layout of
// sc_mech_solve). The same additions in the same order as the reference (and as
// mech.cu's host copy), so the parts and steps are the same bit for bit.
void mech_device_levels(Context& ctx, int64_t n, const int64_t* sites, const double* at, const double* diag,
                        int64_t npairs, const uint32_t* pi, const uint32_t* pj, const double* pb, double size,
                        MechLevels& out);

// The direct top's inverse operator (solve.rs:320-347) on the host: n parts' 6x6
// diagonal blocks and the pairs' blocks (36 values each, row-major), laid out as
// solve.rs:123-135 lays it out.
std::vector<double> mech_top_inverse(int64_t n, const double* diag36, int64_t npairs, const uint32_t* pi,
                                     const uint32_t* pj, const double* pm36, double size);

}  // namespace sc
