// Level 0 of voxel pieces without stored block values. The setup (block inverses, the
// prolongator's K P0, the Galerkin product K P and a top factorised at level 0) reads
// the blocks of the reference's level-0 operator (statics/src/bodies.rs:126-170), but
// every block is one or two 6x6 pieces of a cell's template scaled by that cell's
// stiffness: the diagonal block of a part is its lesser cell's and its greater cell's
// blocks on the shared face, an off-diagonal block K_kq is the one cell that holds both
// faces (two cells share at most one face). So the assembled pattern keeps, per stored
// block, one byte saying where it comes from, and the values are made when read, in the
// same arithmetic the stored values had.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace sc {

constexpr uint8_t K0_DIAG = 0xff;  // desc of a diagonal block; else side << 3 | slot

// The cell-template blocks of level 0: per stored block its desc; per part its axis and
// cells; per cell its faces and stiffness; the template scaled by the spacing (36 x 36).
struct K0View {
    const uint8_t* desc;
    const int8_t* axis;
    const int32_t* cella;
    const int32_t* cellb;
    const int4* cell;
    const double* tpl_s;
};

// What a row needs: its axis and the stiffness of its lesser (A) and greater (B) cell.
struct K0Row {
    int ax;
    bool hasA, hasB;
    double kA, kB;
};

__device__ __forceinline__ K0Row k0_row(const K0View& v, int64_t k) {
    K0Row r;
    r.ax = v.axis[k];
    int32_t A = v.cella[k], B = v.cellb[k];
    r.hasA = A >= 0;
    r.hasB = B >= 0;
    r.kA = r.hasA ? (double)__int_as_float(__ldg(&v.cell[2 * A + 1].z)) : 0.0;
    r.kB = r.hasB ? (double)__int_as_float(__ldg(&v.cell[2 * B + 1].z)) : 0.0;
    return r;
}

// Entry (i, j) of the block with descriptor d in row r; T is the scaled template.
__device__ __forceinline__ double k0_entry(const double* __restrict__ T, const K0Row& r, uint8_t d, int i, int j) {
    const int slA = 2 * r.ax + 1, slB = 2 * r.ax;
    if (d == K0_DIAG) {
        double v = 0.0;
        if (r.hasA) v += r.kA * T[(6 * slA + i) * 36 + 6 * slA + j];
        if (r.hasB) v += r.kB * T[(6 * slB + i) * 36 + 6 * slB + j];
        return v;
    }
    const int slot = d & 7;
    return (d >> 3) ? r.kB * T[(6 * slB + i) * 36 + 6 * slot + j] : r.kA * T[(6 * slA + i) * 36 + 6 * slot + j];
}

}  // namespace sc
