// Device arithmetic shared by the level-0 kernels of voxel pieces (grid.cu's kernels
// in the reference's part order, brick.cu's in brick order): six-vector loads and
// stores, the cell template's row strips (template_gen.cuh), the block-Jacobi factor of a
// face node and the stencil's epilogue modes.
#pragma once
#include <cstdint>

#include "template_gen.cuh"

namespace sc {
namespace {

template <int SLOT, class T>
__device__ __forceinline__ void strip(const T (&x)[6][6], T (&acc)[6]) {
    if constexpr (SLOT == 0) strip_0<T>(x, acc);
    if constexpr (SLOT == 1) strip_1<T>(x, acc);
    if constexpr (SLOT == 2) strip_2<T>(x, acc);
    if constexpr (SLOT == 3) strip_3<T>(x, acc);
    if constexpr (SLOT == 4) strip_4<T>(x, acc);
    if constexpr (SLOT == 5) strip_5<T>(x, acc);
}

template <class T>
__device__ __forceinline__ void load6(const T* __restrict__ v, int32_t k, T (&o)[6]) {
    if constexpr (sizeof(T) == 8) {
        const double2* p = reinterpret_cast<const double2*>(v + 6 * (int64_t)k);
        double2 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
        o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y; o[4] = c.x; o[5] = c.y;
    } else {
        const float2* p = reinterpret_cast<const float2*>(v + 6 * (int64_t)k);
        float2 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
        o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y; o[4] = c.x; o[5] = c.y;
    }
}
template <class T>
__device__ __forceinline__ void store6(T* __restrict__ v, int64_t k, const T (&o)[6]) {
    if constexpr (sizeof(T) == 8) {
        double2* p = reinterpret_cast<double2*>(v + 6 * k);
        p[0] = make_double2(o[0], o[1]);
        p[1] = make_double2(o[2], o[3]);
        p[2] = make_double2(o[4], o[5]);
    } else {
        float2* p = reinterpret_cast<float2*>(v + 6 * k);
        p[0] = make_float2(o[0], o[1]);
        p[1] = make_float2(o[2], o[3]);
        p[2] = make_float2(o[4], o[5]);
    }
}

// t += sum over the six faces F of TPL block (SLOT, F) * x_F. The six faces' loads are
// issued together, branch-free (a held face reads the part's own x and is masked to
// zero), so a thread waits for one round of gathers per cell.
template <int SLOT, int F, class T>
__device__ __forceinline__ void face_macs(const T (&xs)[6][6], T (&t)[6]) {
    if constexpr (F < 6) {
        Blk<SLOT, F>::mac(xs[F], t);
        face_macs<SLOT, F + 1, T>(xs, t);
    }
}

// D^-1 v for a face node on axis AX between cells of stiffness kA (lesser) and kB
// (greater), spacing s: D = s Dm (kA M+ + kB M-) Dm with Dm = diag(1,1,1,s,s,s) and
// kA M+ + kB M- = V^-T diag(kA lambda + kB) V^-1 (generalised eigenvectors of the two
// face blocks, template_gen.cuh), so D^-1 v = (1/s) Dm^-1 V diag(1/(kA lambda + kB)) V' Dm^-1 v.
// (The spacing's powers divide as products with 1/s: one division instead of nine, and
// the same values, the spacing 1/8 being a power of two.)
template <int AX, class T>
__device__ __forceinline__ void dinv(T kA, T kB, T s, const T (&v)[6], T (&y)[6]) {
    const T is = T(1) / s, is2 = is * is;
    T vt[6] = {v[0], v[1], v[2], v[3] * is, v[4] * is, v[5] * is};
    T w[6];
#pragma unroll
    for (int i = 0; i < 6; i++) {
        T acc = T(0);
#pragma unroll
        for (int j = 0; j < 6; j++) acc = fma((T)JAC_V_DEV[AX][j][i], vt[j], acc);
        w[i] = acc / fma(kA, (T)JAC_L_DEV[AX][i], kB);
    }
#pragma unroll
    for (int i = 0; i < 6; i++) {
        T acc = T(0);
#pragma unroll
        for (int j = 0; j < 6; j++) acc = fma((T)JAC_V_DEV[AX][i][j], w[j], acc);
        y[i] = i < 3 ? acc * is : acc * is2;
    }
}

// Epilogues of the stencil (Kx is the row's K x):
//   ST_Y        y = Kx
//   ST_RES      y = r - Kx
//   ST_RES_JAC  y = r - Kx, y2 = D^-1 (r - Kx)
//   ST_RES_W    y = r - w Kx                          (w the piece's smoother step)
//   ST_PROLONG  y += x - w D^-1 Kx                    (x = P0 z; y accumulates)
//   ST_SMOOTH   y = x + w D^-1 (r - Kx)
enum { ST_Y = 0, ST_RES = 1, ST_RES_JAC = 2, ST_RES_W = 3, ST_PROLONG = 4, ST_SMOOTH = 5 };

}  // namespace
}  // namespace sc
