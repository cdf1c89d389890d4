"""Generate template_gen.cuh: the stiffness of one full level-0 cell, as constants.

A free cell joins its 6 face nodes by 15 beams of 4 bonds each (the reference's
`build` and `beam`, statics/src/lattice.rs:76-84, 124-163, with SECTION 0.336 for both
beam classes, lattice.rs:25). Every bond adds T_i' S T_i to node i's own block and
-T_i' S T_j to the pair (i, j), with S = (E nn' + G (I - nn')) a/d and T_v = [I | -[r]x],
r = bond point - node centre (statics/src/model.rs:139-149, statics/src/bodies.rs:137-161).

For a cell of spacing s, stiffness E = k and G = 0.4 k (the ratio of every reference
material, statics/src/model.rs:53-58), the 36x36 cell matrix is

    K_c = k * s * D_s Kt D_s,   D_s = diag(1, 1, 1, s, s, s),

with Kt this file's template at s = 1, E = 1, G = 0.4. Face slots follow VOXEL_FACES
(lattice/src/lib.rs:64): -x, +x, -y, +y, -z, +z.

Emitted:
  * TPL[36][36]            the template (host and device constant tables);
  * stencil_rows<axis>     unrolled products of the two 6-row strips a face node on
                           `axis` meets (as the + face of its lesser cell, slot 2*axis+1,
                           and as the - face of its greater cell, slot 2*axis), with the
                           zero entries left out, for double and float;
  * JAC_V / JAC_L          for each axis, V and lambda with V' M- V = I and V' M+ V = diag(lambda),
                           M+ / M- the own blocks of slots 2*axis+1 / 2*axis: a face node's
                           diagonal block k_A M+ + k_B M- then inverts as
                           V diag(1 / (k_A lambda + k_B)) V'.

Run: python gen_template.py > template_gen.cuh (build() does it when the file is absent).
"""
import math
import sys

import numpy as np

SECTION = (0.336, 0.336)
G_OVER_E = 0.4
FACES = [(-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)]


def unit(v):
    return v * (1.0 / math.sqrt(float(v @ v)))


def template(s=1.0, e=1.0, g=G_OVER_E):
    centre = np.full(3, 0.5 * s)
    xs = [centre + 0.5 * s * np.array(f, float) for f in FACES]
    K = np.zeros((36, 36))
    for a in range(6):
        for b in range(a + 1, 6):
            xa, xb = xs[a], xs[b]
            u, v = xa - centre, xb - centre
            cls = int(round(1.0 + float(u @ v) / (math.sqrt(u @ u) * math.sqrt(v @ v))))
            area = SECTION[cls] * s * s
            n = unit(xb - xa)
            e1 = unit(np.cross(n, [1.0, 0.0, 0.0] if abs(n[0]) < 0.9 else [0.0, 1.0, 0.0]))
            e2 = np.cross(n, e1)
            r = math.sqrt(area / (2.0 * math.pi))
            middle = 0.5 * (xa + xb)
            d = math.sqrt(float((xb - xa) @ (xb - xa)))
            ab = area / 4.0
            S = (e * np.outer(n, n) + g * (np.eye(3) - np.outer(n, n))) * (ab / d)
            for o in (e1 * r, -e1 * r, e2 * r, -e2 * r):
                p = middle + o

                def T(xv):
                    rr = p - xv
                    return np.array([[1, 0, 0, 0, rr[2], -rr[1]],
                                     [0, 1, 0, -rr[2], 0, rr[0]],
                                     [0, 0, 1, rr[1], -rr[0], 0]], float)
                Ta, Tb = T(xa), T(xb)
                K[6 * a:6 * a + 6, 6 * a:6 * a + 6] += Ta.T @ S @ Ta
                K[6 * b:6 * b + 6, 6 * b:6 * b + 6] += Tb.T @ S @ Tb
                K[6 * a:6 * a + 6, 6 * b:6 * b + 6] -= Ta.T @ S @ Tb
                K[6 * b:6 * b + 6, 6 * a:6 * a + 6] -= Tb.T @ S @ Ta
    return K


def clean(K):
    """Symmetrise and zero the entries that are rounding noise of exact zeros."""
    K = 0.5 * (K + K.T)
    K[np.abs(K) < 1e-13 * np.abs(K).max()] = 0.0
    return K


def jacobi_factors(K):
    """Per axis: V, lambda with V' M- V = I, V' M+ V = diag(lambda)."""
    out = []
    for ax in range(3):
        mp = K[6 * (2 * ax + 1):6 * (2 * ax + 2), 6 * (2 * ax + 1):6 * (2 * ax + 2)]
        mm = K[6 * (2 * ax):6 * (2 * ax + 1), 6 * (2 * ax):6 * (2 * ax + 1)]
        L = np.linalg.cholesky(mm)
        Li = np.linalg.inv(L)
        C = Li @ mp @ Li.T
        lam, Q = np.linalg.eigh(0.5 * (C + C.T))
        V = Li.T @ Q
        out.append((V, lam))
    return out


def lit(v):
    return repr(float(v))


def emit(K, fac):
    w = sys.stdout.write
    w("// Generated by gen_template.py: the stiffness of one full level-0 cell at spacing 1,\n")
    w("// E = 1, G = 0.4 (statics/src/lattice.rs:76-163, statics/src/model.rs:139-149).\n")
    w("// Do not edit by hand.\n#pragma once\n\n")
    w("namespace sc {\n\n")
    w(f"constexpr double TPL_G_OVER_E = {lit(G_OVER_E)};\n")
    w("static const double TPL_HOST[36][36] = {\n")
    for i in range(36):
        w("  {" + ", ".join(lit(K[i, j]) for j in range(36)) + "},\n")
    w("};\n\n")
    w("__constant__ double TPL_DEV[36][36] = {\n")
    for i in range(36):
        w("  {" + ", ".join(lit(K[i, j]) for j in range(36)) + "},\n")
    w("};\n\n")
    # Jacobi factors
    w("static const double JAC_V_HOST[3][6][6] = {\n")
    for V, _ in fac:
        w("  {" + ", ".join("{" + ", ".join(lit(V[i, j]) for j in range(6)) + "}" for i in range(6)) + "},\n")
    w("};\nstatic const double JAC_L_HOST[3][6] = {\n")
    for _, lam in fac:
        w("  {" + ", ".join(lit(x) for x in lam) + "},\n")
    w("};\n")
    w("__constant__ double JAC_V_DEV[3][6][6] = {\n")
    for V, _ in fac:
        w("  {" + ", ".join("{" + ", ".join(lit(V[i, j]) for j in range(6)) + "}" for i in range(6)) + "},\n")
    w("};\n__constant__ double JAC_L_DEV[3][6] = {\n")
    for _, lam in fac:
        w("  {" + ", ".join(lit(x) for x in lam) + "},\n")
    w("};\n\n")
    # stencil strips: y += sum_b T[slot][b] * xs[b], xs[b] the six node vectors of the cell
    for slot in range(6):
        w(f"// Row strip of face slot {slot}: acc[i] += sum_b sum_j TPL[6*{slot}+i][6*b+j] * x[b][j]\n")
        w("template <class T>\n")
        w(f"__device__ __forceinline__ void strip_{slot}(const T (&x)[6][6], T (&acc)[6]) {{\n")
        for i in range(6):
            terms = []
            for b in range(6):
                for j in range(6):
                    v = K[6 * slot + i, 6 * b + j]
                    if v != 0.0:
                        terms.append((b, j, v))
            w(f"  {{ T s = acc[{i}];\n")
            for b, j, v in terms:
                w(f"    s = fma(T({lit(v)}), x[{b}][{j}], s);\n")
            w(f"    acc[{i}] = s; }}\n")
        w("}\n\n")
    # per-(slot, face) 6x6 blocks: acc += TPL block (slot, face) * x_face
    w("template <int S, int F>\nstruct Blk;\n")
    for slot in range(6):
        for f in range(6):
            w(f"template <>\nstruct Blk<{slot}, {f}> {{\n  template <class T>\n")
            w("  __device__ __forceinline__ static void mac(const T (&x)[6], T (&acc)[6]) {\n")
            for i in range(6):
                terms = [(j, K[6 * slot + i, 6 * f + j]) for j in range(6) if K[6 * slot + i, 6 * f + j] != 0.0]
                for j, v in terms:
                    w(f"    acc[{i}] = fma(T({lit(v)}), x[{j}], acc[{i}]);\n")
            w("  }\n};\n")
    # the same blocks at level 0's spacing s = UNIT = 1/8 (statics/src/lattice.rs:16): the
    # cell matrix k s D T D with D = diag(1, 1, 1, s, s, s) per face, so a level-0 stencil
    # that reads the motions as they are needs no scaling (every factor is a power of two,
    # so each product, and each FMA's rounding, is the unscaled one's times that factor)
    s0 = 0.125
    d = [1.0, 1.0, 1.0, s0, s0, s0]
    w("// The blocks of k s D T D at level 0's spacing s = 1/8, D = diag(1, 1, 1, s, s, s).\n")
    w("template <int S, int F>\nstruct BlkS;\n")
    for slot in range(6):
        for f in range(6):
            w(f"template <>\nstruct BlkS<{slot}, {f}> {{\n  template <class T>\n")
            w("  __device__ __forceinline__ static void mac(const T (&x)[6], T (&acc)[6]) {\n")
            for i in range(6):
                terms = [(j, K[6 * slot + i, 6 * f + j]) for j in range(6) if K[6 * slot + i, 6 * f + j] != 0.0]
                for j, v in terms:
                    w(f"    acc[{i}] = fma(T({lit(v * s0 * d[i] * d[j])}), x[{j}], acc[{i}]);\n")
            w("  }\n};\n")
    w(f"constexpr double TPL_SPACING0 = {lit(s0)};\n")
    w("\n")
    nnz = int((K != 0).sum())
    w(f"constexpr int TPL_NNZ = {nnz};\n\n")
    w("}  // namespace sc\n")


if __name__ == "__main__":
    K = clean(template())
    emit(K, jacobi_factors(K))
