// Level 0 of voxel pieces on the device.
//
// Numbering follows the reference's `build` (statics/src/lattice.rs:124-163) exactly:
// free cells are visited in flat order ((x*ny)+y)*nz+z; each creates a node for each of
// its faces, in VOXEL_FACES order -x,+x,-y,+y,-z,+z (lattice/src/lib.rs:64), that no
// earlier cell created. A + face is always new (its other cell comes later); a - face
// is new unless the cell before it on that axis is free. A node is held when its other
// cell is held. Free (not held) nodes are the parts, in node order (bodies.rs:435-442).
// So node and part ids come from two exclusive scans, no hashing.
//
// The operator is matrix-free: a free cell's 36x36 stiffness is k * s * D Kt D
// (template_gen.cuh); a part on axis a is the + face (slot 2a+1) of its lesser cell A
// and the - face (slot 2a) of its greater cell B, so its row is
//   y = k_A * strip_{2a+1}(x of A's six faces) + k_B * strip_{2a}(x of B's six faces),
// gathered per part with no atomics. Roofline: HBM. Algorithmic bytes per apply:
// read x and write y (2 * 6 * w per part) plus the cell table (32 B per free cell).
#include <cub/cub.cuh>

#include "level0.cuh"
#include "level0_blocks.cuh"
#include "solver.cuh"
#include "template_gen.cuh"

namespace sc {

namespace {

__device__ __forceinline__ int find_piece(const int64_t* __restrict__ off, int np, int64_t i) {
    int lo = 0, hi = np;  // off[lo] <= i < off[hi]
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (off[mid] <= i)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

__global__ void k_iota(int64_t n, int32_t* __restrict__ v) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) v[i] = (int32_t)i;
}

constexpr int64_t STENCIL_TILE = 1024;

__global__ void k_tile_axis_keys(int64_t n, int64_t tile, const int8_t* __restrict__ axis, uint32_t* __restrict__ keys) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k < n) keys[k] = (uint32_t)(((k / tile) << 2) | (uint32_t)axis[k]);
}

// the stencil's per-slot record: part, lesser cell, greater cell, axis
__global__ void k_slots(int64_t n, const int32_t* __restrict__ perm, const int32_t* __restrict__ cella,
                        const int32_t* __restrict__ cellb, const int8_t* __restrict__ axis, int4* __restrict__ slots) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int32_t k = perm[i];
    slots[i] = make_int4(k, cella[k], cellb[k], (int)axis[k]);
}

struct Dims {
    int32_t nx, ny, nz, pad;
};

__device__ __forceinline__ bool is_free(const uint8_t* st, const Dims& d, int x, int y, int z) {
    if (x < 0 || y < 0 || z < 0 || x >= d.nx || y >= d.ny || z >= d.nz) return false;
    return st[((int64_t)x * d.ny + y) * d.nz + z] == SC_CELL_FREE;
}
__device__ __forceinline__ bool is_held(const uint8_t* st, const Dims& d, int x, int y, int z) {
    if (x < 0 || y < 0 || z < 0 || x >= d.nx || y >= d.ny || z >= d.nz) return false;
    return st[((int64_t)x * d.ny + y) * d.nz + z] == SC_CELL_HELD;
}

// New nodes of a free cell in slot order: slot 2a is new iff the cell before on axis a
// is not free; slot 2a+1 always. Returns a 6-bit mask.
__device__ __forceinline__ int new_mask(const uint8_t* st, const Dims& d, int x, int y, int z) {
    int m = 0;
    if (!is_free(st, d, x - 1, y, z)) m |= 1;
    m |= 2;
    if (!is_free(st, d, x, y - 1, z)) m |= 4;
    m |= 8;
    if (!is_free(st, d, x, y, z - 1)) m |= 16;
    m |= 32;
    return m;
}

__global__ void k_count_cells(int np, const int64_t* __restrict__ goff, const Dims* __restrict__ dims,
                              const uint8_t* __restrict__ st, int64_t ncell, int64_t* __restrict__ new_nodes,
                              int64_t* __restrict__ free_flag) {
    int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    int p = find_piece(goff, np, c);
    Dims d = dims[p];
    const uint8_t* s = st + goff[p];
    int64_t l = c - goff[p];
    int z = (int)(l % d.nz), y = (int)(l / d.nz % d.ny), x = (int)(l / ((int64_t)d.nz * d.ny));
    if (s[l] != SC_CELL_FREE) {
        new_nodes[c] = 0;
        free_flag[c] = 0;
        return;
    }
    new_nodes[c] = __popc(new_mask(s, d, x, y, z));
    free_flag[c] = 1;
}

// For every free cell: the node ids of its 6 faces, and for each node it creates: held
// flag, axis, lesser cell. Each node's lesser and greater free cell (cella / cellb) is
// written exactly once: by its creator, or, for a - face made by the cell before, by
// the greater cell itself.
__global__ void k_cell_nodes(int np, const int64_t* __restrict__ goff, const Dims* __restrict__ dims,
                             const uint8_t* __restrict__ st, int64_t ncell, const int64_t* __restrict__ node_base,
                             const int64_t* __restrict__ cell_index, int64_t* __restrict__ cell_node6,
                             int64_t* __restrict__ node_held, int8_t* __restrict__ node_axis,
                             int64_t* __restrict__ node_site, int32_t* __restrict__ node_cella,
                             int32_t* __restrict__ node_cellb) {
    int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    int p = find_piece(goff, np, c);
    Dims d = dims[p];
    const uint8_t* s = st + goff[p];
    int64_t l = c - goff[p];
    if (s[l] != SC_CELL_FREE) return;
    int z = (int)(l % d.nz), y = (int)(l / d.nz % d.ny), x = (int)(l / ((int64_t)d.nz * d.ny));
    int m = new_mask(s, d, x, y, z);
    int32_t ci = (int32_t)cell_index[c];
    int off = 0;
    for (int slot = 0; slot < 6; slot++) {
        int a = slot >> 1;
        int o[3] = {x, y, z};
        o[a] += (slot & 1) ? 1 : -1;
        int64_t node;
        if (m & (1 << slot)) {
            node = node_base[c] + off;
            off++;
            node_held[node] = is_held(s, d, o[0], o[1], o[2]) ? 1 : 0;
            node_axis[node] = (int8_t)a;
            int lesser[3] = {x, y, z};
            if (!(slot & 1)) lesser[a] -= 1;
            for (int k = 0; k < 3; k++) node_site[3 * node + k] = lesser[k];
            if (slot & 1) {
                node_cella[node] = ci;
                if (!is_free(s, d, o[0], o[1], o[2])) node_cellb[node] = -1;
            } else {
                node_cellb[node] = ci;
                node_cella[node] = -1;
            }
        } else {
            // the cell before on axis a is free and made this node as its + face
            int64_t lc = ((int64_t)o[0] * d.ny + o[1]) * d.nz + o[2];
            int mm = new_mask(s, d, o[0], o[1], o[2]);
            int before = __popc(mm & ((1 << (2 * a + 1)) - 1));
            node = node_base[goff[p] + lc] + before;
            node_cellb[node] = ci;
        }
        cell_node6[6 * (int64_t)ci + slot] = node;
    }
}

__global__ void k_node_parts(int64_t nnodes, const int64_t* __restrict__ held, const int64_t* __restrict__ held_before,
                             int32_t* __restrict__ node_part) {
    int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (v >= nnodes) return;
    node_part[v] = held[v] ? -1 : (int32_t)(v - held_before[v]);
}

__global__ void k_part_data(int64_t nnodes, int np, const int64_t* __restrict__ node_start,
                            const int32_t* __restrict__ node_part, const int8_t* __restrict__ node_axis,
                            const int64_t* __restrict__ node_site, const int32_t* __restrict__ node_cella,
                            const int32_t* __restrict__ node_cellb, const int64_t* __restrict__ part_start,
                            const double* __restrict__ pmass, int32_t* __restrict__ piece,
                            int32_t* __restrict__ part_node, int8_t* __restrict__ axis, int64_t* __restrict__ site,
                            double* __restrict__ centre, int32_t* __restrict__ cella, int32_t* __restrict__ cellb,
                            double* __restrict__ mass, double* __restrict__ loads) {
    int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (v >= nnodes) return;
    int32_t k = node_part[v];
    if (k < 0) return;
    int p = find_piece(node_start, np, v);
    piece[k] = p;
    part_node[k] = (int32_t)(v - node_start[p]);
    int a = node_axis[v];
    axis[k] = (int8_t)a;
    int64_t ls[3];
    for (int q = 0; q < 3; q++) ls[q] = site[3 * k + q] = node_site[3 * v + q];
    // x = (centre(lesser) + centre(greater)) * 0.5, centre(c) = (c + 0.5) * UNIT (lattice.rs:39-41, 137)
    for (int q = 0; q < 3; q++) {
        double ca = ((double)ls[q] + 0.5) * 0.125;
        double cb = ((double)(ls[q] + (q == a ? 1 : 0)) + 0.5) * 0.125;
        centre[3 * k + q] = __dmul_rn(__dadd_rn(ca, cb), 0.5);
    }
    int32_t A = node_cella[v], B = node_cellb[v];
    cella[k] = A;
    cellb[k] = B < 0 ? -1 : B;
    // node.m += rho s^3 / 6 per free cell it touches (lattice.rs:130, 143)
    double mcell = pmass[4 * p];
    double m = 0.0;
    if (A >= 0) m += mcell;
    if (B >= 0) m += mcell;
    mass[k] = m;
    loads[6 * k + 0] = m * pmass[4 * p + 1];
    loads[6 * k + 1] = m * pmass[4 * p + 2];
    loads[6 * k + 2] = m * pmass[4 * p + 3];
    loads[6 * k + 3] = 0.0;
    loads[6 * k + 4] = 0.0;
    loads[6 * k + 5] = 0.0;
}

// per free cell: its six faces' parts (-1 held), k, and bit a set when its +a
// neighbour is free
__global__ void k_cell_table(int np, const int64_t* __restrict__ goff, const Dims* __restrict__ dims,
                             const uint8_t* __restrict__ st, int64_t ncells, const int64_t* __restrict__ cell_node6,
                             const int32_t* __restrict__ node_part, const int64_t* __restrict__ cell_flat,
                             const float* __restrict__ gk, int4* __restrict__ cell) {
    int64_t ci = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (ci >= ncells) return;
    int32_t q[6];
    for (int s = 0; s < 6; s++) q[s] = node_part[cell_node6[6 * ci + s]];
    int64_t c = cell_flat[ci];
    float k = gk[c];
    int p = find_piece(goff, np, c);
    Dims d = dims[p];
    int64_t l = c - goff[p];
    int z = (int)(l % d.nz), y = (int)(l / d.nz % d.ny), x = (int)(l / ((int64_t)d.nz * d.ny));
    const uint8_t* sp = st + goff[p];
    int nbr = (is_free(sp, d, x + 1, y, z) ? 1 : 0) | (is_free(sp, d, x, y + 1, z) ? 2 : 0) |
              (is_free(sp, d, x, y, z + 1) ? 4 : 0);
    cell[2 * ci] = make_int4(q[0], q[1], q[2], q[3]);
    cell[2 * ci + 1] = make_int4(q[4], q[5], __float_as_int(k), nbr);
}

__global__ void k_gridmap(int64_t ncell, const int64_t* __restrict__ free_flag, const int64_t* __restrict__ cell_index,
                          int32_t* __restrict__ gridmap) {
    int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c < ncell) gridmap[c] = free_flag[c] ? (int32_t)cell_index[c] : -1;
}

__global__ void k_node_loads(int64_t n, const int32_t* __restrict__ part_node, const double* __restrict__ node_loads,
                             double* __restrict__ loads) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    for (int q = 0; q < 6; q++) loads[6 * k + q] = node_loads[6 * (int64_t)part_node[k] + q];
}

__global__ void k_cell_flat(int64_t ncell, const int64_t* __restrict__ free_flag, const int64_t* __restrict__ cell_index,
                            int64_t* __restrict__ cell_flat) {
    int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    if (free_flag[c]) cell_flat[cell_index[c]] = c;
}

// ---- assembled level-0 blocks (for the Galerkin setup) ----------------------------
__device__ __forceinline__ double tpl_scaled(int i, int j, double s) {
    double d = TPL_DEV[i][j] * s;
    if ((i % 6) >= 3) d *= s;
    if ((j % 6) >= 3) d *= s;
    return d;
}

__global__ void k_row_count(int64_t n, const int8_t* __restrict__ axis, const int32_t* __restrict__ cella,
                            const int32_t* __restrict__ cellb, const int4* __restrict__ cell, int64_t* __restrict__ cnt) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    int c = 1;
    for (int side = 0; side < 2; side++) {
        int32_t C = side ? cellb[k] : cella[k];
        if (C < 0) continue;
        int4 a = cell[2 * C], b2 = cell[2 * C + 1];
        int32_t q[6] = {a.x, a.y, a.z, a.w, b2.x, b2.y};
        for (int s = 0; s < 6; s++)
            if (q[s] >= 0 && q[s] != (int32_t)k) c++;
    }
    cnt[k] = c;
}

// The level-0 pattern of row k (its own block and every part sharing a cell with it,
// columns sorted) with each block's origin in the cell template (level0_blocks.cuh).
__global__ void k_row_fill(int64_t n, const int32_t* __restrict__ cella,
                           const int32_t* __restrict__ cellb, const int4* __restrict__ cell,
                           const int64_t* __restrict__ rowptr, int32_t* __restrict__ col, uint8_t* __restrict__ desc) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    // gather (column, cell side, slot of column)
    int32_t cols[11];
    int8_t sideof[11], slotof[11];
    int m = 0;
    cols[m] = (int32_t)k;
    sideof[m] = -1;
    slotof[m] = -1;
    m++;
    for (int side = 0; side < 2; side++) {
        int32_t C = side ? cellb[k] : cella[k];
        if (C < 0) continue;
        int4 a = cell[2 * C], b2 = cell[2 * C + 1];
        int32_t q[6] = {a.x, a.y, a.z, a.w, b2.x, b2.y};
        for (int sl = 0; sl < 6; sl++)
            if (q[sl] >= 0 && q[sl] != (int32_t)k) {
                cols[m] = q[sl];
                sideof[m] = (int8_t)side;
                slotof[m] = (int8_t)sl;
                m++;
            }
    }
    // insertion sort by column
    for (int i = 1; i < m; i++) {
        int32_t c0 = cols[i];
        int8_t s0 = sideof[i], l0 = slotof[i];
        int j = i - 1;
        while (j >= 0 && cols[j] > c0) {
            cols[j + 1] = cols[j];
            sideof[j + 1] = sideof[j];
            slotof[j + 1] = slotof[j];
            j--;
        }
        cols[j + 1] = c0;
        sideof[j + 1] = s0;
        slotof[j + 1] = l0;
    }
    int64_t base = rowptr[k];
    for (int e = 0; e < m; e++) {
        col[base + e] = cols[e];
        desc[base + e] = sideof[e] < 0 ? K0_DIAG : (uint8_t)((sideof[e] << 3) | slotof[e]);
    }
}

// the cell template at spacing s (entry (i, j) times s, and s again for each rotation index)
__global__ void k_scaled_template(double s, double* __restrict__ out) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < 36 * 36) out[e] = tpl_scaled(e / 36, e % 36, s);
}

// ---- the matrix-free stencil ---------------------------------------------------------
// acc += k_C * (row strip SLOT of cell C's template) * (x of C's six faces)
template <int SLOT, class T>
__device__ __forceinline__ void cell_term(int4 a, int4 b, int32_t self, T kc, const T* __restrict__ x, T s,
                                          T (&acc)[6]) {
    int32_t q[6] = {a.x, a.y, a.z, a.w, b.x, b.y};
    T xs[6][6];
#pragma unroll
    for (int f = 0; f < 6; f++) load6<T>(x, q[f] >= 0 ? q[f] : self, xs[f]);
#pragma unroll
    for (int f = 0; f < 6; f++) {
        T m = q[f] >= 0 ? T(1) : T(0);
        T ms = m * s;
        xs[f][0] *= m;
        xs[f][1] *= m;
        xs[f][2] *= m;
        xs[f][3] *= ms;
        xs[f][4] *= ms;
        xs[f][5] *= ms;
    }
    T t[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
    face_macs<SLOT, 0, T>(xs, t);
#pragma unroll
    for (int i = 0; i < 6; i++) acc[i] = fma(kc, t[i], acc[i]);
}

template <int AX, class T, int MODE>
__device__ __forceinline__ void stencil_row(int32_t k, int32_t A, int32_t B, int4 a0, int4 a1, int4 b0, int4 b1,
                                            const T* __restrict__ x, const T* __restrict__ r, T* __restrict__ y,
                                            T* __restrict__ y2, T s, T w) {
    T kA = A >= 0 ? (T)__int_as_float(a1.z) : T(0);
    T kB = B >= 0 ? (T)__int_as_float(b1.z) : T(0);
    T acc[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
    if (A >= 0) cell_term<2 * AX + 1, T>(a0, a1, k, kA, x, s, acc);
    if (B >= 0) cell_term<2 * AX, T>(b0, b1, k, kB, x, s, acc);
    T kx[6] = {acc[0] * s, acc[1] * s, acc[2] * s, acc[3] * s * s, acc[4] * s * s, acc[5] * s * s};
    T o[6];
    if constexpr (MODE == ST_Y) {
        store6<T>(y, k, kx);
    } else if constexpr (MODE == ST_RES) {
        load6<T>(r, k, o);
#pragma unroll
        for (int j = 0; j < 6; j++) o[j] -= kx[j];
        store6<T>(y, k, o);
    } else if constexpr (MODE == ST_RES_JAC) {
        load6<T>(r, k, o);
#pragma unroll
        for (int j = 0; j < 6; j++) o[j] -= kx[j];
        store6<T>(y, k, o);
        T d[6];
        dinv<AX, T>(kA, kB, s, o, d);
        store6<T>(y2, k, d);
    } else if constexpr (MODE == ST_RES_W) {
        load6<T>(r, k, o);
#pragma unroll
        for (int j = 0; j < 6; j++) o[j] = fma(-w, kx[j], o[j]);
        store6<T>(y, k, o);
    } else if constexpr (MODE == ST_PROLONG) {
        T d[6], xv[6], acc2[6];
        dinv<AX, T>(kA, kB, s, kx, d);
        load6<T>(x, k, xv);
        load6<T>(y, k, acc2);
#pragma unroll
        for (int j = 0; j < 6; j++) o[j] = acc2[j] + fma(-w, d[j], xv[j]);
        store6<T>(y, k, o);
    } else {
        T rv[6], d[6], xv[6];
        load6<T>(r, k, rv);
#pragma unroll
        for (int j = 0; j < 6; j++) rv[j] -= kx[j];
        dinv<AX, T>(kA, kB, s, rv, d);
        load6<T>(x, k, xv);
#pragma unroll
        for (int j = 0; j < 6; j++) o[j] = fma(w, d[j], xv[j]);
        store6<T>(y, k, o);
    }
}

// Level 0 applied matrix-free over the parts grouped by axis (perm). The register cap
// (four blocks of 256 in FP32, three in FP64) trades a few FP64 spills for occupancy:
// the gathers are latency-bound, and the capped kernel measured 2-4 % faster.
template <class T, int MODE>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 3) k_stencil(int64_t n_perm, const int4* __restrict__ slots,
                                                 const int4* __restrict__ cell,
                                                 const T* __restrict__ x, const T* __restrict__ r, T* __restrict__ y,
                                                 T* __restrict__ y2, T s, const int32_t* __restrict__ piece,
                                                 const double* __restrict__ step, const int32_t* __restrict__ skip_row,
                                                 const int32_t* __restrict__ done) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n_perm) return;
    int4 sl = __ldg(slots + i);  // part, lesser cell, greater cell, axis
    int32_t k = sl.x, A = sl.y, B = sl.z;
    if (skip_row && skip_row[k]) return;
    int p = (done || step) ? piece[k] : 0;
    if (done && done[p]) return;
    T w = step ? (T)step[p] : T(0);
    int32_t Ac = A >= 0 ? A : 0, Bc = B >= 0 ? B : 0;
    int4 a0 = __ldg(cell + 2 * Ac), a1 = __ldg(cell + 2 * Ac + 1);
    int4 b0 = __ldg(cell + 2 * Bc), b1 = __ldg(cell + 2 * Bc + 1);
    if (sl.w == 0)
        stencil_row<0, T, MODE>(k, A, B, a0, a1, b0, b1, x, r, y, y2, s, w);
    else if (sl.w == 1)
        stencil_row<1, T, MODE>(k, A, B, a0, a1, b0, b1, x, r, y, y2, s, w);
    else
        stencil_row<2, T, MODE>(k, A, B, a0, a1, b0, b1, x, r, y, y2, s, w);
}

// ---- the plane-pencil stencil ------------------------------------------------------
// A block owns a PTY x PTZ tile of (y, z) cells of one piece and walks PSX planes of x.
// Each free cell's six faces are gathered once per plane and all six of its template
// strips computed (Y_s = k * strip_s * x~, s = slot): its +y / +z strips go to shared
// memory for the neighbour threads, its +x strip stays in a register for the next plane.
// Every part is written once, by its greater cell (the - face; a + face only where the
// greater cell is not free): Kx of the part on the face between cells L and G along axis
// a is Y_L[2a+1] + Y_G[2a]. A warp of the block recomputes the +y strips of the row
// before the tile and one the +z strips of the column before it; the first plane's +x
// strips come from recomputing the plane before the segment. So a cell is gathered
// about 1 + 1/PSX + 1/PTY + 1/PTZ times instead of six (once per part that touches it).
constexpr int PTY = 8, PTZ = 32, PSX = 16;
constexpr int PENCIL_THREADS = (PTY + 2) * 32;  // 8 tile warps, a +y halo warp, a +z halo warp

struct PencilTile {
    int32_t piece, x0, y0, z0;
};
struct PieceGeo {
    int32_t nx, ny, nz, pad;
    int64_t goff;  // first flat cell of the piece
};

// Y[slot] += k * strip(slot) * x~ for all six slots
template <int SLOT, class T>
__device__ __forceinline__ void slot_out(const T (&xs)[6][6], T kc, T s, T (&y)[6]) {
    T t[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
    face_macs<SLOT, 0, T>(xs, t);
    y[0] = kc * t[0] * s;
    y[1] = kc * t[1] * s;
    y[2] = kc * t[2] * s;
    y[3] = kc * t[3] * s * s;
    y[4] = kc * t[4] * s * s;
    y[5] = kc * t[5] * s * s;
}

template <class T>
__device__ __forceinline__ void gather_cell(int4 a, int4 b, const T* __restrict__ x, T s, T (&xs)[6][6]) {
    int32_t q[6] = {a.x, a.y, a.z, a.w, b.x, b.y};
#pragma unroll
    for (int f = 0; f < 6; f++) load6<T>(x, q[f] >= 0 ? q[f] : 0, xs[f]);
#pragma unroll
    for (int f = 0; f < 6; f++) {
        T m = q[f] >= 0 ? T(1) : T(0);
        T ms = m * s;
        xs[f][0] *= m;
        xs[f][1] *= m;
        xs[f][2] *= m;
        xs[f][3] *= ms;
        xs[f][4] *= ms;
        xs[f][5] *= ms;
    }
}

// the part's epilogue given its Kx, its axis and the stiffness of its lesser / greater cell
template <int AX, class T, int MODE>
__device__ __forceinline__ void pencil_finish(int32_t q, const T (&kx)[6], T kA, T kB, T s, T w,
                                              const T* __restrict__ x, const T* __restrict__ r, T* __restrict__ y,
                                              T* __restrict__ y2) {
    T o[6];
    if constexpr (MODE == ST_Y) {
        store6<T>(y, q, kx);
    } else if constexpr (MODE == ST_RES) {
        load6<T>(r, q, o);
#pragma unroll
        for (int j = 0; j < 6; j++) o[j] -= kx[j];
        store6<T>(y, q, o);
    } else if constexpr (MODE == ST_RES_JAC) {
        load6<T>(r, q, o);
#pragma unroll
        for (int j = 0; j < 6; j++) o[j] -= kx[j];
        store6<T>(y, q, o);
        T d[6];
        dinv<AX, T>(kA, kB, s, o, d);
        store6<T>(y2, q, d);
    } else if constexpr (MODE == ST_RES_W) {
        load6<T>(r, q, o);
#pragma unroll
        for (int j = 0; j < 6; j++) o[j] = fma(-w, kx[j], o[j]);
        store6<T>(y, q, o);
    } else if constexpr (MODE == ST_PROLONG) {
        T d[6], xv[6], acc2[6];
        dinv<AX, T>(kA, kB, s, kx, d);
        load6<T>(x, q, xv);
        load6<T>(y, q, acc2);
#pragma unroll
        for (int j = 0; j < 6; j++) o[j] = acc2[j] + fma(-w, d[j], xv[j]);
        store6<T>(y, q, o);
    } else {
        T rv[6], d[6], xv[6];
        load6<T>(r, q, rv);
#pragma unroll
        for (int j = 0; j < 6; j++) rv[j] -= kx[j];
        dinv<AX, T>(kA, kB, s, rv, d);
        load6<T>(x, q, xv);
#pragma unroll
        for (int j = 0; j < 6; j++) o[j] = fma(w, d[j], xv[j]);
        store6<T>(y, q, o);
    }
}

template <class T, int MODE>
__global__ void __launch_bounds__(PENCIL_THREADS, 2) k_stencil_pencil(
    const PencilTile* __restrict__ tiles, const PieceGeo* __restrict__ geo, const int32_t* __restrict__ gridmap,
    const int4* __restrict__ cell, const T* __restrict__ x, const T* __restrict__ r, T* __restrict__ y,
    T* __restrict__ y2, T s, const double* __restrict__ step, const int32_t* __restrict__ skip_row,
    const int32_t* __restrict__ done) {
    // shared (dynamic): +y and +z strips and k of every tile position and the halo row /
    // column, indexed [ty + 1][tz + 1]; the tile cells' three - strips
    extern __shared__ __align__(16) unsigned char pencil_smem[];
    T(*py)[PTZ + 1][6] = reinterpret_cast<T(*)[PTZ + 1][6]>(pencil_smem);
    T(*pz)[PTZ + 1][6] = py + (PTY + 1);
    T(*kk)[PTZ + 1] = reinterpret_cast<T(*)[PTZ + 1]>(pz + (PTY + 1));
    T(*ym)[PTZ][3][6] = reinterpret_cast<T(*)[PTZ][3][6]>(kk + (PTY + 1));
    const PencilTile tl = tiles[blockIdx.x];
    if (done && done[tl.piece]) return;
    const PieceGeo g = geo[tl.piece];
    const T w = step ? (T)step[tl.piece] : T(0);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // this thread's (ty, tz) in [-1, PTY) x [-1, PTZ); role 0 tile, 1 +y halo, 2 +z halo
    int ty, tz, role;
    if (warp < PTY) {
        ty = warp;
        tz = lane;
        role = 0;
    } else if (warp == PTY) {
        ty = -1;
        tz = lane;
        role = 1;
    } else {
        ty = lane < PTY ? lane : PTY;  // lanes past the column idle
        tz = -1;
        role = 2;
    }
    const int yy = tl.y0 + ty, zz = tl.z0 + tz;
    const bool inside = ty < PTY && yy >= 0 && yy < g.ny && zz >= 0 && zz < g.nz;
    T prevx[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
    T prevk = T(0);
    const int xend = min(tl.x0 + PSX, g.nx);
    for (int xx = tl.x0 - 1; xx < xend; xx++) {
        // the cell here, if free
        int32_t C = -1;
        if (inside && xx >= 0) C = gridmap[g.goff + ((int64_t)xx * g.ny + yy) * g.nz + zz];
        int4 a = make_int4(-1, -1, -1, -1), b = make_int4(-1, -1, 0, 0);
        T kc = T(0);
        if (C >= 0) {
            a = __ldg(cell + 2 * C);
            b = __ldg(cell + 2 * C + 1);
            kc = (T)__int_as_float(b.z);
        }
        T y1[6];
        if (C >= 0) {
            T xs[6][6];
            gather_cell<T>(a, b, x, s, xs);
            if (role == 0 && xx >= tl.x0) {
                T t[6];
                slot_out<0, T>(xs, kc, s, t);
#pragma unroll
                for (int j = 0; j < 6; j++) ym[ty][tz][0][j] = t[j];
                slot_out<2, T>(xs, kc, s, t);
#pragma unroll
                for (int j = 0; j < 6; j++) ym[ty][tz][1][j] = t[j];
                slot_out<4, T>(xs, kc, s, t);
#pragma unroll
                for (int j = 0; j < 6; j++) ym[ty][tz][2][j] = t[j];
            }
            if (role == 0) slot_out<1, T>(xs, kc, s, y1);
            if (xx >= tl.x0 && role != 2) {
                T t3[6];
                slot_out<3, T>(xs, kc, s, t3);
#pragma unroll
                for (int j = 0; j < 6; j++) py[ty + 1][tz + 1][j] = t3[j];
            }
            if (xx >= tl.x0 && role != 1) {
                T t5[6];
                slot_out<5, T>(xs, kc, s, t5);
#pragma unroll
                for (int j = 0; j < 6; j++) pz[ty + 1][tz + 1][j] = t5[j];
            }
        } else if (xx >= tl.x0 && ty < PTY) {
#pragma unroll
            for (int j = 0; j < 6; j++) {
                if (role != 2) py[ty + 1][tz + 1][j] = T(0);
                if (role != 1) pz[ty + 1][tz + 1][j] = T(0);
            }
        }
        if (xx >= tl.x0 && ty < PTY) kk[ty + 1][tz + 1] = kc;
        __syncthreads();
        if (xx >= tl.x0 && role == 0 && C >= 0) {
            int32_t q[6] = {a.x, a.y, a.z, a.w, b.x, b.y};
            int nbr = b.w;  // bit a: the +a neighbour is free
            // - faces: Kx = Y_L[2a+1] + Y_C[2a]
            if (q[0] >= 0 && !(skip_row && skip_row[q[0]])) {
                T kx[6];
#pragma unroll
                for (int j = 0; j < 6; j++) kx[j] = prevx[j] + ym[ty][tz][0][j];
                pencil_finish<0, T, MODE>(q[0], kx, prevk, kc, s, w, x, r, y, y2);
            }
            if (q[2] >= 0 && !(skip_row && skip_row[q[2]])) {
                T kx[6];
#pragma unroll
                for (int j = 0; j < 6; j++) kx[j] = py[ty][tz + 1][j] + ym[ty][tz][1][j];
                pencil_finish<1, T, MODE>(q[2], kx, kk[ty][tz + 1], kc, s, w, x, r, y, y2);
            }
            if (q[4] >= 0 && !(skip_row && skip_row[q[4]])) {
                T kx[6];
#pragma unroll
                for (int j = 0; j < 6; j++) kx[j] = pz[ty + 1][tz][j] + ym[ty][tz][2][j];
                pencil_finish<2, T, MODE>(q[4], kx, kk[ty + 1][tz], kc, s, w, x, r, y, y2);
            }
            // + faces whose greater cell is not free: Kx = Y_C[2a+1]
            if (!(nbr & 1) && q[1] >= 0 && !(skip_row && skip_row[q[1]]))
                pencil_finish<0, T, MODE>(q[1], y1, kc, T(0), s, w, x, r, y, y2);
            if (!(nbr & 2) && q[3] >= 0 && !(skip_row && skip_row[q[3]])) {
                T t[6];
#pragma unroll
                for (int j = 0; j < 6; j++) t[j] = py[ty + 1][tz + 1][j];
                pencil_finish<1, T, MODE>(q[3], t, kc, T(0), s, w, x, r, y, y2);
            }
            if (!(nbr & 4) && q[5] >= 0 && !(skip_row && skip_row[q[5]])) {
                T t[6];
#pragma unroll
                for (int j = 0; j < 6; j++) t[j] = pz[ty + 1][tz + 1][j];
                pencil_finish<2, T, MODE>(q[5], t, kc, T(0), s, w, x, r, y, y2);
            }
        }
        if (role == 0) {
#pragma unroll
            for (int j = 0; j < 6; j++) prevx[j] = C >= 0 ? y1[j] : T(0);
            prevk = kc;
        }
        __syncthreads();
    }
}

// ---- the two-pass (cell, then part) stencil --------------------------------------
// Pass 1 gives each free cell's six face rows of k_c s D Kt D x (36 values, slot by
// slot) to a per-cell buffer: a cell gathers its six faces once, where the per-part
// stencil gathers each face about six times (once per part of the two cells), and
// consecutive cells write consecutive records. Pass 2 walks the parts in slot order and
// adds the two records' rows of its faces, Kx = Y_lesser[2a+1] + Y_greater[2a], before
// the part's epilogue. It moves the 36 values a cell twice more than the per-part
// stencil's algorithmic bytes but reads them coalesced.
template <class T>
__global__ void __launch_bounds__(256) k_cell_rows(int64_t ncells, const int4* __restrict__ cell,
                                                   const T* __restrict__ x, T s, T* __restrict__ ycell,
                                                   const int32_t* __restrict__ cell_piece,
                                                   const int32_t* __restrict__ done) {
    int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    if (done && done[cell_piece[c]]) return;
    const int4 a = __ldg(cell + 2 * c), b = __ldg(cell + 2 * c + 1);
    const T kc = (T)__int_as_float(b.z);
    T xs[6][6];
    gather_cell<T>(a, b, x, s, xs);
    T* out = ycell + 36 * c;
    T y6[6];
    slot_out<0, T>(xs, kc, s, y6);
    store6<T>(out, 0, y6);
    slot_out<1, T>(xs, kc, s, y6);
    store6<T>(out, 1, y6);
    slot_out<2, T>(xs, kc, s, y6);
    store6<T>(out, 2, y6);
    slot_out<3, T>(xs, kc, s, y6);
    store6<T>(out, 3, y6);
    slot_out<4, T>(xs, kc, s, y6);
    store6<T>(out, 4, y6);
    slot_out<5, T>(xs, kc, s, y6);
    store6<T>(out, 5, y6);
}

template <class T, int MODE>
__global__ void __launch_bounds__(256) k_part_rows(int64_t n_perm, const int4* __restrict__ slots,
                                                   const int4* __restrict__ cell, const T* __restrict__ ycell,
                                                   const T* __restrict__ x, const T* __restrict__ r, T* __restrict__ y,
                                                   T* __restrict__ y2, T s, const int32_t* __restrict__ piece,
                                                   const double* __restrict__ step,
                                                   const int32_t* __restrict__ skip_row,
                                                   const int32_t* __restrict__ done) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n_perm) return;
    const int4 sl = __ldg(slots + i);  // part, lesser cell, greater cell, axis
    const int32_t k = sl.x, A = sl.y, B = sl.z;
    if (skip_row && skip_row[k]) return;
    const int p = (done || step) ? piece[k] : 0;
    if (done && done[p]) return;
    const T w = step ? (T)step[p] : T(0);
    T kx[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
    if (A >= 0) {
        T v[6];
        load6<T>(ycell + 36 * (int64_t)A, 2 * sl.w + 1, v);
#pragma unroll
        for (int j = 0; j < 6; j++) kx[j] += v[j];
    }
    if (B >= 0) {
        T v[6];
        load6<T>(ycell + 36 * (int64_t)B, 2 * sl.w, v);
#pragma unroll
        for (int j = 0; j < 6; j++) kx[j] += v[j];
    }
    T kA = T(0), kB = T(0);
    if constexpr (MODE == ST_RES_JAC || MODE == ST_PROLONG || MODE == ST_SMOOTH) {
        if (A >= 0) kA = (T)__int_as_float(__ldg(&cell[2 * A + 1].z));
        if (B >= 0) kB = (T)__int_as_float(__ldg(&cell[2 * B + 1].z));
    }
    if (sl.w == 0)
        pencil_finish<0, T, MODE>(k, kx, kA, kB, s, w, x, r, y, y2);
    else if (sl.w == 1)
        pencil_finish<1, T, MODE>(k, kx, kA, kB, s, w, x, r, y, y2);
    else
        pencil_finish<2, T, MODE>(k, kx, kA, kB, s, w, x, r, y, y2);
}

// a free cell's piece (from its flat index and the pieces' first flat cells)
__global__ void k_cell_piece(int64_t ncells, const int64_t* __restrict__ cell_flat, const int64_t* __restrict__ goff,
                             int np, int32_t* __restrict__ cell_piece) {
    int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    int64_t f = cell_flat[c];
    int lo = 0, hi = np;  // last piece whose first cell is <= f
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (goff[mid] <= f) lo = mid;
        else hi = mid;
    }
    cell_piece[c] = lo;
}

// x = w D^-1 r with D^-1 matrix-free (pre-smoothing, bodies.rs:386)
template <class T>
__global__ void __launch_bounds__(256) k_jacobi_mf(int64_t n, const int4* __restrict__ slots,
                                                   const int4* __restrict__ cell, const T* __restrict__ r,
                                                   T* __restrict__ x, T s, const int32_t* __restrict__ piece,
                                                   const double* __restrict__ step, const int32_t* __restrict__ skip_row,
                                                   const int32_t* __restrict__ done) {
    // over the stencil's slots (parts grouped by axis inside tiles), so a warp runs one
    // axis' factors
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 sl = __ldg(slots + i);  // part, lesser cell, greater cell, axis
    const int32_t k = sl.x, A = sl.y, B = sl.z;
    if (skip_row && skip_row[k]) return;
    int p = piece[k];
    if (done && done[p]) return;
    T w = step ? (T)step[p] : T(1);
    T kA = A >= 0 ? (T)__int_as_float(__ldg(&cell[2 * A + 1].z)) : T(0);
    T kB = B >= 0 ? (T)__int_as_float(__ldg(&cell[2 * B + 1].z)) : T(0);
    T rv[6], d[6];
    load6<T>(r, k, rv);
    int ax = sl.w;
    if (ax == 0)
        dinv<0, T>(kA, kB, s, rv, d);
    else if (ax == 1)
        dinv<1, T>(kA, kB, s, rv, d);
    else
        dinv<2, T>(kA, kB, s, rv, d);
#pragma unroll
    for (int j = 0; j < 6; j++) d[j] *= w;
    store6<T>(x, k, d);
}

// rc[c] = sum over the parts k of body c of R_k' u_k, R_k' u = (u_t, u_w + r_k x u_t):
// the rigid part P0' of the restriction (bodies.rs:239, 388-390)
template <class T>
__global__ void __launch_bounds__(256) k_p0t(int64_t nc, const int64_t* __restrict__ moff,
                                             const int32_t* __restrict__ mem, const T* __restrict__ rvec,
                                             const T* __restrict__ u, T* __restrict__ rc,
                                             const int32_t* __restrict__ piece_c, const int32_t* __restrict__ done) {
    int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= nc) return;
    if (done && done[piece_c[c]]) return;
    T o[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
    for (int64_t t = moff[c]; t < moff[c + 1]; t++) {
        int32_t k = mem[t];
        T uv[6];
        load6<T>(u, k, uv);
        T r0 = rvec[3 * (int64_t)k], r1 = rvec[3 * (int64_t)k + 1], r2 = rvec[3 * (int64_t)k + 2];
        o[0] += uv[0];
        o[1] += uv[1];
        o[2] += uv[2];
        o[3] += uv[3] + (r1 * uv[2] - r2 * uv[1]);
        o[4] += uv[4] + (r2 * uv[0] - r0 * uv[2]);
        o[5] += uv[5] + (r0 * uv[1] - r1 * uv[0]);
    }
    store6<T>(rc, c, o);
}

// e_k = R_k z_{up[k]} = (z_t + z_w x r_k, z_w): the rigid part P0 of the prolongation
template <class T>
__global__ void __launch_bounds__(256) k_p0(int64_t n, const int32_t* __restrict__ up, const T* __restrict__ rvec,
                                            const T* __restrict__ z, T* __restrict__ e, const int32_t* __restrict__ piece,
                                            const int32_t* __restrict__ skip_row, const int32_t* __restrict__ done) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (skip_row && skip_row[k]) return;
    if (done && done[piece[k]]) return;
    int32_t c = up[k];
    T zv[6];
    load6<T>(z, c, zv);
    T r0 = rvec[3 * k], r1 = rvec[3 * k + 1], r2 = rvec[3 * k + 2];
    T o[6] = {zv[0] + (zv[4] * r2 - zv[5] * r1), zv[1] + (zv[5] * r0 - zv[3] * r2), zv[2] + (zv[3] * r1 - zv[4] * r0),
              zv[3], zv[4], zv[5]};
    store6<T>(e, k, o);
}

// Strain energy of each free cell's 60 bonds at motions x: U = 1/2 x_c' K_c x_c with
// K_c = k s D Kt D over its six faces (held faces contribute zero motion).
__global__ void k_cell_energy(int64_t ncells, const int4* __restrict__ cell, const double* __restrict__ x, double s,
                              double* __restrict__ energy) {
    int64_t C = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (C >= ncells) return;
    int4 a = cell[2 * C], b = cell[2 * C + 1];
    int32_t q[6] = {a.x, a.y, a.z, a.w, b.x, b.y};
    double kc = (double)__int_as_float(b.z);
    double xs[36];
    for (int f = 0; f < 6; f++)
        for (int j = 0; j < 6; j++) {
            double v = q[f] >= 0 ? x[6 * (int64_t)q[f] + j] : 0.0;
            xs[6 * f + j] = j >= 3 ? v * s : v;
        }
    double e = 0.0;
    for (int i = 0; i < 36; i++) {
        double t = 0.0;
        for (int j = 0; j < 36; j++) t = fma(TPL_DEV[i][j], xs[j], t);
        e = fma(xs[i], t, e);
    }
    energy[C] = 0.5 * kc * s * e;
}

}  // namespace

// Algorithmic bytes of one stencil launch: x read and y written once (and r read for
// the residual form), 6 values a part; the cells' stiffness (4 B each) and occupancy
// (one bit per grid cell).
template <class T>
static double stencil_bytes(const Batch& b, int vec_passes) {
    const Grid0& g = b.grid;
    double G = g.grid_off.empty() ? 0.0 : (double)g.grid_off.back();
    return (double)sizeof(T) * 6.0 * (double)b.levels[0].n * vec_passes + 4.0 * (double)g.ncells + G / 8.0;
}

template <class T, int MODE>
static void launch_stencil(Context& ctx, const Batch& b, const T* x, const T* r, T* y, T* y2, const double* step,
                           const int32_t* skip_row, const int32_t* done, int passes) {
    const Grid0& g = b.grid;
    const Level& L = b.levels[0];
    int64_t n = g.axis_off[3];
    ProfScope ps(ctx, sizeof(T) == 8 ? SC_FAM_STENCIL64 : SC_FAM_STENCIL32, stencil_bytes<T>(b, passes));
    if (g.bricks.active) {  // the iterations' layout (brick.cu)
        brick_stencil<T, MODE>(ctx, b, x, r, y, y2, step, skip_row, done);
        return;
    }
    if (g.pencil) {
        // one piece per block: the step and done flag are the block's piece's
        size_t smem = sizeof(T) * ((size_t)2 * (PTY + 1) * (PTZ + 1) * 6 + (size_t)(PTY + 1) * (PTZ + 1) +
                                   (size_t)PTY * PTZ * 18);
        static const bool attr_set = [smem] {  // once per instantiation (thread-safe)
            SC_CK(cudaFuncSetAttribute(k_stencil_pencil<T, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
            return true;
        }();
        (void)attr_set;
        k_stencil_pencil<T, MODE><<<(unsigned)g.ntiles, PENCIL_THREADS, smem, ctx.stream>>>(
            reinterpret_cast<const PencilTile*>(g.tiles.get()), reinterpret_cast<const PieceGeo*>(g.geo.get()),
            g.gridmap.get(), g.cell.get(), x, r, y, y2, (T)g.s, step, skip_row, done);
        SC_LAUNCH_CK();
        return;
    }
    if (g.two_pass) {
        T* yc = reinterpret_cast<T*>(sizeof(T) == 8 ? (void*)g.ycell64.get() : (void*)g.ycell32.get());
        k_cell_rows<T><<<grid_for(g.ncells, 256), 256, 0, ctx.stream>>>(g.ncells, g.cell.get(), x, (T)g.s, yc,
                                                                        g.cell_piece.get(), done);
        SC_LAUNCH_CK();
        k_part_rows<T, MODE><<<grid_for(n, 256), 256, 0, ctx.stream>>>(n, g.slots.get(), g.cell.get(), yc, x, r, y,
                                                                       y2, (T)g.s, L.piece.get(), step, skip_row,
                                                                       done);
        SC_LAUNCH_CK();
        return;
    }
    k_stencil<T, MODE><<<grid_for(n, 256), 256, 0, ctx.stream>>>(n, g.slots.get(), g.cell.get(), x, r, y, y2, (T)g.s,
                                                                 L.piece.get(), step, skip_row, done);
    SC_LAUNCH_CK();
}

template <class T>
void stencil_apply(Context& ctx, const Batch& b, const T* x, T* y, const int32_t* skip_row, const int32_t* done) {
    launch_stencil<T, ST_Y>(ctx, b, x, nullptr, y, nullptr, nullptr, skip_row, done, 2);
}
template void stencil_apply<double>(Context&, const Batch&, const double*, double*, const int32_t*, const int32_t*);
template void stencil_apply<float>(Context&, const Batch&, const float*, float*, const int32_t*, const int32_t*);

template <class T>
void stencil_residual(Context& ctx, const Batch& b, const T* x, const T* r, T* y, const int32_t* skip_row,
                      const int32_t* done) {
    launch_stencil<T, ST_RES>(ctx, b, x, r, y, nullptr, nullptr, skip_row, done, 3);
}
template void stencil_residual<double>(Context&, const Batch&, const double*, const double*, double*, const int32_t*,
                                       const int32_t*);
template void stencil_residual<float>(Context&, const Batch&, const float*, const float*, float*, const int32_t*,
                                      const int32_t*);

// Level 0's half of a V-cycle on the way up (bodies.rs:386-390), matrix-free:
//   x = w D^-1 r;  left = r - K x;  t = D^-1 left;  u = left - w K t;  rc = P0' u
// (P' = P0' (I - w K D^-1), P = (I - w D^-1 K) P0, bodies.rs:238-247).
template <class T>
void level0_down(Context& ctx, const Batch& b, const T* r, T* x, T* left, T* t, T* u, T* rc, const int32_t* done) {
    const Grid0& g = b.grid;
    const Level& L = b.levels[0];
    const Level& C = b.levels[1];
    const int32_t* skip = L.top_of_part.get();
    double vb = (double)sizeof(T) * 6.0 * (double)L.n;
    {
        ProfScope ps(ctx, sizeof(T) == 8 ? SC_FAM_SMOOTH64 : SC_FAM_SMOOTH32, 2 * vb + 8.0 * L.n);
        if (g.bricks.active) {
            brick_jacobi<T>(ctx, b, r, x, L.step.get(), skip, done);
        } else {
            k_jacobi_mf<T><<<grid_for(L.n, 256), 256, 0, ctx.stream>>>(L.n, g.slots.get(), g.cell.get(), r, x,
                                                                       (T)g.s, L.piece.get(), L.step.get(), skip,
                                                                       done);
            SC_LAUNCH_CK();
        }
    }
    for (int sweep = 1; sweep < b.sweeps; sweep++) {  // further pre-smoothing sweeps
        level0_smooth<T>(ctx, b, r, x, t, done);
        SC_CK(cudaMemcpyAsync(x, t, 6 * L.n * sizeof(T), cudaMemcpyDeviceToDevice, ctx.stream));
    }
    launch_stencil<T, ST_RES_JAC>(ctx, b, x, r, left, t, nullptr, skip, done, 4);
    launch_stencil<T, ST_RES_W>(ctx, b, t, left, u, nullptr, L.step.get(), skip, done, 3);
    {
        ProfScope ps(ctx, sizeof(T) == 8 ? SC_FAM_TRANSFER64 : SC_FAM_TRANSFER32, vb + (double)sizeof(T) * 3 * L.n +
                     (double)sizeof(T) * 6 * C.n);
        const T* rv = sizeof(T) == 8 ? (const T*)L.mf_r.get() : (const T*)L.mf_r32.get();
        k_p0t<T><<<grid_for(C.n, 256), 256, 0, ctx.stream>>>(C.n, L.mem_off.get(), L.mem.get(), rv, u, rc,
                                                             C.piece.get(), done);
        SC_LAUNCH_CK();
    }
}

// ... and on the way down (bodies.rs:392-401), matrix-free:
//   e = P0 zc;  x += e - w D^-1 K e;  z = x + w D^-1 (r - K x)
template <class T>
void level0_up(Context& ctx, const Batch& b, const T* r, T* x, T* e, const T* zc, T* z, const int32_t* done) {
    const Level& L = b.levels[0];
    const int32_t* skip = L.top_of_part.get();
    double vb = (double)sizeof(T) * 6.0 * (double)L.n;
    {
        ProfScope ps(ctx, sizeof(T) == 8 ? SC_FAM_TRANSFER64 : SC_FAM_TRANSFER32, vb + (double)sizeof(T) * 3 * L.n +
                     4.0 * L.n + (double)sizeof(T) * 6 * b.levels[1].n);
        const T* rv = sizeof(T) == 8 ? (const T*)L.mf_r.get() : (const T*)L.mf_r32.get();
        k_p0<T><<<grid_for(L.n, 256), 256, 0, ctx.stream>>>(L.n, L.up.get(), rv, zc, e, L.piece.get(), skip, done);
        SC_LAUNCH_CK();
    }
    launch_stencil<T, ST_PROLONG>(ctx, b, e, nullptr, x, nullptr, L.step.get(), skip, done, 4);
    for (int sweep = 1; sweep < b.sweeps; sweep++) {  // further post-smoothing sweeps
        launch_stencil<T, ST_SMOOTH>(ctx, b, x, r, e, nullptr, L.step.get(), skip, done, 3);
        SC_CK(cudaMemcpyAsync(x, e, 6 * L.n * sizeof(T), cudaMemcpyDeviceToDevice, ctx.stream));
    }
    launch_stencil<T, ST_SMOOTH>(ctx, b, x, r, z, nullptr, L.step.get(), skip, done, 3);
}

// z = x + w D^-1 (r - K x): one more block-Jacobi sweep
template <class T>
void level0_smooth(Context& ctx, const Batch& b, const T* r, const T* x, T* z, const int32_t* done) {
    const Level& L = b.levels[0];
    launch_stencil<T, ST_SMOOTH>(ctx, b, x, r, z, nullptr, L.step.get(), L.top_of_part.get(), done, 3);
}
template void level0_smooth<double>(Context&, const Batch&, const double*, const double*, double*, const int32_t*);
template void level0_smooth<float>(Context&, const Batch&, const float*, const float*, float*, const int32_t*);

template void level0_down<double>(Context&, const Batch&, const double*, double*, double*, double*, double*, double*,
                                  const int32_t*);
template void level0_down<float>(Context&, const Batch&, const float*, float*, float*, float*, float*, float*,
                                 const int32_t*);
template void level0_up<double>(Context&, const Batch&, const double*, double*, double*, const double*, double*,
                                const int32_t*);
template void level0_up<float>(Context&, const Batch&, const float*, float*, float*, const float*, float*,
                               const int32_t*);

void grid_cell_energy(Context& ctx, const Batch& b, const double* x, double* energy_cells) {
    const Grid0& g = b.grid;
    k_cell_energy<<<grid_for(g.ncells, 128), 128, 0, ctx.stream>>>(g.ncells, g.cell.get(), x, g.s, energy_cells);
    SC_LAUNCH_CK();
}

// Builds level 0 of a batch of voxel pieces. The grids' state/k are uploaded (or
// copied device to device) into one concatenated array.
void grid_level0(Context& ctx, Batch& b, const std::vector<sc_grid>& grids, bool keep_blocks, int32_t tile) {
    const int64_t TILE = tile >= 32 ? tile : STENCIL_TILE;
    PhaseTimer pt(ctx);
    cudaStream_t st = ctx.stream;
    MemStats* ms = &ctx.mem;
    int np = (int)grids.size();
    b.npieces = np;
    std::vector<int64_t> goff(np + 1, 0);
    std::vector<Dims> dims(np);
    for (int p = 0; p < np; p++) {
        const sc_grid& g = grids[p];
        dims[p] = Dims{g.nx, g.ny, g.nz, 0};
        goff[p + 1] = goff[p] + (int64_t)g.nx * g.ny * g.nz;
    }
    int64_t ncell = goff[np];
    DBuf<int64_t> goff_d;
    goff_d.alloc(np + 1, st, ms);
    goff_d.upload(goff.data(), np + 1);
    DBuf<Dims> dims_d;
    dims_d.alloc(np, st, ms);
    dims_d.upload(dims.data(), np);
    DBuf<uint8_t> gst;
    gst.alloc(ncell, st, ms);
    DBuf<float> gk;
    gk.alloc(ncell, st, ms);
    for (int p = 0; p < np; p++) {
        const sc_grid& g = grids[p];
        size_t cnt = (size_t)(goff[p + 1] - goff[p]);
        auto kind = g.on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        SC_CK(cudaMemcpyAsync(gst.get() + goff[p], g.state, cnt, kind, st));
        SC_CK(cudaMemcpyAsync(gk.get() + goff[p], g.k, cnt * sizeof(float), kind, st));
    }
    // counts and scans
    DBuf<int64_t> newn, freef, node_base, cell_index;
    newn.alloc(ncell + 1, st, ms);
    freef.alloc(ncell + 1, st, ms);
    node_base.alloc(ncell + 1, st, ms);
    cell_index.alloc(ncell + 1, st, ms);
    SC_CK(cudaMemsetAsync(newn.get() + ncell, 0, sizeof(int64_t), st));
    SC_CK(cudaMemsetAsync(freef.get() + ncell, 0, sizeof(int64_t), st));
    k_count_cells<<<grid_for(ncell, 256), 256, 0, st>>>(np, goff_d.get(), dims_d.get(), gst.get(), ncell, newn.get(),
                                                        freef.get());
    SC_LAUNCH_CK();
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, newn.get(), node_base.get(), ncell + 1, st);
    cub::DeviceScan::ExclusiveSum(ctx.cub_scratch(tb), tb, newn.get(), node_base.get(), ncell + 1, st);
    cub::DeviceScan::ExclusiveSum(nullptr, tb, freef.get(), cell_index.get(), ncell + 1, st);
    cub::DeviceScan::ExclusiveSum(ctx.cub_scratch(tb), tb, freef.get(), cell_index.get(), ncell + 1, st);
    int64_t nnodes = 0, nfree = 0;
    SC_CK(cudaMemcpyAsync(&nnodes, node_base.get() + ncell, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    SC_CK(cudaMemcpyAsync(&nfree, cell_index.get() + ncell, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    // per-piece node starts
    std::vector<int64_t> node_start(np + 1, 0);
    for (int p = 0; p < np; p++)
        SC_CK(cudaMemcpyAsync(&node_start[p], node_base.get() + goff[p], sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    SC_CK(cudaStreamSynchronize(st));
    node_start[np] = nnodes;
    require(nnodes < (int64_t)INT32_MAX && nfree < (int64_t)INT32_MAX, SC_BAD_INPUT, "piece too large");
    b.node_count.resize(np);
    for (int p = 0; p < np; p++) b.node_count[p] = node_start[p + 1] - node_start[p];
    b.node_start.alloc(np + 1, st, ms);
    b.node_start.upload(node_start.data(), np + 1);

    DBuf<int64_t> cell_node6;
    cell_node6.alloc(6 * std::max<int64_t>(nfree, 1), st, ms);
    DBuf<int64_t> node_held;
    node_held.alloc(nnodes + 1, st, ms);
    DBuf<int8_t> node_axis;
    node_axis.alloc(nnodes + 1, st, ms);
    DBuf<int64_t> node_site;
    node_site.alloc(3 * (nnodes + 1), st, ms);
    DBuf<int32_t> node_cella, node_cellb;
    node_cella.alloc(nnodes + 1, st, ms);
    node_cellb.alloc(nnodes + 1, st, ms);
    k_cell_nodes<<<grid_for(ncell, 256), 256, 0, st>>>(np, goff_d.get(), dims_d.get(), gst.get(), ncell, node_base.get(),
                                                       cell_index.get(), cell_node6.get(), node_held.get(),
                                                       node_axis.get(), node_site.get(), node_cella.get(),
                                                       node_cellb.get());
    SC_LAUNCH_CK();
    // parts: free nodes in node order
    DBuf<int64_t> held_before;
    held_before.alloc(nnodes + 1, st, ms);
    SC_CK(cudaMemsetAsync(node_held.get() + nnodes, 0, sizeof(int64_t), st));
    cub::DeviceScan::ExclusiveSum(nullptr, tb, node_held.get(), held_before.get(), nnodes + 1, st);
    cub::DeviceScan::ExclusiveSum(ctx.cub_scratch(tb), tb, node_held.get(), held_before.get(), nnodes + 1, st);
    DBuf<int32_t> node_part;
    node_part.alloc(nnodes + 1, st, ms);
    k_node_parts<<<grid_for(nnodes, 256), 256, 0, st>>>(nnodes, node_held.get(), held_before.get(), node_part.get());
    SC_LAUNCH_CK();
    std::vector<int64_t> hb(np + 1);
    for (int p = 0; p <= np; p++)
        SC_CK(cudaMemcpyAsync(&hb[p], held_before.get() + node_start[p], sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    SC_CK(cudaStreamSynchronize(st));
    Level& L = b.levels.emplace_back();
    L.pstart.resize(np + 1);
    for (int p = 0; p <= np; p++) L.pstart[p] = node_start[p] - hb[p];
    int64_t n = L.pstart[np];
    L.n = n;
    require(n > 0, SC_BAD_INPUT, "no free node in the batch");
    L.pstart_d.alloc(np + 1, st, ms);
    L.pstart_d.upload(L.pstart.data(), np + 1);
    L.piece.alloc(n, st, ms);
    L.centre.alloc(3 * n, st, ms);
    L.site.alloc(3 * n, st, ms);
    b.part_node.alloc(n, st, ms);
    b.mass.alloc(n, st, ms);
    b.loads.alloc(6 * n, st, ms);
    Grid0& g = b.grid;
    g.s = 0.125;
    g.ncells = nfree;
    g.cella.alloc(n, st, ms);
    g.cellb.alloc(n, st, ms);
    g.axis.alloc(n, st, ms);
    // per piece: a cell's share of weight on each face (lattice.rs:130) and gravity
    std::vector<double> pm(4 * (size_t)np);
    for (int p = 0; p < np; p++) {
        pm[4 * p] = grids[p].rho * g.s * g.s * g.s / 6.0;
        for (int q = 0; q < 3; q++) pm[4 * p + 1 + q] = grids[p].gravity[q];
    }
    DBuf<double> pm_d;
    pm_d.alloc(pm.size(), st, ms);
    pm_d.upload(pm.data(), pm.size());
    k_part_data<<<grid_for(nnodes, 256), 256, 0, st>>>(
        nnodes, np, b.node_start.get(), node_part.get(), node_axis.get(), node_site.get(), node_cella.get(),
        node_cellb.get(), L.pstart_d.get(), pm_d.get(), L.piece.get(),
        b.part_node.get(), g.axis.get(), L.site.get(), L.centre.get(), g.cella.get(), g.cellb.get(), b.mass.get(),
        b.loads.get());
    SC_LAUNCH_CK();
    // caller loads instead of mass * gravity (node order) where given
    for (int p = 0; p < np; p++) {
        if (!grids[p].loads) continue;
        DBuf<double> nl;
        nl.alloc(6 * std::max<int64_t>(b.node_count[p], 1), st, ms);
        SC_CK(cudaMemcpyAsync(nl.get(), grids[p].loads, 6 * b.node_count[p] * sizeof(double),
                              grids[p].on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
        int64_t k0 = L.pstart[p], cnt = L.pstart[p + 1] - k0;
        if (cnt > 0) {
            k_node_loads<<<grid_for(cnt, 256), 256, 0, st>>>(cnt, b.part_node.get() + k0, nl.get(),
                                                             b.loads.get() + 6 * k0);
            SC_LAUNCH_CK();
        }
    }
    // cell table
    g.cell_flat.alloc(std::max<int64_t>(nfree, 1), st, ms);
    k_cell_flat<<<grid_for(ncell, 256), 256, 0, st>>>(ncell, freef.get(), cell_index.get(), g.cell_flat.get());
    SC_LAUNCH_CK();
    g.cell.alloc(2 * std::max<int64_t>(nfree, 1), st, ms);
    k_cell_table<<<grid_for(nfree, 256), 256, 0, st>>>(np, goff_d.get(), dims_d.get(), gst.get(), nfree,
                                                        cell_node6.get(), node_part.get(), g.cell_flat.get(), gk.get(),
                                                        g.cell.get());
    SC_LAUNCH_CK();
    // the pencil stencil's grid map and tiles
    g.gridmap.alloc(ncell, st, ms);
    k_gridmap<<<grid_for(ncell, 256), 256, 0, st>>>(ncell, freef.get(), cell_index.get(), g.gridmap.get());
    {
        std::vector<PencilTile> tiles;
        std::vector<PieceGeo> geo(np);
        for (int p = 0; p < np; p++) {
            const Dims& d = dims[p];
            geo[p] = PieceGeo{d.nx, d.ny, d.nz, 0, goff[p]};
            for (int x0 = 0; x0 < d.nx; x0 += PSX)
                for (int y0 = 0; y0 < d.ny; y0 += PTY)
                    for (int z0 = 0; z0 < d.nz; z0 += PTZ) tiles.push_back(PencilTile{p, x0, y0, z0});
        }
        g.ntiles = (int64_t)tiles.size();
        g.tiles.alloc(tiles.size() * sizeof(PencilTile), st, ms);
        SC_CK(cudaMemcpyAsync(g.tiles.get(), tiles.data(), tiles.size() * sizeof(PencilTile), cudaMemcpyHostToDevice, st));
        g.geo.alloc(geo.size() * sizeof(PieceGeo), st, ms);
        SC_CK(cudaMemcpyAsync(g.geo.get(), geo.data(), geo.size() * sizeof(PieceGeo), cudaMemcpyHostToDevice, st));
        SC_CK(cudaStreamSynchronize(st));  // the host vectors go out of scope
    }
    g.pencil = tile == 1;
    g.two_pass = tile == 2;
    g.use_bricks = tile == 0;
    g.dims_h.resize(3 * (size_t)np);
    for (int p = 0; p < np; p++) {
        g.dims_h[3 * p] = dims[p].nx;
        g.dims_h[3 * p + 1] = dims[p].ny;
        g.dims_h[3 * p + 2] = dims[p].nz;
    }
    if (g.two_pass) {
        g.cell_piece.alloc(std::max<int64_t>(nfree, 1), st, ms);
        if (nfree > 0) {
            k_cell_piece<<<grid_for(nfree, 256), 256, 0, st>>>(nfree, g.cell_flat.get(), goff_d.get(), np,
                                                              g.cell_piece.get());
            SC_LAUNCH_CK();
        }
        g.ycell64.alloc(36 * std::max<int64_t>(nfree, 1), st, ms);
        g.ycell32.alloc(36 * std::max<int64_t>(nfree, 1), st, ms);
    }
    SC_LAUNCH_CK();
    // parts in order, grouped by axis only within tiles of STENCIL_TILE parts: the
    // stencil sweeps the piece once in part order (x neighbours stay in L2) while a
    // warp mostly runs one axis' code
    {
        DBuf<int32_t> ids, ids_out;
        ids.alloc(n, st, ms);
        ids_out.alloc(n, st, ms);
        DBuf<uint32_t> keys, keys_out;
        keys.alloc(n, st, ms);
        keys_out.alloc(n, st, ms);
        k_iota<<<grid_for(n, 256), 256, 0, st>>>(n, ids.get());
        SC_LAUNCH_CK();
        k_tile_axis_keys<<<grid_for(n, 256), 256, 0, st>>>(n, TILE, g.axis.get(), keys.get());
        SC_LAUNCH_CK();
        int end_bit = 2;
        while (end_bit < 32 && ((uint64_t)1 << (end_bit - 2)) * (uint64_t)TILE <= (uint64_t)n) end_bit++;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.get(), keys_out.get(), ids.get(), ids_out.get(), n, 0,
                                        end_bit, st);
        cub::DeviceRadixSort::SortPairs(ctx.cub_scratch(tb), tb, keys.get(), keys_out.get(), ids.get(),
                                        ids_out.get(), n, 0, end_bit, st);
        g.perm = std::move(ids_out);
        g.axis_off[0] = 0;
        g.axis_off[1] = g.axis_off[2] = g.axis_off[3] = n;
        g.slots.alloc(n, st, ms);
        k_slots<<<grid_for(n, 256), 256, 0, st>>>(n, g.perm.get(), g.cella.get(), g.cellb.get(), g.axis.get(),
                                                   g.slots.get());
        SC_LAUNCH_CK();
    }
    // assembled blocks for the setup (the solve itself applies level 0 matrix-free)
    if (keep_blocks) {
        L.rowptr.alloc(n + 1, st, ms);
        {
            DBuf<int64_t> cnt;
            cnt.alloc(n + 1, st, ms);
            SC_CK(cudaMemsetAsync(cnt.get() + n, 0, sizeof(int64_t), st));
            k_row_count<<<grid_for(n, 256), 256, 0, st>>>(n, g.axis.get(), g.cella.get(), g.cellb.get(), g.cell.get(),
                                                          cnt.get());
            SC_LAUNCH_CK();
            cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.get(), L.rowptr.get(), n + 1, st);
            cub::DeviceScan::ExclusiveSum(ctx.cub_scratch(tb), tb, cnt.get(), L.rowptr.get(), n + 1, st);
        }
        SC_CK(cudaMemcpyAsync(&L.nnzb, L.rowptr.get() + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        SC_CK(cudaStreamSynchronize(st));
        L.col.alloc(L.nnzb, st, ms);
        L.desc.alloc(L.nnzb, st, ms);
        k_row_fill<<<grid_for(n, 128), 128, 0, st>>>(n, g.cella.get(), g.cellb.get(), g.cell.get(),
                                                     L.rowptr.get(), L.col.get(), L.desc.get());
        SC_LAUNCH_CK();
        g.tpl_s.alloc(36 * 36, st, ms);
        k_scaled_template<<<grid_for(36 * 36, 256), 256, 0, st>>>(g.s, g.tpl_s.get());
        SC_LAUNCH_CK();
    }
    L.matrix_free = true;
    g.grid_off = std::move(goff);
    SC_CK(cudaStreamSynchronize(st));
    pt.mark("level 0 (grid)");
}

}  // namespace sc
