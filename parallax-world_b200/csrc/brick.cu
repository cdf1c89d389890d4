// Level 0 of voxel pieces in brick order: the layout the conjugate gradients and the
// V-cycle's level-0 half run in, and its stencil.
//
// Why: in the reference's part order (first touch, statics/src/lattice.rs:124-163) a
// part's two cells reach faces far apart in memory (a -x face was made ny*nz cells
// earlier), and a per-part gather reads each face's six values about eleven times
// through L1, with two cell records and a slot record besides. Here the grid is cut into
// bricks of BX x BY x BZ cells; every face belongs to the brick of its greater cell (its
// - side), and a brick at the + end of the piece also owns the faces on the piece's +
// boundary (a plane of extra slots). A brick's parts are stored contiguously, in slot
// order (x faces, then y faces, then z faces; each z fastest), bricks of a piece in grid
// order (z fastest), pieces in order, so every piece keeps its range of part indices and
// the chunked dot products and axpys are unchanged.
//
// The stencil gives each brick one thread block. The block copies into a dense box in
// shared memory the x of every face its parts' two cells touch, with asynchronous copies
// (cp.async, global to shared memory without registers, all issued, then awaited once):
// its own parts, a contiguous run read in order and placed by each part's 16-bit code
// (axis and brick-local position), and its halo, a list of (box entry, part) pairs
// resolved once per solve from the twelve neighbour bricks' slot masks (bricks_build).
// The k of its cells and of the one-cell layers on its -x, -y and -z sides come the same
// way. Then each thread takes a part (in storage order, so its epilogue's loads and
// stores are contiguous) and adds the strips of its lesser and greater cell's rows of
// the level-0 cell matrix k s D T D (the template with the spacing folded into its
// constants, BlkS, so the box holds the motions as they are).
//
// The reference's order stays the order of everything else: the hierarchy is built in
// it (so the bit-exact parity holds), the caller's loads come in and the motions go out
// in it. bricks_enter permutes the loads and the level-0 arrays the transfers read
// (bodies' member lists, each part's body and offset from its centroid, the dense tops
// of pieces solved at level 0) into brick order before the iterations; bricks_leave
// puts them back and returns the solution in part order.
#include <cub/cub.cuh>

#include "level0.cuh"
#include "solver.cuh"

namespace sc {

namespace {

constexpr int BX = 4, BY = 8, BZ = 8;
constexpr int BCELLS = BX * BY * BZ;
// owned slots per axis a: (BX + [a==0]) x (BY + [a==1]) x (BZ + [a==2])
constexpr int NS0 = (BX + 1) * BY * BZ, NS1 = BX * (BY + 1) * BZ, NS2 = BX * BY * (BZ + 1);
constexpr int NSLOT = NS0 + NS1 + NS2;
constexpr int MW = (NSLOT + 31) / 32;  // mask words a brick
// the box of axis-a faces a brick reads: positions lo-1 .. hi along a, lo-1 .. hi-1
// along the other two
constexpr int XB0 = (BX + 2) * (BY + 1) * (BZ + 1), XB1 = (BX + 1) * (BY + 2) * (BZ + 1),
              XB2 = (BX + 1) * (BY + 1) * (BZ + 2);
constexpr int NBOX = XB0 + XB1 + XB2;
constexpr int KB = (BX + 1) * (BY + 1) * (BZ + 1);  // cells lo-1 .. hi-1
constexpr int NNB = 13;                             // the brick and the twelve it reads from
constexpr int HKX = BY * BZ, HKY = BX * BZ, HKZ = BX * BY, HK = HKX + HKY + HKZ;  // halo cells
constexpr int BRICK_THREADS = 256;
static_assert(NSLOT < 4096, "slot indices take 12 bits (halo_table)");
static_assert(BRICK_THREADS == BCELLS, "the k box is filled a cell a thread");

// The bricks a brick reads from, as offsets in brick units: itself, its six face
// neighbours, and the six edge neighbours one step back along one axis and one step
// forward along another (the -x halo cells' +y faces, ...).
#define SC_NB_OFFSETS                                                                                            \
    {{0, 0, 0}, {-1, 0, 0}, {0, -1, 0}, {0, 0, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {-1, 1, 0}, {-1, 0, 1},     \
     {1, -1, 0}, {0, -1, 1}, {1, 0, -1}, {0, 1, -1}}
constexpr int8_t NB_OFF_H[NNB][3] = SC_NB_OFFSETS;
__constant__ int8_t NB_OFF[NNB][3] = SC_NB_OFFSETS;
#undef SC_NB_OFFSETS
// the table index of offset (ox, oy, oz), by (ox+1)*9 + (oy+1)*3 + (oz+1); -1 where unused
struct CodeTable {
    int8_t v[27];
};
constexpr CodeTable make_code_table() {
    CodeTable t{};
    for (int i = 0; i < 27; i++) t.v[i] = -1;
    for (int q = 0; q < NNB; q++)
        t.v[(NB_OFF_H[q][0] + 1) * 9 + (NB_OFF_H[q][1] + 1) * 3 + (NB_OFF_H[q][2] + 1)] = (int8_t)q;
    return t;
}
static_assert(make_code_table().v[13] == 0 && make_code_table().v[4] == 1 && make_code_table().v[22] == 4,
              "offset codes");

__host__ __device__ constexpr int slot_ext(int a, int d) {
    return (d == 0 ? BX : d == 1 ? BY : BZ) + (a == d ? 1 : 0);
}
__host__ __device__ constexpr int slot_off(int a) { return a == 0 ? 0 : a == 1 ? NS0 : NS0 + NS1; }
__host__ __device__ inline int slot_of(int a, int l0, int l1, int l2) {
    return slot_off(a) + (l0 * slot_ext(a, 1) + l1) * slot_ext(a, 2) + l2;
}
__host__ __device__ constexpr int box_ext(int a, int d) { return slot_ext(a, d) + 1; }
__host__ __device__ constexpr int box_off(int a) { return a == 0 ? 0 : a == 1 ? XB0 : XB0 + XB1; }
// box entry of axis-a face position c (brick-local cell coordinates, -1 .. B)
__device__ __forceinline__ int box_index(int a, int c0, int c1, int c2) {
    return box_off(a) + ((c0 + 1) * box_ext(a, 1) + (c1 + 1)) * box_ext(a, 2) + (c2 + 1);
}
__device__ __forceinline__ int kbox_index(int c0, int c1, int c2) {
    return ((c0 + 1) * (BY + 1) + (c1 + 1)) * (BZ + 1) + (c2 + 1);
}

struct BrickGeo {
    int32_t nx, ny, nz, pad;
    int32_t nbx, nby, nbz, pad2;
    int64_t goff;  // first flat cell of the piece in the batch's grids
    int64_t pos0;  // first brick position of the piece
};

struct BrickView {
    const int32_t* start;  // n_bricks + 1: each brick's first part
    const uint32_t* mask;  // MW words a brick: bit = slot holds a part
    const uint16_t* pre;   // MW a brick: parts in the words before
    const int4* info;      // piece, brick coordinates
    const int32_t* nbr;    // NNB a brick: the bricks of NB_OFF_H, -1 where none
    const float* kd;       // BCELLS a brick: each cell's k, 0 where not free
    const BrickGeo* geo;   // per piece
    const uint16_t* code;  // per part (brick order): its part_code
    const int32_t* hstart; // n_bricks + 1: each brick's halo list
    const uint16_t* hent;  // per halo item: the box entry it fills
    const int32_t* hsrc;   // per halo item: the part (brick order) it comes from
    const float* hk;       // per brick, HK values: the k of the cells of its -x, -y, -z layers
};

// A part's slot as the part phase reads it: axis (bits 12-13), brick-local face position
// l (l0 bits 8-10, l1 bits 4-7, l2 bits 0-3).
__host__ __device__ constexpr uint32_t part_code(int a, int l0, int l1, int l2) {
    return ((uint32_t)a << 12) | ((uint32_t)l0 << 8) | ((uint32_t)l1 << 4) | (uint32_t)l2;
}
static_assert(BX + 1 < 8 && BY + 1 < 16 && BZ + 1 < 16, "part_code fields");

// The entries of a brick's box that other bricks hold, the same for every brick (the
// brick's own parts go to the box straight from their run, by their part_code). Entry i
// is the face of axis a at brick-local position c, read by some part. x: bits 27-30 the
// brick (index into NB_OFF) holding it and bits 0-11 its slot there; bits 25-26 the
// axis a; bits 12-23 the entry i; bit 24 the entry lies on the + plane of axis a, where
// it belongs to the next brick along a -- or, for bricks at the piece's + end along a,
// to the plane of extra slots of the brick one step back from there (y: that brick,
// bits 27-30, and slot, bits 0-11; brick 0 is the brick itself, whose own parts are
// filled as those are).
std::vector<uint2> halo_table() {
    std::vector<uint2> t;
    constexpr CodeTable code = make_code_table();
    const int B[3] = {BX, BY, BZ};
    for (int i = 0; i < NBOX; i++) {
        const int a = i < XB0 ? 0 : i < XB0 + XB1 ? 1 : 2;
        const int rem = i - box_off(a);
        const int e2 = box_ext(a, 2), e1 = box_ext(a, 1);
        const int c[3] = {rem / (e2 * e1) - 1, rem / e2 % e1 - 1, rem % e2 - 1};
        if ((c[0] < 0) + (c[1] < 0) + (c[2] < 0) > 1) continue;  // read by no part
        int o[3], l[3], oa[3], la[3];
        for (int d = 0; d < 3; d++) {
            if (c[d] < 0) {
                o[d] = oa[d] = -1;
                l[d] = la[d] = B[d] - 1;
            } else if (c[d] >= B[d]) {  // only along a
                o[d] = 1;
                l[d] = 0;
                oa[d] = 0;
                la[d] = B[d];
            } else {
                o[d] = oa[d] = 0;
                l[d] = la[d] = c[d];
            }
        }
        const int q = code.v[(o[0] + 1) * 9 + (o[1] + 1) * 3 + (o[2] + 1)];
        const int qa = code.v[(oa[0] + 1) * 9 + (oa[1] + 1) * 3 + (oa[2] + 1)];
        if (q == 0) continue;  // an own slot
        const bool plane = c[a] >= B[a];
        t.push_back(make_uint2(((uint32_t)q << 27) | ((uint32_t)a << 25) | ((plane ? 1u : 0u) << 24) |
                                   ((uint32_t)i << 12) | (uint32_t)slot_of(a, l[0], l[1], l[2]),
                               ((uint32_t)qa << 27) | (uint32_t)slot_of(a, la[0], la[1], la[2])));
    }
    return t;
}

__device__ __forceinline__ int find_pos_piece(const BrickGeo* __restrict__ geo, int np, int64_t pos) {
    int lo = 0, hi = np;  // geo[lo].pos0 <= pos < geo[hi].pos0
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (geo[mid].pos0 <= pos)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// ---- building the layout ----------------------------------------------------------------
// a brick position for every free cell (a brick holds the k of its free cells even where
// none of its slots is a part: a free cell whose - faces are all held still has + faces)
__global__ void k_mark_cell_bricks(int64_t ncells, const int64_t* __restrict__ cell_flat, const BrickGeo* __restrict__ geo,
                                   int np, int32_t* __restrict__ flag) {
    int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    int64_t f = cell_flat[c];
    int lo = 0, hi = np;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (geo[mid].goff <= f)
            lo = mid;
        else
            hi = mid;
    }
    const BrickGeo g = geo[lo];
    int64_t l = f - g.goff;
    int z = (int)(l % g.nz), y = (int)(l / g.nz % g.ny), x = (int)(l / ((int64_t)g.nz * g.ny));
    flag[g.pos0 + ((int64_t)(x / BX) * g.nby + y / BY) * g.nbz + z / BZ] = 1;
}

// each part's brick position and slot: the key it is sorted by
__global__ void k_part_keys(int64_t n, const int32_t* __restrict__ piece, const int64_t* __restrict__ site,
                            const int8_t* __restrict__ axis, const BrickGeo* __restrict__ geo,
                            int32_t* __restrict__ flag, uint64_t* __restrict__ key, int32_t* __restrict__ ids) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    const BrickGeo g = geo[piece[k]];
    const int a = axis[k];
    int p[3] = {(int)site[3 * k], (int)site[3 * k + 1], (int)site[3 * k + 2]};
    p[a] += 1;  // the greater cell: the face is its - face
    const int nb[3] = {g.nbx, g.nby, g.nbz};
    const int B[3] = {BX, BY, BZ};
    int bb[3], l[3];
    for (int d = 0; d < 3; d++) {
        bb[d] = min(p[d] / B[d], nb[d] - 1);
        l[d] = p[d] - bb[d] * B[d];
    }
    int64_t pos = g.pos0 + ((int64_t)bb[0] * g.nby + bb[1]) * g.nbz + bb[2];
    flag[pos] = 1;
    key[k] = (uint64_t)pos * NSLOT + (uint64_t)slot_of(a, l[0], l[1], l[2]);
    ids[k] = (int32_t)k;
}

__global__ void k_brick_counts(int64_t n, const uint64_t* __restrict__ key, const int32_t* __restrict__ bid,
                               int32_t* __restrict__ cnt, uint32_t* __restrict__ mask) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t pos = (int64_t)(key[i] / NSLOT);
    int slot = (int)(key[i] % NSLOT);
    int32_t b = bid[pos];
    atomicAdd(cnt + b, 1);
    atomicOr(mask + (int64_t)b * MW + slot / 32, 1u << (slot & 31));
}

// per brick: piece, coordinates, neighbours, mask prefix counts
__global__ void k_brick_info(int64_t npos, const int32_t* __restrict__ flag, const int32_t* __restrict__ bid,
                             const BrickGeo* __restrict__ geo, int np, const uint32_t* __restrict__ mask,
                             int4* __restrict__ info, int32_t* __restrict__ nbr, uint16_t* __restrict__ pre) {
    int64_t pos = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (pos >= npos || !flag[pos]) return;
    const int32_t b = bid[pos];
    const int p = find_pos_piece(geo, np, pos);
    const BrickGeo g = geo[p];
    const int64_t l = pos - g.pos0;
    const int bz = (int)(l % g.nbz), by = (int)(l / g.nbz % g.nby), bx = (int)(l / ((int64_t)g.nbz * g.nby));
    info[b] = make_int4(p, bx, by, bz);
    for (int q = 0; q < NNB; q++) {
        const int x = bx + NB_OFF[q][0], y = by + NB_OFF[q][1], z = bz + NB_OFF[q][2];
        int32_t id = -1;
        if (x >= 0 && y >= 0 && z >= 0 && x < g.nbx && y < g.nby && z < g.nbz) {
            const int64_t o = g.pos0 + ((int64_t)x * g.nby + y) * g.nbz + z;
            if (flag[o]) id = bid[o];
        }
        nbr[(int64_t)b * NNB + q] = id;
    }
    int s = 0;
    for (int w = 0; w < MW; w++) {
        pre[(int64_t)b * MW + w] = (uint16_t)s;
        s += __popc(mask[(int64_t)b * MW + w]);
    }
}

// each brick's cells' k (0 where not free or outside the piece)
__global__ void k_brick_k(int64_t nb, const int4* __restrict__ info, const BrickGeo* __restrict__ geo,
                          const int32_t* __restrict__ gridmap, const int4* __restrict__ cell, float* __restrict__ kd) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nb * BCELLS) return;
    const int64_t b = i / BCELLS;
    const int c = (int)(i % BCELLS);
    const int4 in = info[b];
    const BrickGeo g = geo[in.x];
    const int x = in.y * BX + c / (BY * BZ), y = in.z * BY + c / BZ % BY, z = in.w * BZ + c % BZ;
    float k = 0.0f;
    if (x < g.nx && y < g.ny && z < g.nz) {
        const int32_t ci = gridmap[g.goff + ((int64_t)x * g.ny + y) * g.nz + z];
        if (ci >= 0) k = __int_as_float(cell[2 * (int64_t)ci + 1].z);
    }
    kd[i] = k;
}

__global__ void k_invert_perm(int64_t n, const int32_t* __restrict__ ref_of_bo, int32_t* __restrict__ bo_of_ref) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) bo_of_ref[ref_of_bo[i]] = (int32_t)i;
}

// each part's lesser and greater cell's k, the axis in their sign bits (the block-Jacobi
// smoother's only inputs): axis bit 0 on the first, bit 1 on the second
__global__ void k_brick_jacobi_k(int64_t n, const int32_t* __restrict__ ref_of_bo, const int8_t* __restrict__ axis,
                                 const int32_t* __restrict__ cella, const int32_t* __restrict__ cellb,
                                 const int4* __restrict__ cell, float2* __restrict__ kk) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t k = ref_of_bo[i];
    const int a = axis[k];
    const int32_t A = cella[k], B = cellb[k];
    const float kA = A >= 0 ? __int_as_float(cell[2 * (int64_t)A + 1].z) : 0.0f;
    const float kB = B >= 0 ? __int_as_float(cell[2 * (int64_t)B + 1].z) : 0.0f;
    kk[i] = make_float2(copysignf(kA, (a & 1) ? -1.0f : 1.0f), copysignf(kB, (a & 2) ? -1.0f : 1.0f));
}

// ---- permutations ------------------------------------------------------------------------
// dst[i] = src[idx[i]], W values an entry
template <class T, int W>
__global__ void k_gather_rows(int64_t n, const int32_t* __restrict__ idx, const T* __restrict__ src, T* __restrict__ dst) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t s = idx[i];
#pragma unroll
    for (int j = 0; j < W; j++) dst[W * i + j] = src[W * s + j];
}

__global__ void k_map_ids(int64_t n, const int32_t* __restrict__ map, int32_t* __restrict__ v) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) v[i] = map[v[i]];
}

// a dense top of a piece solved at level 0, its rows and columns permuted: out(I, J) =
// in(perm(I), perm(J)) with perm the piece's local part permutation (`map`: global part
// of each global part), 6 x 6 blocks
__global__ void k_permute_top(const int32_t* __restrict__ top, const int64_t* __restrict__ pstart,
                              const int64_t* __restrict__ kinv_off, const double* __restrict__ in,
                              double* __restrict__ out, const int32_t* __restrict__ map) {
    const int p = top[blockIdx.x];
    const int64_t k0 = pstart[p];
    const int64_t np = pstart[p + 1] - k0, n = 6 * np;
    const double* A = in + kinv_off[blockIdx.x];
    double* O = out + kinv_off[blockIdx.x];
    for (int64_t e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int64_t J = e / n, I = e % n;
        const int64_t sj = 6 * (map[k0 + J / 6] - k0) + J % 6, si = 6 * (map[k0 + I / 6] - k0) + I % 6;
        O[e] = A[sj * n + si];
    }
}

// ---- the stencil -------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ void lds6(const T* __restrict__ box, int e, T (&o)[6]) {
    if constexpr (sizeof(T) == 8) {
        const double2* q = reinterpret_cast<const double2*>(box + 6 * e);
        const double2 a = q[0], b = q[1], c = q[2];
        o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y; o[4] = c.x; o[5] = c.y;
    } else {
        const float2* q = reinterpret_cast<const float2*>(box + 6 * e);
        const float2 a = q[0], b = q[1], c = q[2];
        o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y; o[4] = c.x; o[5] = c.y;
    }
}
template <class T>
__device__ __forceinline__ void sts6(T* __restrict__ box, int e, const T (&o)[6]) {
    if constexpr (sizeof(T) == 8) {
        double2* q = reinterpret_cast<double2*>(box + 6 * e);
        q[0] = make_double2(o[0], o[1]);
        q[1] = make_double2(o[2], o[3]);
        q[2] = make_double2(o[4], o[5]);
    } else {
        float2* q = reinterpret_cast<float2*>(box + 6 * e);
        q[0] = make_float2(o[0], o[1]);
        q[1] = make_float2(o[2], o[3]);
        q[2] = make_float2(o[4], o[5]);
    }
}

// t += (row strip SLOT of the level-0 cell template k s D T D, spacing baked in: BlkS) *
// (the six faces of cell c, from the box)
template <int SLOT, int F, class T>
__device__ __forceinline__ void face_macs_s(const T (&xs)[6][6], T (&t)[6]) {
    if constexpr (F < 6) {
        BlkS<SLOT, F>::mac(xs[F], t);
        face_macs_s<SLOT, F + 1, T>(xs, t);
    }
}

// acc += kc * (row strip SLOT of the cell matrix) * (the six faces of cell c)
template <int SLOT, class T>
__device__ __forceinline__ void box_term(const T* __restrict__ box, int c0, int c1, int c2, T kc, T (&acc)[6]) {
    T xs[6][6];
    lds6<T>(box, box_index(0, c0, c1, c2), xs[0]);
    lds6<T>(box, box_index(0, c0 + 1, c1, c2), xs[1]);
    lds6<T>(box, box_index(1, c0, c1, c2), xs[2]);
    lds6<T>(box, box_index(1, c0, c1 + 1, c2), xs[3]);
    lds6<T>(box, box_index(2, c0, c1, c2), xs[4]);
    lds6<T>(box, box_index(2, c0, c1, c2 + 1), xs[5]);
    T t[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
    face_macs_s<SLOT, 0, T>(xs, t);
#pragma unroll
    for (int i = 0; i < 6; i++) acc[i] = fma(kc, t[i], acc[i]);
}

// one part on axis AX at brick-local face position l: Kx from its lesser cell (l - e_AX,
// strip 2AX+1) and greater cell (l, strip 2AX), then the epilogue (grid.cu's modes)
template <int AX, class T, int MODE>
__device__ __forceinline__ void brick_part(const T* __restrict__ box, const float* __restrict__ kbox, int l0, int l1,
                                           int l2, int32_t q, const T* __restrict__ r, T* __restrict__ y,
                                           T* __restrict__ y2, T s, T w) {
    constexpr int BA = AX == 0 ? BX : AX == 1 ? BY : BZ;
    const int la = AX == 0 ? l0 : AX == 1 ? l1 : l2;
    const T kG = la < BA ? (T)kbox[kbox_index(l0, l1, l2)] : T(0);  // beyond the piece on its + plane
    const T kL = (T)kbox[kbox_index(l0 - (AX == 0), l1 - (AX == 1), l2 - (AX == 2))];
    T acc[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
    if (kL != T(0)) box_term<2 * AX + 1, T>(box, l0 - (AX == 0), l1 - (AX == 1), l2 - (AX == 2), kL, acc);
    if (kG != T(0)) box_term<2 * AX, T>(box, l0, l1, l2, kG, acc);
    const T(&kx)[6] = acc;
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
        dinv<AX, T>(kL, kG, s, o, d);
        store6<T>(y2, q, d);
    } else if constexpr (MODE == ST_RES_W) {
        load6<T>(r, q, o);
#pragma unroll
        for (int j = 0; j < 6; j++) o[j] = fma(-w, kx[j], o[j]);
        store6<T>(y, q, o);
    } else if constexpr (MODE == ST_PROLONG) {
        T d[6], xv[6], acc2[6];
        dinv<AX, T>(kL, kG, s, kx, d);
        lds6<T>(box, box_index(AX, l0, l1, l2), xv);
        load6<T>(y, q, acc2);
#pragma unroll
        for (int j = 0; j < 6; j++) o[j] = acc2[j] + fma(-w, d[j], xv[j]);
        store6<T>(y, q, o);
    } else {
        T rv[6], d[6], xv[6];
        load6<T>(r, q, rv);
#pragma unroll
        for (int j = 0; j < 6; j++) rv[j] -= kx[j];
        dinv<AX, T>(kL, kG, s, rv, d);
        lds6<T>(box, box_index(AX, l0, l1, l2), xv);
#pragma unroll
        for (int j = 0; j < 6; j++) o[j] = fma(w, d[j], xv[j]);
        store6<T>(y, q, o);
    }
}

// cp.async: an asynchronous copy of 8 or 16 bytes from global to shared memory
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// one part's six values into the box: 16-byte copies for FP64 where x is 16-byte aligned
// (a part is 48 bytes), else 8-byte ones (FP32 parts are 24 bytes)
template <class T>
__device__ __forceinline__ void copy_part(T* dst, const T* src, bool vec16) {
    if (sizeof(T) == 8 && vec16) {
        cp_async16(dst, src);
        cp_async16(dst + 2, src + 2);
        cp_async16(dst + 4, src + 4);
    } else {
        constexpr int STEP = 8 / sizeof(T);
#pragma unroll
        for (int j = 0; j < 6; j += STEP) cp_async8(dst + j, src + j);
    }
}

// Shared memory of one brick: the x box (NBOX faces, 6 values each), the k box and the
// brick's parts' part_codes in storage order.
template <class T>
constexpr size_t brick_smem() {
    return sizeof(T) * 6 * NBOX + sizeof(float) * KB + sizeof(uint16_t) * (NSLOT + 8);
}

// the box entry of an own part's face, from its part_code
__device__ __forceinline__ int own_entry(uint32_t c) {
    const int a = (c >> 12) & 3, l0 = (c >> 8) & 7, l1 = (c >> 4) & 15, l2 = c & 15;
    return a == 0 ? box_index(0, l0, l1, l2) : a == 1 ? box_index(1, l0, l1, l2) : box_index(2, l0, l1, l2);
}

// Resident blocks an SM the register cap aims at: five in FP32 (shared memory allows
// five), four where the epilogue applies the block-Jacobi factor (more registers, which
// five blocks would spill), three in FP64 (shared memory allows three).
template <class T, int MODE>
constexpr int brick_min_blocks() {
    return sizeof(T) == 8 ? 3 : (MODE == ST_RES_JAC || MODE == ST_PROLONG || MODE == ST_SMOOTH) ? 4 : 5;
}

// Level 0 applied over bricks, one thread block a brick (see the file's head). The same
// epilogues as grid.cu's k_stencil: y = Kx, r - Kx, ... (ST_* in level0.cuh).
template <class T, int MODE>
__global__ void __launch_bounds__(BRICK_THREADS, brick_min_blocks<T, MODE>()) k_brick_stencil(BrickView v, const T* __restrict__ x,
                                                                 const T* __restrict__ r, T* __restrict__ y,
                                                                 T* __restrict__ y2, T s,
                                                                 const double* __restrict__ step,
                                                                 const int32_t* __restrict__ skip_row,
                                                                 const int32_t* __restrict__ done) {
    extern __shared__ __align__(16) unsigned char brick_sm[];
    T* box = reinterpret_cast<T*>(brick_sm);
    float* kbox = reinterpret_cast<float*>(box + 6 * NBOX);
    uint16_t* codes = reinterpret_cast<uint16_t*>(kbox + KB);
    const int b = blockIdx.x;
    const int4 inf = v.info[b];
    if (done && done[inf.x]) return;
    const int32_t start = v.start[b], cnt = v.start[b + 1] - start;
    if (cnt == 0) return;                            // only cells: nothing of its own to write
    if (skip_row && skip_row[start]) return;         // the piece is solved at level 0
    const T w = step ? (T)step[inf.x] : T(0);
    // the box starts at zero: faces that are no part stay so
    {
        constexpr int N16 = (int)(sizeof(T) * 6 * NBOX / 16);
        float4* z = reinterpret_cast<float4*>(box);
        for (int i = threadIdx.x; i < N16; i += BRICK_THREADS) z[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
    // The box is filled by asynchronous copies (cp.async: global memory straight to shared
    // memory, no registers in between) issued together and awaited once: the brick's own
    // parts, their run read in order, each to its face's entry (by its part_code, kept for
    // the part phase), and the halo parts of its resolved list (bricks_build).
    const bool vec16 = sizeof(T) == 8 && ((reinterpret_cast<uintptr_t>(x) & 15) == 0);
    for (int t = threadIdx.x; t < cnt; t += BRICK_THREADS) {
        const uint32_t c = __ldg(v.code + start + t);
        codes[t] = (uint16_t)c;
        copy_part<T>(box + 6 * own_entry(c), x + 6 * ((int64_t)start + t), vec16);
    }
    {
        const int32_t h0 = __ldg(v.hstart + b), h1 = __ldg(v.hstart + b + 1);
        for (int32_t h = h0 + threadIdx.x; h < h1; h += BRICK_THREADS)
            copy_part<T>(box + 6 * (int)__ldg(v.hent + h), x + 6 * (int64_t)__ldg(v.hsrc + h), vec16);
    }
    // k of the brick's cells and of the single layers before it (-x, -y, -z)
    {
        const int t = threadIdx.x;  // BRICK_THREADS == BCELLS: one cell of the brick a thread
        kbox[kbox_index(t / (BY * BZ), t / BZ % BY, t % BZ)] = __ldg(v.kd + (int64_t)b * BCELLS + t);
        if (t < HK) {
            int h0, h1, h2;
            if (t < HKX) {
                h0 = -1, h1 = t / BZ, h2 = t % BZ;
            } else if (t < HKX + HKY) {
                h0 = (t - HKX) / BZ, h1 = -1, h2 = (t - HKX) % BZ;
            } else {
                h0 = (t - HKX - HKY) / BY, h1 = (t - HKX - HKY) % BY, h2 = -1;
            }
            kbox[kbox_index(h0, h1, h2)] = __ldg(v.hk + (int64_t)b * HK + t);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    // the brick's parts, in storage order (their vectors from the brick's first part on)
    const T* rb = r ? r + 6 * (int64_t)start : nullptr;
    T* yb = y + 6 * (int64_t)start;
    T* y2b = y2 ? y2 + 6 * (int64_t)start : nullptr;
    for (int t = threadIdx.x; t < cnt; t += BRICK_THREADS) {
        const uint32_t c = codes[t];
        const int a = (c >> 12) & 3, l0 = (c >> 8) & 7, l1 = (c >> 4) & 15, l2 = c & 15;
        if (a == 0)
            brick_part<0, T, MODE>(box, kbox, l0, l1, l2, t, rb, yb, y2b, s, w);
        else if (a == 1)
            brick_part<1, T, MODE>(box, kbox, l0, l1, l2, t, rb, yb, y2b, s, w);
        else
            brick_part<2, T, MODE>(box, kbox, l0, l1, l2, t, rb, yb, y2b, s, w);
    }
}

// x = w D^-1 r over brick-ordered parts (pre-smoothing, bodies.rs:386)
template <class T>
__global__ void __launch_bounds__(256) k_brick_jacobi(int64_t n, const float2* __restrict__ kk, const T* __restrict__ r,
                                                      T* __restrict__ x, T s, const int32_t* __restrict__ piece,
                                                      const double* __restrict__ step,
                                                      const int32_t* __restrict__ skip_row,
                                                      const int32_t* __restrict__ done) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (skip_row && skip_row[i]) return;
    const int p = piece[i];
    if (done && done[p]) return;
    const T w = step ? (T)step[p] : T(1);
    const float2 e = __ldg(kk + i);
    const int ax = (signbit(e.x) ? 1 : 0) | (signbit(e.y) ? 2 : 0);
    const T kA = (T)fabsf(e.x), kB = (T)fabsf(e.y);
    T rv[6], d[6];
    load6<T>(r, (int32_t)i, rv);
    if (ax == 0)
        dinv<0, T>(kA, kB, s, rv, d);
    else if (ax == 1)
        dinv<1, T>(kA, kB, s, rv, d);
    else
        dinv<2, T>(kA, kB, s, rv, d);
#pragma unroll
    for (int j = 0; j < 6; j++) d[j] *= w;
    store6<T>(x, i, d);
}

// A brick's halo, resolved once for the solve: for each entry of the halo table, the
// part (brick order) that fills it, where the neighbour brick holds one there. Pass 0
// counts a brick's items, pass 1 writes them at the brick's offset.
template <int PASS>
__global__ void k_halo_lists(int32_t nb, const int4* __restrict__ info, const BrickGeo* __restrict__ geo,
                             const int32_t* __restrict__ nbr, const uint32_t* __restrict__ mask,
                             const uint16_t* __restrict__ pre, const int32_t* __restrict__ start,
                             const uint2* __restrict__ tbl, int32_t nhalo, int32_t* __restrict__ count,
                             const int32_t* __restrict__ hstart, uint16_t* __restrict__ hent,
                             int32_t* __restrict__ hsrc) {
    const int32_t b = blockIdx.x;
    if (b >= nb) return;
    const int4 in = info[b];
    const BrickGeo g = geo[in.x];
    const bool last[3] = {in.y == g.nbx - 1, in.z == g.nby - 1, in.w == g.nbz - 1};
    __shared__ int32_t n_items;
    if (threadIdx.x == 0) n_items = 0;
    __syncthreads();
    for (int h = threadIdx.x; h < nhalo; h += blockDim.x) {
        const uint2 ee = tbl[h];
        const int a = (ee.x >> 25) & 3;
        const uint32_t e = (((ee.x >> 24) & 1u) && last[a]) ? ee.y : ee.x;
        const int q = (e >> 27) & 15, slot = e & 0xFFF;
        if (q == 0) continue;  // the brick's own plane part
        const int32_t id = nbr[(int64_t)b * NNB + q];
        if (id < 0) continue;
        const uint32_t m = mask[(int64_t)id * MW + slot / 32];
        if (!((m >> (slot & 31)) & 1u)) continue;
        const int32_t src = start[id] + pre[(int64_t)id * MW + slot / 32] + __popc(m & ((1u << (slot & 31)) - 1u));
        const int32_t k = atomicAdd(&n_items, 1);
        if (PASS == 1) {
            hent[hstart[b] + k] = (uint16_t)((ee.x >> 12) & 0xFFF);
            hsrc[hstart[b] + k] = src;
        }
    }
    __syncthreads();
    if (PASS == 0 && threadIdx.x == 0) count[b] = n_items;
}

// per brick the k of the cells of its -x, -y and -z layers (the neighbours' boundary cells)
__global__ void k_halo_k(int32_t nb, const int32_t* __restrict__ nbr, const float* __restrict__ kd,
                         float* __restrict__ hk) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)nb * HK) return;
    const int64_t b = i / HK;
    const int t = (int)(i % HK);
    int q, src;
    if (t < HKX) {
        q = 1;
        src = ((BX - 1) * BY + t / BZ) * BZ + t % BZ;
    } else if (t < HKX + HKY) {
        q = 2;
        src = ((t - HKX) / BZ * BY + BY - 1) * BZ + (t - HKX) % BZ;
    } else {
        q = 3;
        src = ((t - HKX - HKY) / BY * BY + (t - HKX - HKY) % BY) * BZ + BZ - 1;
    }
    const int32_t id = nbr[b * NNB + q];
    hk[i] = id >= 0 ? kd[(int64_t)id * BCELLS + src] : 0.0f;
}

BrickView view_of(const Bricks& K) {
    BrickView v;
    v.start = K.start.get();
    v.mask = K.mask.get();
    v.pre = K.pre.get();
    v.info = K.info.get();
    v.nbr = K.nbr.get();
    v.kd = K.kd.get();
    v.geo = reinterpret_cast<const BrickGeo*>(K.geo.get());
    v.code = K.code.get();
    v.hstart = K.hstart.get();
    v.hent = K.hent.get();
    v.hsrc = K.hsrc.get();
    v.hk = K.hk.get();
    return v;
}

// each brick-ordered part's part_code, from its sort key's slot
__global__ void k_part_codes(int64_t n, const uint64_t* __restrict__ key, uint16_t* __restrict__ code) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int e = (int)(key[i] % NSLOT);
    int a = 0;
    if (e >= NS0 + NS1) {
        a = 2;
        e -= NS0 + NS1;
    } else if (e >= NS0) {
        a = 1;
        e -= NS0;
    }
    const int e2 = slot_ext(a, 2), e1 = slot_ext(a, 1);
    code[i] = (uint16_t)part_code(a, e / (e2 * e1), e / e2 % e1, e % e2);
}

}  // namespace

// Builds the brick layout of a batch's level 0 (voxel pieces) from its part data.
void bricks_build(Context& ctx, Batch& b) {
    Grid0& g = b.grid;
    Level& L = b.levels[0];
    Bricks& K = g.bricks;
    cudaStream_t st = ctx.stream;
    MemStats* ms = &ctx.mem;
    const int np = b.npieces;
    const int64_t n = L.n;
    std::vector<BrickGeo> geo(np);
    int64_t npos = 0;
    for (int p = 0; p < np; p++) {
        BrickGeo& q = geo[p];
        q.nx = g.dims_h[3 * p];
        q.ny = g.dims_h[3 * p + 1];
        q.nz = g.dims_h[3 * p + 2];
        q.nbx = (q.nx + BX - 1) / BX;
        q.nby = (q.ny + BY - 1) / BY;
        q.nbz = (q.nz + BZ - 1) / BZ;
        q.goff = g.grid_off[p];
        q.pos0 = npos;
        q.pad = q.pad2 = 0;
        npos += (int64_t)q.nbx * q.nby * q.nbz;
    }
    K.geo.alloc(np * sizeof(BrickGeo), st, ms);
    SC_CK(cudaMemcpyAsync(K.geo.get(), geo.data(), np * sizeof(BrickGeo), cudaMemcpyHostToDevice, st));
    const std::vector<uint2> tbl = halo_table();
    K.nhalo = (int32_t)tbl.size();
    K.halo.alloc(tbl.size() * sizeof(uint2), st, ms);
    SC_CK(cudaMemcpyAsync(K.halo.get(), tbl.data(), tbl.size() * sizeof(uint2), cudaMemcpyHostToDevice, st));
    const BrickGeo* geo_d = reinterpret_cast<const BrickGeo*>(K.geo.get());
    DBuf<int32_t> flag, bid;
    flag.alloc(npos + 1, st, ms);
    flag.zero();
    bid.alloc(npos + 1, st, ms);
    if (g.ncells > 0) {
        k_mark_cell_bricks<<<grid_for(g.ncells, 256), 256, 0, st>>>(g.ncells, g.cell_flat.get(), geo_d, np, flag.get());
        SC_LAUNCH_CK();
    }
    DBuf<uint64_t> key, key_s;
    DBuf<int32_t> ids;
    key.alloc(n, st, ms);
    key_s.alloc(n, st, ms);
    ids.alloc(n, st, ms);
    K.ref_of_bo.alloc(n, st, ms);
    k_part_keys<<<grid_for(n, 256), 256, 0, st>>>(n, L.piece.get(), L.site.get(), g.axis.get(), geo_d, flag.get(),
                                                  key.get(), ids.get());
    SC_LAUNCH_CK();
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, flag.get(), bid.get(), npos + 1, st);
    cub::DeviceScan::ExclusiveSum(ctx.cub_scratch(tb), tb, flag.get(), bid.get(), npos + 1, st);
    int end_bit = 1;
    while (end_bit < 64 && ((uint64_t)1 << end_bit) <= (uint64_t)npos * NSLOT) end_bit++;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, key.get(), key_s.get(), ids.get(), K.ref_of_bo.get(), n, 0, end_bit,
                                    st);
    cub::DeviceRadixSort::SortPairs(ctx.cub_scratch(tb), tb, key.get(), key_s.get(), ids.get(), K.ref_of_bo.get(), n,
                                    0, end_bit, st);
    int32_t nb = 0;
    SC_CK(cudaMemcpyAsync(&nb, bid.get() + npos, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    SC_CK(cudaStreamSynchronize(st));
    K.n_bricks = nb;
    const int64_t nb1 = std::max<int64_t>(nb, 1);
    DBuf<int32_t> cnt;
    cnt.alloc(nb1 + 1, st, ms);
    cnt.zero();
    K.mask.alloc(nb1 * MW, st, ms);
    K.mask.zero();
    k_brick_counts<<<grid_for(n, 256), 256, 0, st>>>(n, key_s.get(), bid.get(), cnt.get(), K.mask.get());
    SC_LAUNCH_CK();
    K.start.alloc(nb1 + 1, st, ms);
    cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.get(), K.start.get(), nb + 1, st);
    cub::DeviceScan::ExclusiveSum(ctx.cub_scratch(tb), tb, cnt.get(), K.start.get(), nb + 1, st);
    K.info.alloc(nb1, st, ms);
    K.nbr.alloc(nb1 * NNB, st, ms);
    K.pre.alloc(nb1 * MW, st, ms);
    k_brick_info<<<grid_for(npos, 256), 256, 0, st>>>(npos, flag.get(), bid.get(), geo_d, np, K.mask.get(),
                                                      K.info.get(), K.nbr.get(), K.pre.get());
    SC_LAUNCH_CK();
    K.kd.alloc(nb1 * BCELLS, st, ms);
    if (nb > 0) {
        k_brick_k<<<grid_for((int64_t)nb * BCELLS, 256), 256, 0, st>>>(nb, K.info.get(), geo_d, g.gridmap.get(),
                                                                        g.cell.get(), K.kd.get());
        SC_LAUNCH_CK();
    }
    K.code.alloc(n, st, ms);
    k_part_codes<<<grid_for(n, 256), 256, 0, st>>>(n, key_s.get(), K.code.get());
    SC_LAUNCH_CK();
    // each brick's halo list and the k of its neighbours' boundary cells
    K.hstart.alloc(nb1 + 1, st, ms);
    K.hk.alloc(nb1 * HK, st, ms);
    if (nb > 0) {
        const uint2* tbl_d = reinterpret_cast<const uint2*>(K.halo.get());
        DBuf<int32_t> hcount;
        hcount.alloc(nb1 + 1, st, ms);
        hcount.zero();
        k_halo_lists<0><<<nb, 256, 0, st>>>(nb, K.info.get(), geo_d, K.nbr.get(), K.mask.get(), K.pre.get(),
                                             K.start.get(), tbl_d, K.nhalo, hcount.get(), nullptr, nullptr, nullptr);
        SC_LAUNCH_CK();
        cub::DeviceScan::ExclusiveSum(nullptr, tb, hcount.get(), K.hstart.get(), nb + 1, st);
        cub::DeviceScan::ExclusiveSum(ctx.cub_scratch(tb), tb, hcount.get(), K.hstart.get(), nb + 1, st);
        int32_t items = 0;
        SC_CK(cudaMemcpyAsync(&items, K.hstart.get() + nb, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        SC_CK(cudaStreamSynchronize(st));
        K.hent.alloc(std::max<int32_t>(items, 1), st, ms);
        K.hsrc.alloc(std::max<int32_t>(items, 1), st, ms);
        k_halo_lists<1><<<nb, 256, 0, st>>>(nb, K.info.get(), geo_d, K.nbr.get(), K.mask.get(), K.pre.get(),
                                             K.start.get(), tbl_d, K.nhalo, nullptr, K.hstart.get(), K.hent.get(),
                                             K.hsrc.get());
        SC_LAUNCH_CK();
        k_halo_k<<<grid_for((int64_t)nb * HK, 256), 256, 0, st>>>(nb, K.nbr.get(), K.kd.get(), K.hk.get());
        SC_LAUNCH_CK();
    }
    K.bo_of_ref.alloc(n, st, ms);
    k_invert_perm<<<grid_for(n, 256), 256, 0, st>>>(n, K.ref_of_bo.get(), K.bo_of_ref.get());
    SC_LAUNCH_CK();
    K.kk.alloc(n, st, ms);
    k_brick_jacobi_k<<<grid_for(n, 256), 256, 0, st>>>(n, K.ref_of_bo.get(), g.axis.get(), g.cella.get(),
                                                        g.cellb.get(), g.cell.get(), K.kk.get());
    SC_LAUNCH_CK();
    SC_CK(cudaStreamSynchronize(st));  // the host's geo vector goes out of scope
}

// v (n rows of W values) into the order `idx` gives: v[i] = old v[idx[i]]
template <class T, int W>
static void permute_rows(Context& ctx, DBuf<T>& v, int64_t n, const int32_t* idx) {
    if (n <= 0 || v.size() < (size_t)(W * n)) return;
    DBuf<T> out;
    out.alloc(W * n, ctx.stream, &ctx.mem);
    k_gather_rows<T, W><<<grid_for(n, 256), 256, 0, ctx.stream>>>(n, idx, v.get(), out.get());
    SC_LAUNCH_CK();
    v = std::move(out);
}

static void permute_tops(Context& ctx, Level& L, const int32_t* map) {
    if (L.top_h.empty() || !L.kinv.size()) return;
    DBuf<double> out;
    out.alloc(L.kinv.size(), ctx.stream, &ctx.mem);
    k_permute_top<<<(unsigned)L.top_h.size(), 256, 0, ctx.stream>>>(L.top.get(), L.pstart_d.get(), L.kinv_off.get(),
                                                                    L.kinv.get(), out.get(), map);
    SC_LAUNCH_CK();
    L.kinv = std::move(out);
}

// Into brick order for the iterations: the loads, each part's body and offset, the
// bodies' member lists and the dense tops of pieces solved at level 0.
void bricks_enter(Context& ctx, Batch& b) {
    Grid0& g = b.grid;
    Bricks& K = g.bricks;
    Level& L = b.levels[0];
    const int64_t n = L.n;
    const int32_t* r_of_b = K.ref_of_bo.get();
    permute_rows<double, 6>(ctx, b.loads, n, r_of_b);
    permute_rows<double, 3>(ctx, L.mf_r, n, r_of_b);
    permute_rows<float, 3>(ctx, L.mf_r32, n, r_of_b);
    permute_rows<int32_t, 1>(ctx, L.up, n, r_of_b);
    if (L.mem.size()) {
        k_map_ids<<<grid_for((int64_t)L.mem.size(), 256), 256, 0, ctx.stream>>>((int64_t)L.mem.size(),
                                                                               K.bo_of_ref.get(), L.mem.get());
        SC_LAUNCH_CK();
    }
    // out(I, J) = in(ref(I), ref(J)): ref of a brick-ordered part is ref_of_bo
    permute_tops(ctx, L, r_of_b);
    K.active = true;
}

// Back to the reference's order; x (brick order, 6 per part) too when given.
void bricks_leave(Context& ctx, Batch& b, DBuf<double>* x) {
    Grid0& g = b.grid;
    Bricks& K = g.bricks;
    if (!K.active) return;
    Level& L = b.levels[0];
    const int64_t n = L.n;
    const int32_t* b_of_r = K.bo_of_ref.get();
    permute_rows<double, 6>(ctx, b.loads, n, b_of_r);
    permute_rows<double, 3>(ctx, L.mf_r, n, b_of_r);
    permute_rows<float, 3>(ctx, L.mf_r32, n, b_of_r);
    permute_rows<int32_t, 1>(ctx, L.up, n, b_of_r);
    if (L.mem.size()) {
        k_map_ids<<<grid_for((int64_t)L.mem.size(), 256), 256, 0, ctx.stream>>>((int64_t)L.mem.size(),
                                                                               K.ref_of_bo.get(), L.mem.get());
        SC_LAUNCH_CK();
    }
    permute_tops(ctx, L, b_of_r);
    if (x) permute_rows<double, 6>(ctx, *x, n, b_of_r);
    K.active = false;
}

template <class T>
void brick_permute(Context& ctx, const Batch& b, const T* in, T* out, bool to_bricks) {
    const Bricks& K = b.grid.bricks;
    const int64_t n = b.levels[0].n;
    if (n <= 0) return;
    k_gather_rows<T, 6><<<grid_for(n, 256), 256, 0, ctx.stream>>>(n, to_bricks ? K.ref_of_bo.get() : K.bo_of_ref.get(),
                                                                  in, out);
    SC_LAUNCH_CK();
}
template void brick_permute<double>(Context&, const Batch&, const double*, double*, bool);
template void brick_permute<float>(Context&, const Batch&, const float*, float*, bool);

template <class T, int MODE>
void brick_stencil(Context& ctx, const Batch& b, const T* x, const T* r, T* y, T* y2, const double* step,
                   const int32_t* skip_row, const int32_t* done) {
    const Bricks& K = b.grid.bricks;
    if (K.n_bricks <= 0) return;
    constexpr size_t smem = brick_smem<T>();
    static const bool attr_set = [] {  // once per instantiation (thread-safe)
        SC_CK(cudaFuncSetAttribute(k_brick_stencil<T, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        return true;
    }();
    (void)attr_set;
    k_brick_stencil<T, MODE><<<(unsigned)K.n_bricks, BRICK_THREADS, smem, ctx.stream>>>(
        view_of(K), x, r, y, y2, (T)b.grid.s, step, skip_row, done);
    SC_LAUNCH_CK();
}

#define SC_BRICK_MODES(T)                                                                                            \
    template void brick_stencil<T, ST_Y>(Context&, const Batch&, const T*, const T*, T*, T*, const double*,          \
                                         const int32_t*, const int32_t*);                                           \
    template void brick_stencil<T, ST_RES>(Context&, const Batch&, const T*, const T*, T*, T*, const double*,        \
                                           const int32_t*, const int32_t*);                                         \
    template void brick_stencil<T, ST_RES_JAC>(Context&, const Batch&, const T*, const T*, T*, T*, const double*,    \
                                               const int32_t*, const int32_t*);                                     \
    template void brick_stencil<T, ST_RES_W>(Context&, const Batch&, const T*, const T*, T*, T*, const double*,      \
                                             const int32_t*, const int32_t*);                                       \
    template void brick_stencil<T, ST_PROLONG>(Context&, const Batch&, const T*, const T*, T*, T*, const double*,    \
                                               const int32_t*, const int32_t*);                                     \
    template void brick_stencil<T, ST_SMOOTH>(Context&, const Batch&, const T*, const T*, T*, T*, const double*,     \
                                              const int32_t*, const int32_t*);
SC_BRICK_MODES(double)
SC_BRICK_MODES(float)
#undef SC_BRICK_MODES

template <class T>
void brick_jacobi(Context& ctx, const Batch& b, const T* r, T* x, const double* step, const int32_t* skip_row,
                  const int32_t* done) {
    const Level& L = b.levels[0];
    k_brick_jacobi<T><<<grid_for(L.n, 256), 256, 0, ctx.stream>>>(L.n, b.grid.bricks.kk.get(), r, x, (T)b.grid.s,
                                                                  L.piece.get(), step, skip_row, done);
    SC_LAUNCH_CK();
}
template void brick_jacobi<double>(Context&, const Batch&, const double*, double*, const double*, const int32_t*,
                                   const int32_t*);
template void brick_jacobi<float>(Context&, const Batch&, const float*, float*, const double*, const int32_t*,
                                  const int32_t*);

}  // namespace sc
