// The statics solve on the device: a batch of independent pieces, each with its own
// smoothed-aggregation hierarchy (statics/src/bodies.rs:123-282), solved by conjugate
// gradients (bodies.rs:338-373) preconditioned by V-cycles (bodies.rs:377-403), all
// pieces advanced together by batched kernels. A single structure is a batch of one.
//
// Layout in HBM, per level: parts of piece 0, then piece 1, ... (pieces contiguous);
// six-vectors as 6 consecutive values per part (48 B FP64, 24 B FP32); operators as
// block-sparse rows of 6x6 blocks (36 values, row-major), both triangles stored, columns
// sorted; level 0 of voxel pieces is matrix-free (a per-cell template, see grid.cu).
#pragma once
#include <cuda_runtime.h>

#include <chrono>
#include <memory>
#include <vector>

#include "common.cuh"

namespace sc {

constexpr int CHUNK = 4096;  // parts per reduction chunk (chunks never cross pieces)

// Level 0 of voxel pieces in brick order (brick.cu): the layout of the iterations.
struct Bricks {
    int32_t n_bricks = 0;
    bool active = false;        // the batch's level-0 vectors and transfer arrays are in brick order
    DBuf<int32_t> start;        // n_bricks + 1: each brick's first part (brick order)
    DBuf<uint32_t> mask;        // per brick: one bit per slot, set where the slot holds a part
    DBuf<uint16_t> pre;         // per brick and mask word: parts in the words before it
    DBuf<int4> info;            // per brick: piece, brick coordinates
    DBuf<int32_t> nbr;          // per brick: the 13 bricks its stencil reads from (-1 none)
    DBuf<float> kd;             // per brick: each cell's k (0 where not free)
    DBuf<uint8_t> geo;          // per piece: dimensions, brick grid, first cell and brick
    DBuf<uint8_t> halo;         // the entries of a brick's shared-memory box its neighbours fill
    int32_t nhalo = 0;
    DBuf<uint16_t> code;        // per brick-ordered part: its axis and brick-local position
    DBuf<int32_t> hstart;       // n_bricks + 1: each brick's halo list
    DBuf<uint16_t> hent;        // per halo item: the box entry it fills
    DBuf<int32_t> hsrc;         // per halo item: the brick-ordered part it comes from
    DBuf<float> hk;             // per brick: the k of its -x, -y, -z neighbours' boundary cells
    DBuf<int32_t> ref_of_bo;    // brick-ordered part -> the reference's part index
    DBuf<int32_t> bo_of_ref;    // and back
    DBuf<float2> kk;            // per brick-ordered part: its cells' k, its axis in their signs
};

// Level 0 of voxel pieces: the cells, and for each part its two cells.
struct Grid0 {
    int64_t ncells = 0;
    double s = 0.125;           // spacing (statics/src/lattice.rs:16, 34-36)
    DBuf<int4> cell;            // 2 int4 per free cell: part ids of slots 0..5 (-1 held), k bits, 0
    DBuf<int32_t> perm;         // parts in order, grouped by axis inside tiles of 1024 parts
    DBuf<int4> slots;           // per perm slot: part, lesser cell, greater cell, axis
    bool pencil = false;        // the plane-pencil stencil (tile 1) or the per-slot one
    bool two_pass = false;      // the two-pass stencil (tile 2): per-cell rows, then per part
    DBuf<int32_t> cell_piece;   // two-pass: per free cell its piece
    DBuf<double> ycell64;       // two-pass: 36 values per free cell
    DBuf<float> ycell32;
    DBuf<int32_t> gridmap;      // per grid cell: its free-cell index or -1
    DBuf<uint8_t> tiles;        // pencil tiles (piece, x0, y0, z0)
    DBuf<uint8_t> geo;          // per piece: dims and first flat cell
    int64_t ntiles = 0;
    int64_t axis_off[4] = {0, 0, 0, 0};  // axis_off[3]: parts in perm
    DBuf<int32_t> cella, cellb; // per part: its lesser cell (node is that cell's + face) and greater cell; -1 if not free
    DBuf<int8_t> axis;          // per part
    DBuf<int64_t> cell_flat;    // per free cell: its flat index in the batch's concatenated grids
    DBuf<double> tpl_s;         // the cell template at spacing s, 36 x 36 (setup only)
    std::vector<int64_t> grid_off;  // per piece: first flat cell index; npieces + 1
    std::vector<int32_t> dims_h;    // per piece: nx, ny, nz
    bool use_bricks = false;        // the iterations run in brick order (sc_options.tile 0)
    Bricks bricks;
};

struct Level {
    int64_t n = 0;                   // parts
    int64_t nnzb = 0;                // stored blocks
    std::vector<int64_t> pstart;     // host copy: piece p's parts are [pstart[p], pstart[p+1])
    DBuf<int64_t> pstart_d;
    DBuf<int32_t> piece;             // part -> piece
    DBuf<double> centre;             // 3 per part
    DBuf<int64_t> site;              // 3 per part: a member node's lesser cell, level-0 units

    bool matrix_free = false;        // level 0 of voxel pieces: apply through Grid0
    DBuf<int64_t> rowptr;
    DBuf<int32_t> col;
    DBuf<double> val;                // 36 per stored block; empty on a matrix-free level 0
    DBuf<float> val32;
    DBuf<uint8_t> desc;              // matrix-free level 0, setup only: each stored block's
                                     // origin in the cell template (level0_blocks.cuh)
    DBuf<double> inv;                // inverse of each part's own block
    DBuf<float> inv32;
    DBuf<double> step;               // per piece: 4/3 / lambda_max(D^-1 K)

    // reductions over each piece's parts
    int64_t nchunks = 0;
    DBuf<int64_t> chunk_lo;          // nchunks + 1 bounds
    DBuf<int32_t> chunk_piece;
    DBuf<int64_t> piece_chunk;       // per piece: first chunk; npieces + 1

    // to the next level (absent at the last)
    DBuf<int32_t> up;                // body at the next level, -1 where the piece tops out here
    int64_t pnnz = 0;
    DBuf<int64_t> prow;              // P: n rows
    DBuf<int32_t> pcol;
    DBuf<double> pval;
    DBuf<float> pval32;
    DBuf<int64_t> tptr;              // P transposed: coarse row c's entries tent[tptr[c]..tptr[c+1])
    DBuf<int64_t> tent;              //   (index into pcol / pval), in fine-row order
    DBuf<int32_t> trow;              //   and the fine row of each
    DBuf<double> ptval;              // P' blocks in that order (restriction as a block-sparse product)
    DBuf<float> ptval32;

    // pieces solved directly at this level
    std::vector<int32_t> top_h;
    DBuf<int32_t> top;               // piece ids
    DBuf<int64_t> kinv_off;          // per top piece: offset of its dense inverse
    DBuf<double> kinv;
    DBuf<int32_t> top_of_part;       // per part: 1 if its piece tops out here

    // level 0 of voxel pieces: matrix-free transfers need each part's offset from its
    // body's centroid and the bodies' member lists (parts in order)
    DBuf<double> mf_r;
    DBuf<float> mf_r32;
    DBuf<int64_t> mem_off;
    DBuf<int32_t> mem;

    // cycle work vectors (levels >= 1 keep r and z for the level above; level 0 of
    // voxel pieces also t and u)
    DBuf<double> r, x, left, z, t, u;
    DBuf<float> r32, x32, left32, z32, t32, u32;
};

struct Batch {
    int32_t npieces = 0;
    std::vector<Level> levels;
    Grid0 grid;                      // when level 0 is matrix-free
    std::vector<int32_t> piece_levels;  // per piece: number of levels
    std::vector<int32_t> piece_status;
    DBuf<int32_t> status_d;          // per piece sc_status from device checks
    std::vector<int64_t> node_count; // per piece: nodes of its lattice
    DBuf<int64_t> node_start;        // per piece: first node (output motions)
    DBuf<int32_t> part_node;         // per level-0 part: its node (within the piece)
    DBuf<double> loads;              // level-0 right-hand side, 6 per part
    DBuf<double> mass;               // per part (voxel pieces)
    double setup_ms = 0;
    int32_t base_level = 0;          // Lattice::level of level 0 (octree keys start one above)
    int32_t sweeps = 1;              // block-Jacobi sweeps before and after each coarse correction
};

struct Context;

// --- grid.cu ------------------------------------------------------------------------
// Build level 0 (numbering, cells, centres, sites, loads, assembled blocks for setup)
// for voxel pieces already on the device.
void grid_level0(Context& ctx, Batch& b, const std::vector<sc_grid>& grids, bool keep_blocks, int32_t tile);
template <class T>
void stencil_apply(Context& ctx, const Batch& b, const T* x, T* y, const int32_t* skip_row, const int32_t* done);
template <class T>
void stencil_residual(Context& ctx, const Batch& b, const T* x, const T* r, T* y, const int32_t* skip_row,
                      const int32_t* done);
void grid_cell_energy(Context& ctx, const Batch& b, const double* x, double* energy_cells);
template <class T>
void level0_down(Context& ctx, const Batch& b, const T* r, T* x, T* left, T* t, T* u, T* rc, const int32_t* done);
template <class T>
void level0_up(Context& ctx, const Batch& b, const T* r, T* x, T* e, const T* zc, T* z, const int32_t* done);
template <class T>
void level0_smooth(Context& ctx, const Batch& b, const T* r, const T* x, T* z, const int32_t* done);

// --- brick.cu -------------------------------------------------------------------------
void bricks_build(Context& ctx, Batch& b);
void bricks_enter(Context& ctx, Batch& b);
void bricks_leave(Context& ctx, Batch& b, DBuf<double>* x);
template <class T>
void brick_permute(Context& ctx, const Batch& b, const T* in, T* out, bool to_bricks);
template <class T, int MODE>
void brick_stencil(Context& ctx, const Batch& b, const T* x, const T* r, T* y, T* y2, const double* step,
                   const int32_t* skip_row, const int32_t* done);
template <class T>
void brick_jacobi(Context& ctx, const Batch& b, const T* r, T* x, const double* step, const int32_t* skip_row,
                  const int32_t* done);

// --- lattice.cu -----------------------------------------------------------------------
void lattice_level0(Context& ctx, Batch& b, const sc_lattice& L, const uint8_t* alive, const uint8_t* gone,
                    const double* loads);

// --- mech.cu: the engine's solver (mechanics/src/solve.rs) -----------------------------
int mech_solve(Context& ctx, int64_t n, const int64_t* sites, const double* at, const double* diag, int64_t npairs,
               const uint32_t* pi, const uint32_t* pj, const double* pb, const double* b, double* x, double tol,
               double size, int32_t* nlevels);
void mech_levels(int64_t n, const int64_t* sites, const double* at, const double* diag, int64_t npairs,
                 const uint32_t* pi, const uint32_t* pj, const double* pb, double size, std::vector<int64_t>& sizes,
                 std::vector<double>& steps);
void mech_levels_device(Context& ctx, int64_t n, const int64_t* sites, const double* at, const double* diag,
                        int64_t npairs, const uint32_t* pi, const uint32_t* pj, const double* pb, double size,
                        std::vector<int64_t>& sizes, std::vector<double>& steps);
void mech_voxel_system(const uint8_t* state, const float* e, int nx, int ny, int nz, double h, double dt,
                       double mass, std::vector<int64_t>& sites, std::vector<double>& at, std::vector<double>& diag,
                       std::vector<uint32_t>& pi, std::vector<uint32_t>& pj, std::vector<double>& pb,
                       std::vector<double>& b);

// --- gather.cu: a coarser level measured from a finer one (statics/src/gather.rs) --------
struct Gathered {
    int32_t level = 0;
    std::vector<double> x, m;
    std::vector<uint8_t> held;
    std::vector<int64_t> around;
    std::vector<int32_t> mat;
    std::vector<int64_t> bi, bj;
    std::vector<int32_t> bmat;  // each bond's material: its cell's
    std::vector<double> p, n, a, d, e, g, ft, fc, fs;
};
// dev: measure the cells on that context's device (NULL: on the host's cores)
void gather_level(Context* dev, const sc_lattice& L, const sc_strength& S, const int32_t* node_mat,
                  const sc_material* materials, int32_t n_materials, bool against_full, int32_t threads,
                  Gathered& out);
void gather_full(const sc_material& m, double* out);

// --- capi.cu / settle.cu -----------------------------------------------------------------
// motions of a lattice into out_dev (6 per node, device); the solve's status
sc_status lattice_motions(Context& ctx, const sc_lattice& L, const uint8_t* alive, const uint8_t* gone,
                          const double* loads, const sc_options& opt, double* out_dev, sc_solve_info* info);
sc_status used_standing(Context& ctx, const sc_lattice& L, const sc_strength& S, const sc_options& opt,
                        double* used, sc_solve_info* info);
sc_status settle(Context& ctx, const sc_lattice& L, const sc_strength& S, const sc_options& opt, uint8_t* gone,
                 sc_settle_info* out);
sc_status as_generated(Context& ctx, const sc_lattice& L, const sc_strength& S, const sc_lattice& G,
                       const sc_strength& GS, const sc_options& opt, double* ft, double* fc, double* fs);

// --- hierarchy.cu ---------------------------------------------------------------------
void setup_chunks(Context& ctx, Level& L, int32_t npieces);
void build_hierarchy(Context& ctx, Batch& b, const sc_options& opt);
void invert_blocks(Context& ctx, Level& L);
void to_float(Context& ctx, const DBuf<double>& a, DBuf<float>& b);

// --- cycle.cu -------------------------------------------------------------------------
struct SolveStats {
    std::vector<int64_t> iterations;
    std::vector<int64_t> refinements;
    std::vector<double> residual;
    std::vector<double> floor;  // per piece: the relative residual rounding x to FP64 leaves
    double work = 0;
};
void pcg_fp64(Context& ctx, Batch& b, const sc_options& opt, DBuf<double>& x, SolveStats& st);
void pcg_mixed(Context& ctx, Batch& b, const sc_options& opt, DBuf<double>& x, SolveStats& st);
void pcg_fp32_cycle(Context& ctx, Batch& b, const sc_options& opt, DBuf<double>& x, SolveStats& st);
template <class T>
void level_apply(Context& ctx, const Batch& b, int l, const T* x, T* y);
void seg_dot(Context& ctx, const Level& L, const double* a, const double* bb, double* out_per_piece);

// Per-family kernel timing with CUDA events on the context's stream.
struct Profiler {
    uint32_t mask = 0;
    struct Pending {
        int fam;
        cudaEvent_t a, b;
        double bytes;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;
    int64_t launches[SC_FAM_COUNT] = {};
    double ms[SC_FAM_COUNT] = {};
    double bytes[SC_FAM_COUNT] = {};
    cudaEvent_t get();
    void flush();
    void reset();
    ~Profiler();
};

struct Context;
// Records a start event now and a stop event at scope exit, for family `fam`.
struct ProfScope {
    Context* c = nullptr;
    int fam = 0;
    double bytes = 0;
    cudaEvent_t a = nullptr;
    ProfScope(Context& ctx, int family, double algorithmic_bytes);
    ~ProfScope();
};

struct Context {
    int device = 0;
    Profiler prof;
    cudaStream_t stream = nullptr;
    MemStats mem;
    std::string last_error;
    // scratch for reductions
    DBuf<double> partial;
    DBuf<double> scal;
    void* cub_tmp = nullptr;
    size_t cub_bytes = 0;
    std::unique_ptr<Batch> last;     // the last solve's hierarchy (parity queries)
    int32_t* pinned = nullptr;       // 16 bytes of pinned host memory for small reads
    cudaGraphConditionalHandle loop_handle = 0;  // the device-side CG loop's condition
    void* cub_scratch(size_t bytes);
    int32_t* pinned_i32();
    ~Context();
};

// Wall-clock phases of a setup: with SC_TIMING=1 in the environment, mark() waits for
// the stream and prints the milliseconds since the previous mark to stderr; otherwise
// it does nothing.
struct PhaseTimer {
    Context& ctx;
    bool on;
    std::chrono::steady_clock::time_point t;
    double alloc_ms0 = 0;
    int64_t allocs0 = 0;
    explicit PhaseTimer(Context& c);
    void mark(const char* phase);
    void note(const char* fmt, ...);  // a line of its own (when on)
};

}  // namespace sc
