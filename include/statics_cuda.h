/*
 * statics_cuda.h — C ABI of the B200 (sm_100a) statics solver.
 *
 * The solver answers the reference's `statics::bodies::motions`
 * (SupraSummus/parallax-world, statics/src/bodies.rs:429): every free node's 6-DOF
 * motion (translation, rotation) under its loads, by conjugate gradients
 * preconditioned with a smoothed-aggregation V-cycle over "bodies within bodies"
 * (octree cells of 2^l level-0 cells, statics/src/lattice.rs:45-47), the top level
 * solved by a dense Cholesky factor (statics/src/bodies.rs:286-328).
 *
 * Plain C types only: every array is caller-owned; host pointers unless a struct says
 * otherwise. Every entry point returns an sc_status (SC_OK = 0) and never aborts; a
 * context is used by one host thread at a time.
 */
#ifndef STATICS_CUDA_H
#define STATICS_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum sc_status {
    SC_OK = 0,
    SC_MAXITER = 1,    /* iteration cap reached before the tolerance (reference: silent, bodies.rs:351) */
    SC_BREAKDOWN = 2,  /* p'Ap <= 0 or a NaN in the CG recurrence */
    SC_NOT_SPD = 3,    /* the top level's Cholesky met a non-positive pivot (reference: NaN, bodies.rs:308) */
    SC_BAD_INPUT = 4,  /* sizes, pointers or indices out of range */
    SC_TIMEOUT = 5,    /* the solve ran past sc_options.timeout_ms */
    SC_CUDA = 6,       /* a CUDA runtime error; sc_last_error() has the text */
    SC_NO_DEVICE = 7   /* no usable sm_100 device */
} sc_status;

enum { SC_CELL_EMPTY = 0, SC_CELL_FREE = 1, SC_CELL_HELD = 2 };
enum { SC_K_UNIFORM = 0, SC_K_LOGNORMAL = 1 };
enum { SC_FP64 = 0, SC_MIXED = 1, SC_MIXED_FP32_KRYLOV = 2 };

typedef struct sc_options {
    double tol;        /* stop at ||r|| <= tol ||b||; reference 1e-6 (bodies.rs:432) */
    int64_t max_iter;  /* CG iteration cap; reference 100000 (bodies.rs:351) */
    int64_t few;       /* coarsen while a piece has more parts than this; reference 64 (bodies.rs:430) */
    int32_t precision; /* SC_FP64: the reference's algorithm in FP64. SC_MIXED: FP64 conjugate
                          gradients (vectors, operator, dots, scalars) preconditioned by the V-cycle
                          in FP32 (stencil, smoother, transfers, coarse operators; FP64 top solve).
                          SC_MIXED_FP32_KRYLOV: one CG with FP32 vectors and stencil as well, FP64
                          dots and scalars, and the FP64 true residual replacing the FP32 one every
                          few iterations (reliable updates) */
    int32_t sweeps;    /* block-Jacobi sweeps before and after each coarse correction; the
                          reference does 1 (bodies.rs:386, 397-401) */
    double inner_tol;  /* unused (kept for layout) */
    int64_t timeout_ms;/* wall-clock bound of one call; 0 = none */
    int32_t tile;      /* voxel pieces, the level-0 stencil of the iterations: 0 = the brick
                          stencil (the iterations run in brick order: bricks of 4 x 8 x 8 cells,
                          each brick's faces and halo staged in shared memory); a power of two
                          >= 32 = the per-part stencil in the reference's part order, with that
                          window of parts grouped by axis; 1 = the plane-pencil stencil; 2 = the
                          two-pass stencil. The setup always uses the per-part stencil. */
    int32_t reserved;
} sc_options;

/* The reference's constants (tol 1e-6, FEW 64, cap 100000, one sweep), FP64. */
void sc_default_options(sc_options* opt);

typedef struct sc_context sc_context;

/* A solver on CUDA device `device`. Replaces nothing in the reference (which keeps no
 * state between calls); it owns the device buffers reused across calls. */
sc_status sc_create(int32_t device, sc_context** out);
void sc_destroy(sc_context* ctx);
const char* sc_last_error(const sc_context* ctx);
const char* sc_status_string(sc_status s);

/* What a solve did. */
#define SC_MAX_LEVELS 24
typedef struct sc_solve_info {
    int64_t iterations;      /* CG iterations */
    int64_t refinements;     /* FP64 true-residual replacements: SC_MIXED_FP32_KRYLOV's reliable
                                updates; under SC_FP64 and SC_MIXED, the times the recursive residual
                                met tol while the true one |b - K x| did not, and was replaced by it */
    int32_t levels;          /* levels of the hierarchy, level 0 included */
    int32_t status;          /* sc_status of the solve (batched solves: of this piece) */
    int64_t parts[SC_MAX_LEVELS];   /* parts per level */
    int64_t blocks[SC_MAX_LEVELS];  /* stored 6x6 blocks per level (both triangles, diagonal included) */
    double steps[SC_MAX_LEVELS];    /* smoother step 4/3 / lambda_max per level (bodies.rs:174) */
    double residual;         /* final relative residual ||b - A x|| / ||b||, recomputed in FP64 */
    double work;             /* the reference's Work counter: parts + pairs per level apply (bodies.rs:194) */
    double setup_ms;         /* hierarchy construction, device time */
    double solve_ms;         /* conjugate gradients, device time */
    int64_t n_nodes;         /* nodes of the lattice */
    int64_t n_parts;         /* free nodes: level-0 unknowns / 6 */
    int64_t peak_bytes;      /* device memory held by the solve at its peak */
    double residual_floor;   /* |K d| / |b| for d = x moved by one unit in the last place of each
                                value (random signs): about the least relative residual any FP64
                                vector of motions has for this piece. Where it is above tol (slender
                                pieces with large motions) the solve stops at it instead: `residual`
                                is then at most about this, and the status SC_OK. */
} sc_solve_info;

/* ---------------------------------------------------------------------------
 * Voxel pieces (the structured fast path).
 *
 * A piece is a grid of level-0 cells, flat index ((x*ny)+y)*nz+z (the order
 * statics/src/lattice.rs:87-102 visits sites). Its lattice is the reference's
 * `build(0, solids)` (statics/src/lattice.rs:124-163): a node on every face of a free
 * cell, numbered in first-touch order, held where the other cell is held; 15 beams of
 * 4 bonds join each free cell's faces; each cell has E = k, G = g_over_e * k, density
 * rho. Each node's load is its mass times `gravity` (force and no moment).
 * ------------------------------------------------------------------------- */
typedef struct sc_grid {
    int32_t nx, ny, nz;
    const uint8_t* state; /* SC_CELL_EMPTY / FREE / HELD, nx*ny*nz */
    const float* k;       /* stiffness per cell, nx*ny*nz */
    double g_over_e;      /* 0.4 for every reference material (statics/src/model.rs:53-58) */
    double rho;           /* density; 512 gives a level-0 cell (0.125 m) a mass of 1 */
    double gravity[3];    /* load per unit mass, e.g. {0, 0, -1} */
    int32_t on_device;    /* state and k are device pointers */
    const double* loads;  /* optional: 6 per node (node order), used instead of mass * gravity;
                             host memory, or device memory when on_device */
} sc_grid;

/* Seeded synthetic piece: value noise of period 8, threshold 0.5, bottom z layer held,
 * the component joined to it kept; k uniform [0.5, 2] (SC_K_UNIFORM) or lognormal
 * (mu 0, sigma 0.5) clipped to [0.1, 10] (SC_K_LOGNORMAL). Host memory, no device use.
 * Replaces nothing in the reference: it makes the benchmark's inputs. */
sc_status sc_generate_piece(int32_t nx, int32_t ny, int32_t nz, uint64_t seed, int32_t k_dist, uint8_t* state,
                            float* k);

/* Nodes and free nodes of a piece's lattice (host arithmetic, no device use). */
sc_status sc_grid_count(const sc_grid* g, int64_t* n_nodes, int64_t* n_parts);

/* Replaces `statics::bodies::motions` (statics/src/bodies.rs:429) for a voxel piece
 * with every bond alive and no node gone: writes 6 values per node (n_nodes x 6, the
 * reference's node order; held nodes zero) into `motions`, which holds `capacity`
 * doubles. `motions_on_device` says whether it is a device pointer. */
sc_status sc_solve_grid(sc_context* ctx, const sc_grid* g, const sc_options* opt, double* motions,
                        int64_t capacity, int32_t motions_on_device, sc_solve_info* info);

/* Many pieces at once: each its own hierarchy and its own CG, advanced together by
 * batched kernels in one CUDA graph per iteration. The pieces are solved in groups of at
 * most 5 M grid cells, taken largest first. motions[i] receives piece i's n_nodes x 6
 * values (host pointers); infos[i] its info. No counterpart in the reference, which
 * solves one structure per call. */
sc_status sc_solve_grid_batch(sc_context* ctx, int32_t n, const sc_grid* grids, const sc_options* opt,
                              double* const* motions, sc_solve_info* infos);

/* Compliance C = f.u of a piece and its gradient with respect to each cell's
 * stiffness: dC/dk_c = -2 U_c / k_c, U_c the strain energy of the cell's 60 bonds
 * (Bond::energy, statics/src/model.rs:132-136) at the solved motions. dc_dk has nx*ny*nz
 * entries (zero for cells that are not free). No counterpart in the reference: the
 * backward of `motions` for compliance. */
sc_status sc_compliance_grad(sc_context* ctx, const sc_grid* g, const sc_options* opt, double* compliance,
                             double* dc_dk, double* motions, int64_t capacity, sc_solve_info* info);

/* Level 0's operator on a piece: y = K x over the free nodes (n_parts x 6, part order),
 * the reference's Level::new + Level::apply (statics/src/bodies.rs:126-206), in FP64
 * (SC_FP64) or FP32 arithmetic (SC_MIXED), by the stencil the solve's iterations use
 * (brick order; x and y are permuted in and out). Host arrays. For parity checks. */
sc_status sc_grid_apply(sc_context* ctx, const sc_grid* g, int32_t precision, const double* x, double* y);
/* The same by the stencil `tile` selects (sc_options.tile): 0 the brick-ordered one
 * above, a power of two >= 32 the per-part stencil in part order (the setup's), 1 the
 * plane-pencil stencil, 2 the two-pass stencil. */
sc_status sc_grid_apply_tile(sc_context* ctx, const sc_grid* g, int32_t precision, int32_t tile, const double* x,
                             double* y);

/* After a solve: the body of each part at level `level` (the reference's `up` from
 * bodies_of, statics/src/bodies.rs:472-496), parts[level] entries; and piece-level
 * hierarchy sizes. For parity checks. */
sc_status sc_last_up(sc_context* ctx, int32_t level, int32_t* up, int64_t capacity);

/* ---------------------------------------------------------------------------
 * General lattices (any `Lattice`: the reference's level 0, or a gathered level).
 * Structure-of-arrays copy of statics/src/lattice.rs:61-71 and model.rs:92-111.
 * ------------------------------------------------------------------------- */
typedef struct sc_lattice {
    int32_t level;          /* Lattice::level */
    int64_t n_nodes;
    int64_t n_bonds;
    const double* x;        /* node centres, 3 per node */
    const uint8_t* held;    /* 1 if held */
    const int64_t* around;  /* the two cells each node lies between, 6 per node (lesser first) */
    const int64_t* bond_i;  /* bond ends */
    const int64_t* bond_j;
    const double* bond_p;   /* 3 per bond */
    const double* bond_n;   /* 3 per bond */
    const double* bond_a;
    const double* bond_d;
    const double* bond_e;   /* the bond's material's E */
    const double* bond_g;   /* the bond's material's G */
} sc_lattice;

/* Replaces `statics::bodies::motions` (statics/src/bodies.rs:429) for any lattice:
 * alive (n_bonds, may be NULL: all alive), gone (n_nodes, may be NULL: none gone),
 * loads (6 per node), motions out (6 per node; held and gone nodes zero). */
sc_status sc_motions(sc_context* ctx, const sc_lattice* lattice, const uint8_t* alive, const uint8_t* gone,
                     const double* loads, const sc_options* opt, double* motions, sc_solve_info* info);

/* ---------------------------------------------------------------------------
 * Measurement. No counterpart in the reference (which times whole calls with
 * Instant, statics/examples/statics.rs:135-140, 373-391).
 * ------------------------------------------------------------------------- */
enum {
    SC_FAM_STENCIL64 = 0, /* level-0 matrix-free stencil, FP64 */
    SC_FAM_STENCIL32 = 1, /* the same, FP32 */
    SC_FAM_SPMV64 = 2,    /* block-sparse operator products, FP64 */
    SC_FAM_SPMV32 = 3,
    SC_FAM_TRANSFER64 = 4,/* restriction and prolongation */
    SC_FAM_TRANSFER32 = 5,
    SC_FAM_SMOOTH64 = 6,  /* block-Jacobi steps */
    SC_FAM_SMOOTH32 = 7,
    SC_FAM_TOP = 8,       /* dense top-level solves */
    SC_FAM_COUNT = 9
};
/* Bracket every launch of the families in `mask` (bit f = family f) with CUDA events
 * on the context's stream, and reset the tallies. mask 0 turns it off. */
sc_status sc_profile(sc_context* ctx, uint32_t mask);
/* Tallies since sc_profile: launches, summed device milliseconds and algorithmic bytes
 * (what the kernels must read and write: vectors, blocks, cell table). */
sc_status sc_profile_read(sc_context* ctx, int32_t family, int64_t* launches, double* ms, double* bytes);
/* Kernels this library has launched in this process. */
int64_t sc_launches(void);
/* The CUDA stream (cudaStream_t) the context launches on. */
sc_status sc_context_stream(sc_context* ctx, void** stream);

/* ---------------------------------------------------------------------------
 * The callers of motions: the structure standing, and settling.
 * ------------------------------------------------------------------------- */
/* Per node its mass (Node::m) and per bond its material's strengths (Mat::ft, fc, fs),
 * statics/src/model.rs:43-51, 92-111: what the loads and the bonds' use need beyond
 * sc_lattice. Host arrays. */
typedef struct sc_strength {
    const double* m;   /* n_nodes */
    const double* ft;  /* n_bonds: tensile */
    const double* fc;  /* n_bonds: compressive */
    const double* fs;  /* n_bonds: shear */
} sc_strength;

/* Replaces statics::bodies::used_standing (statics/src/bodies.rs:550-554): every bond
 * alive, the nodes not joined to a held node through bonds gone, each node's weight
 * (m * 9.81 down y, bodies.rs:408) as its load; writes each bond's used fraction of its
 * strength (Bond::used, model.rs:123-129; 0 for a bond with a gone end) into used
 * (n_bonds, host). */
sc_status sc_used_standing(sc_context* ctx, const sc_lattice* lattice, const sc_strength* strength,
                           const sc_options* opt, double* used, sc_solve_info* info);

typedef struct sc_settle_info {
    double fell;     /* the fallen fraction of the free mass (Outcome::fallen) */
    int64_t rounds;  /* solves run */
    double work;     /* the reference's Work counter over all rounds */
    int32_t status;  /* the worst sc_status of the rounds' solves */
    int32_t pad;
} sc_settle_info;

/* Replaces statics::bodies::settle (statics/src/bodies.rs:511-541): rounds of motions under
 * the weights, each breaking every beam (4 consecutive bonds) with an alive bond used
 * beyond 1 whose ends stand, and dropping the nodes no longer joined to a held node,
 * until a round breaks nothing. gone: n_nodes bytes (host), 1 for a fallen node. */
sc_status sc_settle(sc_context* ctx, const sc_lattice* lattice, const sc_strength* strength, const sc_options* opt,
                    uint8_t* gone, sc_settle_info* out);

/* Replaces statics::bodies::as_generated (statics/src/bodies.rs:611-625): the strength a
 * lattice needs to stand as its world was generated, MARGIN = 2 times (bodies.rs:605).
 * Every beam of `generated` (bonds keyed by the cells their two end nodes lie between,
 * `around`, the lesser pair first) needs the most of its strength any of its bonds uses
 * standing (sc_used_standing of `generated`, solved on the device); each bond of
 * `lattice` on such a beam becomes max(2 * that, 1) times as strong (Mat::stronger,
 * statics/src/model.rs:71-73), the others keep theirs. The reference changes the
 * lattice's materials in place; here the new strengths go to ft, fc, fs (n_bonds of
 * `lattice`, host) and the inputs stay as they are. */
sc_status sc_as_generated(sc_context* ctx, const sc_lattice* lattice, const sc_strength* strength,
                          const sc_lattice* generated, const sc_strength* generated_strength,
                          const sc_options* opt, double* ft, double* fc, double* fs);

/* ---------------------------------------------------------------------------
 * Coarser levels measured from finer ones: statics::gather (statics/src/gather.rs).
 *
 * A material's values as the gather uses them (statics/src/model.rs:43-51: E, G and the
 * tensile, compressive and shear strengths). Nodes name their material by its index in a
 * caller's table; a material is its index (the reference tells materials by name).
 * ------------------------------------------------------------------------- */
typedef struct sc_material {
    double e, g, ft, fc, fs;
} sc_material;

typedef struct sc_gathered sc_gathered;

/* Replaces statics::gather::gathered (statics/src/gather.rs:193-195; against_full != 0)
 * and measured(fine, false) (gather.rs:230-395; against_full == 0): the next level up of
 * `fine`, each coarse cell's beams measured from its matter (each face a rigid handle
 * moved alone along each axis, the free parts at rest, the handles' reactions fitted by
 * non-negative least squares with beams between faces, each beam's strength from the
 * finer bonds' use when it is pulled alone) and its weight shared out on its faces.
 * `strength` gives each node's mass and each bond's strengths; node_mat (n_nodes) each
 * node's material in `materials` (n_materials entries). Host arrays. With a context the
 * cells are measured on its device, one thread block a cell; with ctx NULL on the host's
 * cores (threads: 0 = all); the indexing around them runs on the host either way. The
 * result is the reference's bit for bit: nodes in the order of their face keys, four
 * bonds a beam. *out receives a handle to read with
 * sc_gathered_read and free with sc_gathered_free; *n_nodes, *n_bonds its sizes.
 * SC_BAD_INPUT for a bond whose ends share no cell (the reference panics), indexes out of
 * range, non-finite or non-positive bond or material values, or (on the device) a coarse
 * cell with more than 12 finer parts, 6 faces or 480 finer bonds, which no lattice that
 * build or a gather makes has. */
sc_status sc_gather(sc_context* ctx, const sc_lattice* fine, const sc_strength* strength, const int32_t* node_mat,
                    const sc_material* materials, int32_t n_materials, int32_t against_full, int32_t threads,
                    sc_gathered** out, int64_t* n_nodes, int64_t* n_bonds);
/* Copies a gathered level out; any pointer may be NULL. Per node: x (3), m, held, around
 * (6: the two coarse sites it lies between, lesser first), mat (index in the table). Per
 * bond: ends, material (its cell's, an index in the table), p (3), n (3), a, d, E, G and
 * the strengths ft, fc, fs (the cell's material made stronger by the beam's measured
 * factor, Mat::stronger, model.rs:71-73). */
sc_status sc_gathered_read(const sc_gathered* g, int32_t* level, double* x, double* m, uint8_t* held,
                           int64_t* around, int32_t* mat, int64_t* bond_i, int64_t* bond_j, int32_t* bond_mat,
                           double* bond_p,
                           double* bond_n, double* bond_a, double* bond_d, double* bond_e, double* bond_g,
                           double* ft, double* fc, double* fs);
void sc_gathered_free(sc_gathered* g);
/* gather.rs:203-226: a full cell of `m` measured a level up, per class (180°, 90°):
 * out[2 k] its beams' section over the spacing squared, out[2 k + 1] their strength over
 * the material's. The calibration sc_gather applies when against_full != 0. */
sc_status sc_gather_full(const sc_material* m, double* out);

/* ---------------------------------------------------------------------------
 * Compliance without device allocation. No counterpart in the reference.
 *
 * For callers that must not have the library allocate device memory: an engine that
 * owns the GPU's memory through its own arena, or a per-frame loop that cannot afford
 * cudaMalloc's implicit device synchronisation. It computes C = f . u (n_values doubles each, device pointers; e.g.
 * the loads and the motions of sc_solve_grid, node order) into *compliance (a device
 * pointer), on `stream` (a cudaStream_t; NULL = the legacy default stream), with a
 * deterministic two-stage sum (fixed 8192-value chunks, a tree in each chunk, the chunks
 * in a fixed order; equal to the solver's dot products up to rounding), and allocates
 * nothing: its partial sums live in one 512 KB array inside the library, reserved on
 * every GPU that loads it until the process exits. At most SC_NOALLOC_MAX_VALUES values
 * (SC_BAD_INPUT beyond). Every call looks that array's address up in the CUDA context
 * current on the calling thread (the address follows the context, not the device
 * number), so call it with the device of the pointers current. Every call shares the
 * array: calls whose kernels may overlap on the GPU race and can return wrong sums, so
 * order them on one stream. Asynchronous: *compliance is ready when `stream` reaches
 * this point. SC_CUDA when the lookup or a launch fails (an error the caller left
 * pending is neither consumed nor reported).
 * ------------------------------------------------------------------------- */
#define SC_NOALLOC_MAX_VALUES (8192LL * 65536LL)
sc_status sc_compliance_noalloc(const double* loads, const double* motions, int64_t n_values, double* compliance,
                                void* stream);

/* ---------------------------------------------------------------------------
 * The engine's solver, mechanics::solve::Solver (mechanics/src/solve.rs:356-538).
 *
 * The system: n unknowns with their octree site (3 int64), position `at` (3 doubles)
 * and 3x3 diagonal block (9 doubles, row-major); npairs pairs (pi, pj, 3x3 block pb:
 * pb in row pi, column pj, its transpose in row pj, column pi; a pair twice adds). All
 * host arrays. Makes the levels on the device (Solver::new(system, size): rigid aggregates
 * by octree cell, their Galerkin blocks, Cholesky inverses with dropped pivots, a direct top) and
 * solves by PCG from x (3 n doubles, in/out) until r' P r <= tol^2 b' P b, P the V-cycle
 * preconditioner (Solver::solve). *rounds: the rounds taken (at most 300), or -1 where
 * the levels do not fit the system (not positive; the reference's None). *levels: the
 * coarse levels made.
 * ------------------------------------------------------------------------- */
/* A voxel piece at rest as such a system (mechanics/src/lib.rs:375-423, 638-676): each free
 * cell (state 1; 0 empty, 2 held; x-major) an 8-node element of the unit cube's
 * stiffness (Poisson's ratio 0.3) times e[cell] h, welded to its free neighbours; corners
 * touching a held cell held; diagonal m I + (dt^2 + 0.3 dt) E h K_aa (m: `mass` / 8 from
 * each cell at a corner); b = m (0, -9.81 dt, 0). Call with sites = NULL for the counts
 * (*n, *npairs), then with arrays of those sizes (*n, *npairs set to their capacity). */
sc_status sc_mech_voxel_system(const uint8_t* state, const float* e, int32_t nx, int32_t ny, int32_t nz, double h,
                               double dt, double mass, int64_t* n, int64_t* npairs, int64_t* sites, double* at,
                               double* diag, uint32_t* pi, uint32_t* pj, double* pb, double* b);
/* Only the levels (Solver::new, host code, no device): *nlevels coarse levels, the parts
 * of each (sizes, up to max_levels), and the smoother steps: steps[0] the nodes', steps[l
 * + 1] coarse level l's (0 for the direct top); steps holds max_levels + 1 values.
 * SC_BAD_INPUT when steps is NULL, or sizes is NULL with max_levels > 0. */
sc_status sc_mech_levels(int64_t n, const int64_t* sites, const double* at, const double* diag, int64_t npairs,
                         const uint32_t* pi, const uint32_t* pj, const double* pb, double size, int32_t max_levels,
                         int64_t* sizes, double* steps, int32_t* nlevels);
/* The same levels made on the context's device, as sc_mech_solve makes them (the same
 * parts and steps, bit for bit, as sc_mech_levels): Solver::new (solve.rs:361-386). */
sc_status sc_mech_levels_on(sc_context* ctx, int64_t n, const int64_t* sites, const double* at, const double* diag,
                            int64_t npairs, const uint32_t* pi, const uint32_t* pj, const double* pb, double size,
                            int32_t max_levels, int64_t* sizes, double* steps, int32_t* nlevels);
sc_status sc_mech_solve(sc_context* ctx, int64_t n, const int64_t* sites, const double* at, const double* diag,
                        int64_t npairs, const uint32_t* pi, const uint32_t* pj, const double* pb, const double* b,
                        double* x, double tol, double size, int32_t* rounds, int32_t* levels);

#ifdef __cplusplus
}
#endif
#endif /* STATICS_CUDA_H */
