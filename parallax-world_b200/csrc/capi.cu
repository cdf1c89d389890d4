// The C ABI (include/statics_cuda.h): validation, one solve per call, statuses instead
// of exceptions, results scattered back to the reference's node order.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "kernels.cuh"
#include "template_gen.cuh"

struct sc_gathered {
    sc::Gathered g;
};

struct sc_context {
    sc::Context c;
};

namespace sc {

PhaseTimer::PhaseTimer(Context& c) : ctx(c) {
    const char* e = std::getenv("SC_TIMING");
    on = e && e[0] == '1';
    t = std::chrono::steady_clock::now();
    alloc_ms0 = c.mem.alloc_ms;
    allocs0 = c.mem.allocs;
}

void PhaseTimer::note(const char* fmt, ...) {
    if (!on) return;
    va_list ap;
    va_start(ap, fmt);
    std::fprintf(stderr, "[sc] ");
    std::vfprintf(stderr, fmt, ap);
    std::fprintf(stderr, "\n");
    va_end(ap);
}

void PhaseTimer::mark(const char* phase) {
    if (!on) return;
    SC_CK(cudaStreamSynchronize(ctx.stream));
    auto now = std::chrono::steady_clock::now();
    cudaMemPool_t pool;
    uint64_t reserved = 0;
    if (cudaDeviceGetDefaultMemPool(&pool, ctx.device) == cudaSuccess)
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
    std::fprintf(stderr, "[sc] %-22s %9.2f ms  alloc %8.2f ms (%lld)  held %6.2f GB  peak %6.2f GB  pool %6.2f GB\n",
                 phase, std::chrono::duration<double, std::milli>(now - t).count(), ctx.mem.alloc_ms - alloc_ms0,
                 (long long)(ctx.mem.allocs - allocs0), ctx.mem.now / 1e9, ctx.mem.peak / 1e9, reserved / 1e9);
    t = now;
    alloc_ms0 = ctx.mem.alloc_ms;
    allocs0 = ctx.mem.allocs;
}

std::atomic<int64_t> g_launches{0};

cudaEvent_t Profiler::get() {
    if (!pool.empty()) {
        cudaEvent_t e = pool.back();
        pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    SC_CK(cudaEventCreate(&e));
    return e;
}

void Profiler::flush() {
    if (pending.empty()) return;
    SC_CK(cudaEventSynchronize(pending.back().b));
    for (auto& p : pending) {
        float t = 0;
        SC_CK(cudaEventElapsedTime(&t, p.a, p.b));
        launches[p.fam] += 1;
        ms[p.fam] += t;
        bytes[p.fam] += p.bytes;
        pool.push_back(p.a);
        pool.push_back(p.b);
    }
    pending.clear();
}

void Profiler::reset() {
    flush();
    for (int f = 0; f < SC_FAM_COUNT; f++) {
        launches[f] = 0;
        ms[f] = 0;
        bytes[f] = 0;
    }
}

Profiler::~Profiler() {
    for (auto& p : pending) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    for (auto e : pool) cudaEventDestroy(e);
}

ProfScope::ProfScope(Context& ctx, int family, double algorithmic_bytes) {
    if (!(ctx.prof.mask & (1u << family))) return;
    c = &ctx;
    fam = family;
    bytes = algorithmic_bytes;
    a = ctx.prof.get();
    SC_CK(cudaEventRecord(a, ctx.stream));
}

ProfScope::~ProfScope() {
    if (!c) return;
    cudaEvent_t b = c->prof.get();
    cudaEventRecord(b, c->stream);
    c->prof.pending.push_back({fam, a, b, bytes});
    if (c->prof.pending.size() > 4096) c->prof.flush();
}

void* Context::cub_scratch(size_t bytes) {
    if (bytes > cub_bytes) {
        if (cub_tmp) cudaFreeAsync(cub_tmp, stream);
        size_t want = std::max(bytes, cub_bytes * 2);
        SC_CK(cudaMallocAsync(&cub_tmp, want, stream));
        cub_bytes = want;
    }
    return cub_tmp;
}

int32_t* Context::pinned_i32() {
    if (!pinned) SC_CK(cudaMallocHost((void**)&pinned, 16));
    return pinned;
}

Context::~Context() {
    last.reset();
    partial.release();
    scal.release();
    if (cub_tmp) cudaFreeAsync(cub_tmp, stream);
    mem.trim(stream);
    if (stream) {
        cudaStreamSynchronize(stream);
        cudaStreamDestroy(stream);
    }
    if (pinned) cudaFreeHost(pinned);
}

namespace {

__global__ void k_scatter(int64_t n, const int32_t* __restrict__ piece, const int64_t* __restrict__ node_start,
                          const int32_t* __restrict__ part_node, const double* __restrict__ x, double* __restrict__ out) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    int64_t v = node_start[piece[k]] + part_node[k];
    for (int q = 0; q < 6; q++) out[6 * v + q] = x[6 * k + q];
}

// dC/dk = -2 U / k per free cell, written at the cell's flat index
__global__ void k_grad(int64_t nc, const int4* __restrict__ cell, const int64_t* __restrict__ cell_flat,
                       const double* __restrict__ energy, double* __restrict__ grad) {
    int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= nc) return;
    double k = (double)__int_as_float(cell[2 * c + 1].z);
    grad[cell_flat[c]] = -2.0 * energy[c] / k;
}

template <class F>
sc_status guarded(sc_context* ctx, F&& f) {
    if (!ctx) return SC_BAD_INPUT;
    try {
        SC_CK(cudaSetDevice(ctx->c.device));
        f();
        ctx->c.last_error.clear();
        return SC_OK;
    } catch (const Error& e) {
        ctx->c.last_error = e.what();
        if (e.status == SC_CUDA) cudaGetLastError();
        return e.status;
    } catch (const std::bad_alloc&) {
        ctx->c.last_error = "host allocation failed";
        return SC_CUDA;
    } catch (const std::exception& e) {
        ctx->c.last_error = e.what();
        return SC_CUDA;
    }
}

void check_grid(const sc_grid& g) {
    require(g.nx > 0 && g.ny > 0 && g.nz > 0, SC_BAD_INPUT, "grid dimensions must be positive");
    require((int64_t)g.nx * g.ny * g.nz < (int64_t)1 << 31, SC_BAD_INPUT, "grid too large");
    require(g.state && g.k, SC_BAD_INPUT, "grid state and k are required");
    require(std::fabs(g.g_over_e - TPL_G_OVER_E) < 1e-12, SC_BAD_INPUT,
            "voxel pieces take G/E = 0.4 (every reference material's); use sc_motions for others");
    require(g.rho > 0 && std::isfinite(g.rho), SC_BAD_INPUT, "rho must be positive");
}

void check_options(const sc_options& o) {
    require(o.tol >= 0 && std::isfinite(o.tol), SC_BAD_INPUT, "tol must be finite and non-negative");
    require(o.max_iter >= 0, SC_BAD_INPUT, "max_iter must be non-negative");
    require(o.few >= 1, SC_BAD_INPUT, "few must be at least 1");
    require(o.precision == SC_FP64 || o.precision == SC_MIXED || o.precision == SC_MIXED_FP32_KRYLOV, SC_BAD_INPUT,
            "unknown precision");
    require(o.sweeps >= 1 && o.sweeps <= 8, SC_BAD_INPUT, "sweeps must be 1 to 8");
    require(o.tile == 0 || o.tile == 1 || o.tile == 2 || (o.tile >= 32 && o.tile <= (1 << 20) && (o.tile & (o.tile - 1)) == 0), SC_BAD_INPUT,
            "tile must be 0, 1, 2 or a power of two from 32");
}

// The reference's Work for a solve of one piece: parts + pairs per level apply
// (bodies.rs:194): the CG's level-0 apply each iteration, and two applies per level
// above the top in each V-cycle (one before the loop, one per iteration).
double work_of(const Batch& b, int piece, int64_t iters) {
    double w = 0;
    const Level& L0 = b.levels[0];
    auto parts = [&](const Level& L) { return (double)(L.pstart[piece + 1] - L.pstart[piece]); };
    (void)L0;
    int nl = b.piece_levels[piece];
    // pairs of a piece's level: (blocks - parts) / 2 over its rows
    auto pairs = [&](int l) -> double {
        const Level& L = b.levels[l];
        if (b.npieces == 1) return (double)(L.nnzb - L.n) / 2.0;
        return 0.0;  // batched pieces: not tracked
    };
    w += (double)iters * (parts(b.levels[0]) + pairs(0));
    for (int l = 0; l + 1 < nl; l++) w += (double)(iters + 1) * 2.0 * (parts(b.levels[l]) + pairs(l));
    return w;
}

void fill_info(const Batch& b, int piece, const SolveStats& st, sc_solve_info* info, double solve_ms, int64_t peak) {
    if (!info) return;
    std::memset(info, 0, sizeof(*info));
    info->iterations = st.iterations.empty() ? 0 : st.iterations[piece];
    info->refinements = st.refinements.empty() ? 0 : st.refinements[piece];
    int nl = b.piece_levels.empty() ? 1 : b.piece_levels[piece];
    info->levels = nl;
    for (int l = 0; l < nl && l < SC_MAX_LEVELS; l++) {
        const Level& L = b.levels[l];
        info->parts[l] = L.pstart[piece + 1] - L.pstart[piece];
        info->blocks[l] = b.npieces == 1 ? L.nnzb : 0;
    }
    info->residual = st.residual.empty() ? 0 : st.residual[piece];
    info->residual_floor = st.floor.empty() ? 0 : st.floor[piece];
    info->work = work_of(b, piece, info->iterations);
    info->setup_ms = b.setup_ms;
    info->solve_ms = solve_ms;
    info->n_nodes = b.node_count[piece];
    info->n_parts = b.levels[0].pstart[piece + 1] - b.levels[0].pstart[piece];
    info->peak_bytes = peak;
    info->status = b.piece_status.empty() ? 0 : b.piece_status[piece];
}

void read_steps(Context& ctx, const Batch& b, int piece, sc_solve_info* info) {
    if (!info) return;
    for (int l = 0; l < info->levels && l < SC_MAX_LEVELS; l++) {
        double s = 0;
        SC_CK(cudaMemcpyAsync(&s, b.levels[l].step.get() + piece, sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
        SC_CK(cudaStreamSynchronize(ctx.stream));
        info->steps[l] = s;
    }
}

// Solves a batch already at level 0; returns per-piece statuses.
sc_status solve_batch(Context& ctx, Batch& b, const sc_options& opt, DBuf<double>& x, SolveStats& st, double& solve_ms) {
    b.sweeps = opt.sweeps;
    build_hierarchy(ctx, b, opt);
    PhaseTimer pt(ctx);
    if (b.levels[0].matrix_free && b.grid.use_bricks) {
        // the iterations run in brick order (brick.cu); its layout counts as setup
        auto tb = std::chrono::steady_clock::now();
        bricks_build(ctx, b);
        bricks_enter(ctx, b);
        SC_CK(cudaStreamSynchronize(ctx.stream));
        b.setup_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tb).count();
        pt.mark("brick layout");
    }
    auto t0 = std::chrono::steady_clock::now();
    if (opt.precision == SC_MIXED)
        pcg_fp32_cycle(ctx, b, opt, x, st);
    else if (opt.precision == SC_MIXED_FP32_KRYLOV)
        pcg_mixed(ctx, b, opt, x, st);
    else
        pcg_fp64(ctx, b, opt, x, st);
    bricks_leave(ctx, b, &x);  // x back in the reference's part order
    SC_CK(cudaStreamSynchronize(ctx.stream));
    solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    pt.mark("conjugate gradients");
    b.piece_status = b.status_d.to_host();
    int worst = 0;
    for (int s : b.piece_status) worst = std::max(worst, s);
    return (sc_status)worst;
}

}  // namespace
}  // namespace sc

namespace sc {

void check_lattice(const sc_lattice& lat) {
    require(lat.n_nodes > 0 && lat.n_bonds >= 0, SC_BAD_INPUT, "empty lattice");
    require(lat.x && lat.held && lat.around, SC_BAD_INPUT, "node arrays are required");
    require(lat.n_bonds == 0 || (lat.bond_i && lat.bond_j && lat.bond_p && lat.bond_n && lat.bond_a && lat.bond_d &&
                                 lat.bond_e && lat.bond_g),
            SC_BAD_INPUT, "bond arrays are required");
    for (int64_t b = 0; b < lat.n_bonds; b++)
        require(lat.bond_i[b] >= 0 && lat.bond_i[b] < lat.n_nodes && lat.bond_j[b] >= 0 &&
                    lat.bond_j[b] < lat.n_nodes,
                SC_BAD_INPUT, "bond end out of range");
}

// motions (bodies.rs:429-468) of a lattice into out (6 per node, device), zeros for held
// and gone nodes; returns the solve's status (the hierarchy stays as ctx.last)
sc_status lattice_motions(Context& c, const sc_lattice& lat, const uint8_t* alive, const uint8_t* gone,
                          const double* loads, const sc_options& opt, double* out, sc_solve_info* info) {
    auto b = std::make_unique<Batch>();
    c.last.reset();  // the previous solve's hierarchy is not kept through this one
    // Every node held or gone: nothing to solve, every motion zero (the reference's CG
    // stops at once on an empty right-hand side, bodies.rs:350-352).
    bool any_part = false;
    for (int64_t v = 0; v < lat.n_nodes && !any_part; v++) any_part = !lat.held[v] && !(gone && gone[v]);
    if (!any_part) {
        SC_CK(cudaMemsetAsync(out, 0, 6 * lat.n_nodes * sizeof(double), c.stream));
        SC_CK(cudaStreamSynchronize(c.stream));
        if (info) {
            std::memset(info, 0, sizeof(*info));
            info->levels = 0;
            info->n_nodes = lat.n_nodes;
        }
        return SC_OK;
    }
    SC_CK(cudaStreamSynchronize(c.stream));
    c.mem.peak = c.mem.now;
    lattice_level0(c, *b, lat, alive, gone, loads);
    DBuf<double> x;
    SolveStats st;
    double solve_ms = 0;
    sc_status solve_status = solve_batch(c, *b, opt, x, st, solve_ms);
    SC_CK(cudaMemsetAsync(out, 0, 6 * lat.n_nodes * sizeof(double), c.stream));
    const Level& L = b->levels[0];
    k_scatter<<<grid_for(L.n, 256), 256, 0, c.stream>>>(L.n, L.piece.get(), b->node_start.get(), b->part_node.get(),
                                                         x.get(), out);
    SC_LAUNCH_CK();
    SC_CK(cudaStreamSynchronize(c.stream));
    fill_info(*b, 0, st, info, solve_ms, c.mem.peak);
    read_steps(c, *b, 0, info);
    c.last = std::move(b);
    return solve_status;
}

}  // namespace sc

using namespace sc;

extern "C" {

void sc_default_options(sc_options* o) {
    if (!o) return;
    o->tol = 1e-6;
    o->max_iter = 100000;
    o->few = 64;
    o->precision = SC_FP64;
    o->sweeps = 1;
    o->inner_tol = 1e-4;
    o->timeout_ms = 0;
    o->tile = 0;
    o->reserved = 0;
}

const char* sc_status_string(sc_status s) {
    switch (s) {
        case SC_OK: return "ok";
        case SC_MAXITER: return "iteration cap reached";
        case SC_BREAKDOWN: return "conjugate gradients broke down (p'Ap <= 0 or NaN)";
        case SC_NOT_SPD: return "top level not positive definite";
        case SC_BAD_INPUT: return "bad input";
        case SC_TIMEOUT: return "time limit reached";
        case SC_CUDA: return "CUDA error";
        case SC_NO_DEVICE: return "no sm_100 device";
    }
    return "unknown status";
}

sc_status sc_create(int32_t device, sc_context** out) {
    if (!out) return SC_BAD_INPUT;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        return SC_NO_DEVICE;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) return SC_NO_DEVICE;
    auto* ctx = new sc_context;
    ctx->c.device = device;
    sc_status s = guarded(ctx, [&] {
        SC_CK(cudaStreamCreateWithFlags(&ctx->c.stream, cudaStreamNonBlocking));
        cudaMemPool_t pool;
        SC_CK(cudaDeviceGetDefaultMemPool(&pool, device));
        uint64_t thr = UINT64_MAX;
        SC_CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
        size_t free_b = 0, total_b = 0;
        SC_CK(cudaSetDevice(device));
        SC_CK(cudaMemGetInfo(&free_b, &total_b));
        ctx->c.mem.cap = total_b / 2;
    });
    if (s != SC_OK) {
        delete ctx;
        return s;
    }
    *out = ctx;
    return SC_OK;
}

void sc_destroy(sc_context* ctx) { delete ctx; }

const char* sc_last_error(const sc_context* ctx) { return ctx ? ctx->c.last_error.c_str() : "no context"; }

sc_status sc_grid_count(const sc_grid* g, int64_t* n_nodes, int64_t* n_parts) {
    if (!g || !n_nodes || !n_parts || g->on_device) return SC_BAD_INPUT;
    if (g->nx <= 0 || g->ny <= 0 || g->nz <= 0 || !g->state) return SC_BAD_INPUT;
    // the reference's node creation (lattice.rs:124-163): a free cell's + faces are new, a
    // - face is new unless the cell before it on that axis is free; a node is held when
    // its other cell is held. Rows along z, the four neighbouring rows by pointer.
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const int64_t syz = (int64_t)ny * nz;
    int64_t nodes = 0, held = 0;
    auto face = [&](int other, bool plus) {
        if (plus || other != SC_CELL_FREE) {
            nodes++;
            held += other == SC_CELL_HELD;
        }
    };
    for (int x = 0; x < nx; x++)
        for (int y = 0; y < ny; y++) {
            const uint8_t* row = g->state + ((int64_t)x * ny + y) * nz;
            const uint8_t* xm = x > 0 ? row - syz : nullptr;
            const uint8_t* xp = x + 1 < nx ? row + syz : nullptr;
            const uint8_t* ym = y > 0 ? row - nz : nullptr;
            const uint8_t* yp = y + 1 < ny ? row + nz : nullptr;
            for (int z = 0; z < nz; z++) {
                if (row[z] != SC_CELL_FREE) continue;
                face(xm ? xm[z] : SC_CELL_EMPTY, false);
                face(xp ? xp[z] : SC_CELL_EMPTY, true);
                face(ym ? ym[z] : SC_CELL_EMPTY, false);
                face(yp ? yp[z] : SC_CELL_EMPTY, true);
                face(z > 0 ? row[z - 1] : SC_CELL_EMPTY, false);
                face(z + 1 < nz ? row[z + 1] : SC_CELL_EMPTY, true);
            }
        }
    *n_nodes = nodes;
    *n_parts = nodes - held;
    return SC_OK;
}

sc_status sc_mech_voxel_system(const uint8_t* state, const float* e, int32_t nx, int32_t ny, int32_t nz, double h,
                               double dt, double mass, int64_t* n, int64_t* npairs, int64_t* sites, double* at,
                               double* diag, uint32_t* pi, uint32_t* pj, double* pb, double* b) {
    if (!state || !e || nx <= 0 || ny <= 0 || nz <= 0 || !n || !npairs || !(h > 0.0) || !(dt > 0.0)) return SC_BAD_INPUT;
    try {
        std::vector<int64_t> s;
        std::vector<double> a, d, p, bb;
        std::vector<uint32_t> i, j;
        mech_voxel_system(state, e, nx, ny, nz, h, dt, mass, s, a, d, i, j, p, bb);
        const int64_t nn = (int64_t)s.size() / 3, mm = (int64_t)i.size();
        if (sites) {
            if (*n < nn || *npairs < mm || !at || !diag || !b || (mm > 0 && (!pi || !pj || !pb))) return SC_BAD_INPUT;
            std::copy(s.begin(), s.end(), sites);
            std::copy(a.begin(), a.end(), at);
            std::copy(d.begin(), d.end(), diag);
            std::copy(bb.begin(), bb.end(), b);
            std::copy(i.begin(), i.end(), pi);
            std::copy(j.begin(), j.end(), pj);
            std::copy(p.begin(), p.end(), pb);
        }
        *n = nn;
        *npairs = mm;
        return SC_OK;
    } catch (const std::exception&) {
        return SC_CUDA;
    }
}

sc_status sc_gather(sc_context* ctx, const sc_lattice* fine, const sc_strength* strength, const int32_t* node_mat,
                    const sc_material* materials, int32_t n_materials, int32_t against_full, int32_t threads,
                    sc_gathered** out, int64_t* n_nodes, int64_t* n_bonds) {
    if (!fine || !strength || !materials || !out || !n_nodes || !n_bonds || n_materials < 1) return SC_BAD_INPUT;
    const sc_lattice& L = *fine;
    const sc_strength& S = *strength;
    const int64_t nn = L.n_nodes, nb = L.n_bonds;
    if (nn < 0 || nb < 0 || L.level < 0 || L.level > 60) return SC_BAD_INPUT;
    if (nn > 0 && (!L.x || !L.held || !L.around || !S.m || !node_mat)) return SC_BAD_INPUT;
    if (nb > 0 && (!L.bond_i || !L.bond_j || !L.bond_p || !L.bond_n || !L.bond_a || !L.bond_d || !L.bond_e ||
                   !L.bond_g || !S.ft || !S.fc || !S.fs))
        return SC_BAD_INPUT;
    auto positive = [](double v) { return std::isfinite(v) && v > 0.0; };
    for (int32_t k = 0; k < n_materials; k++) {
        const sc_material& m = materials[k];
        if (!positive(m.e) || !positive(m.g) || !positive(m.ft) || !positive(m.fc) || !positive(m.fs))
            return SC_BAD_INPUT;
    }
    for (int64_t v = 0; v < nn; v++) {
        if (node_mat[v] < 0 || node_mat[v] >= n_materials || !std::isfinite(S.m[v])) return SC_BAD_INPUT;
        for (int q = 0; q < 3; q++)
            if (!std::isfinite(L.x[3 * v + q])) return SC_BAD_INPUT;
    }
    for (int64_t b = 0; b < nb; b++) {
        if (L.bond_i[b] < 0 || L.bond_i[b] >= nn || L.bond_j[b] < 0 || L.bond_j[b] >= nn) return SC_BAD_INPUT;
        for (int q = 0; q < 3; q++)
            if (!std::isfinite(L.bond_p[3 * b + q]) || !std::isfinite(L.bond_n[3 * b + q])) return SC_BAD_INPUT;
        if (!positive(L.bond_a[b]) || !positive(L.bond_d[b]) || !positive(L.bond_e[b]) || !positive(L.bond_g[b]) ||
            !positive(S.ft[b]) || !positive(S.fc[b]) || !positive(S.fs[b]))
            return SC_BAD_INPUT;
    }
    auto run = [&](sc::Context* dev) {
        auto g = std::make_unique<sc_gathered>();
        sc::gather_level(dev, L, S, node_mat, materials, n_materials, against_full != 0, threads, g->g);
        *n_nodes = (int64_t)g->g.m.size();
        *n_bonds = (int64_t)g->g.bi.size();
        *out = g.release();
    };
    if (ctx) return guarded(ctx, [&] { run(&ctx->c); });
    try {
        run(nullptr);
        return SC_OK;
    } catch (const sc::Error& e) {
        return e.status;
    } catch (const std::exception&) {
        return SC_CUDA;
    }
}

sc_status sc_gathered_read(const sc_gathered* gp, int32_t* level, double* x, double* m, uint8_t* held,
                           int64_t* around, int32_t* mat, int64_t* bond_i, int64_t* bond_j, int32_t* bond_mat,
                           double* bond_p,
                           double* bond_n, double* bond_a, double* bond_d, double* bond_e, double* bond_g,
                           double* ft, double* fc, double* fs) {
    if (!gp) return SC_BAD_INPUT;
    const sc::Gathered& g = gp->g;
    auto put = [](auto* dst, const auto& src) {
        if (dst && !src.empty()) std::memcpy(dst, src.data(), src.size() * sizeof(src[0]));
    };
    if (level) *level = g.level;
    put(x, g.x);
    put(m, g.m);
    put(held, g.held);
    put(around, g.around);
    put(mat, g.mat);
    put(bond_i, g.bi);
    put(bond_j, g.bj);
    put(bond_mat, g.bmat);
    put(bond_p, g.p);
    put(bond_n, g.n);
    put(bond_a, g.a);
    put(bond_d, g.d);
    put(bond_e, g.e);
    put(bond_g, g.g);
    put(ft, g.ft);
    put(fc, g.fc);
    put(fs, g.fs);
    return SC_OK;
}

void sc_gathered_free(sc_gathered* g) { delete g; }

sc_status sc_gather_full(const sc_material* m, double* out) {
    if (!m || !out) return SC_BAD_INPUT;
    auto positive = [](double v) { return std::isfinite(v) && v > 0.0; };
    if (!positive(m->e) || !positive(m->g) || !positive(m->ft) || !positive(m->fc) || !positive(m->fs))
        return SC_BAD_INPUT;
    try {
        sc::gather_full(*m, out);
        return SC_OK;
    } catch (const std::exception&) {
        return SC_CUDA;
    }
}

sc_status sc_mech_levels(int64_t n, const int64_t* sites, const double* at, const double* diag, int64_t npairs,
                         const uint32_t* pi, const uint32_t* pj, const double* pb, double size, int32_t max_levels,
                         int64_t* sizes, double* steps, int32_t* nlevels) {
    if (n <= 0 || npairs < 0 || !sites || !at || !diag || !nlevels || !(size > 0.0) || max_levels < 0) return SC_BAD_INPUT;
    if (!steps || (max_levels > 0 && !sizes)) return SC_BAD_INPUT;
    if (npairs > 0 && (!pi || !pj || !pb)) return SC_BAD_INPUT;
    for (int64_t p = 0; p < npairs; p++)
        if ((int64_t)pi[p] >= n || (int64_t)pj[p] >= n || pi[p] == pj[p]) return SC_BAD_INPUT;
    try {
        std::vector<int64_t> sz;
        std::vector<double> st;
        mech_levels(n, sites, at, diag, npairs, pi, pj, pb, size, sz, st);
        *nlevels = (int32_t)sz.size();
        for (size_t l = 0; l < sz.size() && (int32_t)l < max_levels; l++) sizes[l] = sz[l];
        for (size_t l = 0; l < st.size() && (int32_t)l <= max_levels; l++) steps[l] = st[l];
        return SC_OK;
    } catch (const std::exception&) {
        return SC_CUDA;
    }
}

sc_status sc_mech_levels_on(sc_context* ctx, int64_t n, const int64_t* sites, const double* at, const double* diag,
                            int64_t npairs, const uint32_t* pi, const uint32_t* pj, const double* pb, double size,
                            int32_t max_levels, int64_t* sizes, double* steps, int32_t* nlevels) {
    if (n <= 0 || npairs < 0 || !sites || !at || !diag || !nlevels || !(size > 0.0) || max_levels < 0) return SC_BAD_INPUT;
    if (!steps || (max_levels > 0 && !sizes)) return SC_BAD_INPUT;
    if (npairs > 0 && (!pi || !pj || !pb)) return SC_BAD_INPUT;
    for (int64_t p = 0; p < npairs; p++)
        if ((int64_t)pi[p] >= n || (int64_t)pj[p] >= n || pi[p] == pj[p]) return SC_BAD_INPUT;
    return guarded(ctx, [&] {
        std::vector<int64_t> sz;
        std::vector<double> st;
        mech_levels_device(ctx->c, n, sites, at, diag, npairs, pi, pj, pb, size, sz, st);
        *nlevels = (int32_t)sz.size();
        for (size_t l = 0; l < sz.size() && (int32_t)l < max_levels; l++) sizes[l] = sz[l];
        for (size_t l = 0; l < st.size() && (int32_t)l <= max_levels; l++) steps[l] = st[l];
    });
}

sc_status sc_mech_solve(sc_context* ctx, int64_t n, const int64_t* sites, const double* at, const double* diag,
                        int64_t npairs, const uint32_t* pi, const uint32_t* pj, const double* pb, const double* b,
                        double* x, double tol, double size, int32_t* rounds, int32_t* levels) {
    if (n < 0 || npairs < 0 || !rounds || !levels) return SC_BAD_INPUT;
    if (n > 0 && (!sites || !at || !diag || !b || !x)) return SC_BAD_INPUT;
    if (npairs > 0 && (!pi || !pj || !pb)) return SC_BAD_INPUT;
    if (!(tol > 0.0) || !(size > 0.0)) return SC_BAD_INPUT;
    for (int64_t p = 0; p < npairs; p++)
        if ((int64_t)pi[p] >= n || (int64_t)pj[p] >= n || pi[p] == pj[p]) return SC_BAD_INPUT;
    return guarded(ctx, [&] {
        ctx->c.last.reset();
        *levels = 0;
        *rounds = mech_solve(ctx->c, n, sites, at, diag, npairs, pi, pj, pb, b, x, tol, size, levels);
    });
}

sc_status sc_solve_grid(sc_context* ctx, const sc_grid* g, const sc_options* opt, double* motions, int64_t capacity,
                        int32_t motions_on_device, sc_solve_info* info) {
    if (!g || !opt || !motions) return SC_BAD_INPUT;
    sc_status solve_status = SC_OK;
    sc_status s = guarded(ctx, [&] {
        Context& c = ctx->c;
        check_grid(*g);
        check_options(*opt);
        auto b = std::make_unique<Batch>();
        c.last.reset();  // the previous solve's hierarchy is not kept through this one
        SC_CK(cudaStreamSynchronize(c.stream));
        c.mem.peak = c.mem.now;
        grid_level0(c, *b, {*g}, true, opt->tile);
        int64_t nodes = b->node_count[0];
        require(capacity >= 6 * nodes, SC_BAD_INPUT, "motions buffer holds fewer than 6 * n_nodes values");
        DBuf<double> x;
        SolveStats st;
        double solve_ms = 0;
        solve_status = solve_batch(c, *b, *opt, x, st, solve_ms);
        DBuf<double> out;
        double* dst = motions;
        if (!motions_on_device) {
            out.alloc(6 * nodes, c.stream, &c.mem);
            dst = out.get();
        }
        SC_CK(cudaMemsetAsync(dst, 0, 6 * nodes * sizeof(double), c.stream));
        const Level& L = b->levels[0];
        k_scatter<<<grid_for(L.n, 256), 256, 0, c.stream>>>(L.n, L.piece.get(), b->node_start.get(),
                                                             b->part_node.get(), x.get(), dst);
        SC_LAUNCH_CK();
        if (!motions_on_device) out.download(motions, 6 * nodes);
        SC_CK(cudaStreamSynchronize(c.stream));
        fill_info(*b, 0, st, info, solve_ms, c.mem.peak);
        read_steps(c, *b, 0, info);
        c.last = std::move(b);
    });
    return s != SC_OK ? s : solve_status;
}

// Pieces per batched solve are grouped so that a group's hierarchy setup stays within
// device memory: at most this many grid cells a group (a 128^3 piece is 2.1 M).
static const int64_t BATCH_CELLS = 5LL << 20;

sc_status sc_solve_grid_batch(sc_context* ctx, int32_t n, const sc_grid* grids, const sc_options* opt,
                              double* const* motions, sc_solve_info* infos) {
    if (n <= 0 || !grids || !opt || !motions) return SC_BAD_INPUT;
    sc_status solve_status = SC_OK;
    sc_status s = guarded(ctx, [&] {
        Context& c = ctx->c;
        check_options(*opt);
        std::vector<sc_grid> all(grids, grids + n);
        for (auto& g : all) check_grid(g);
        c.last.reset();  // the previous solve's hierarchy is not kept through this one
        SC_CK(cudaStreamSynchronize(c.stream));
        c.mem.peak = c.mem.now;
        // groups of pieces taken largest first (ties in the caller's order), so a group's
        // pieces are of one size class and the groups' setups of similar size
        std::vector<int> order(n);
        for (int i = 0; i < n; i++) order[i] = i;
        auto cells_of = [&](int i) { return (int64_t)all[i].nx * all[i].ny * all[i].nz; };
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cells_of(a) > cells_of(b); });
        int first = 0;
        while (first < n) {
            // the next group: the next pieces in that order up to the cell budget (at least one)
            int last = first;
            int64_t cells = 0;
            while (last < n) {
                int64_t gc = cells_of(order[last]);
                if (last > first && cells + gc > BATCH_CELLS) break;
                cells += gc;
                last++;
            }
            std::vector<sc_grid> gs;
            for (int q = first; q < last; q++) gs.push_back(all[order[q]]);
            int m = last - first;
            c.last.reset();
            auto b = std::make_unique<Batch>();
            grid_level0(c, *b, gs, true, opt->tile);
            DBuf<double> x;
            SolveStats st;
            double solve_ms = 0;
            sc_status gsts = solve_batch(c, *b, *opt, x, st, solve_ms);
            solve_status = std::max(solve_status, gsts);
            std::vector<int64_t> start(m + 1, 0);
            for (int p = 0; p < m; p++) start[p + 1] = start[p] + b->node_count[p];
            int64_t total = start[m];
            DBuf<double> out;
            out.alloc(6 * std::max<int64_t>(total, 1), c.stream, &c.mem);
            out.zero();
            const Level& L = b->levels[0];
            k_scatter<<<grid_for(L.n, 256), 256, 0, c.stream>>>(L.n, L.piece.get(), b->node_start.get(),
                                                                 b->part_node.get(), x.get(), out.get());
            SC_LAUNCH_CK();
            for (int p = 0; p < m; p++)
                if (motions[order[first + p]])
                    SC_CK(cudaMemcpyAsync(motions[order[first + p]], out.get() + 6 * start[p],
                                          6 * b->node_count[p] * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
            SC_CK(cudaStreamSynchronize(c.stream));
            if (infos) {
                for (int p = 0; p < m; p++) fill_info(*b, p, st, infos + order[first + p], solve_ms, c.mem.peak);
                for (size_t l = 0; l < b->levels.size() && l < SC_MAX_LEVELS; l++) {
                    std::vector<double> steps = b->levels[l].step.to_host();
                    for (int p = 0; p < m; p++)
                        if ((int)l < infos[order[first + p]].levels) infos[order[first + p]].steps[l] = steps[p];
                }
            }
            c.last = std::move(b);
            first = last;
        }
    });
    return s != SC_OK ? s : solve_status;
}

sc_status sc_compliance_grad(sc_context* ctx, const sc_grid* g, const sc_options* opt, double* compliance,
                             double* dc_dk, double* motions, int64_t capacity, sc_solve_info* info) {
    if (!g || !opt || !dc_dk) return SC_BAD_INPUT;
    sc_status solve_status = SC_OK;
    sc_status s = guarded(ctx, [&] {
        Context& c = ctx->c;
        check_grid(*g);
        check_options(*opt);
        require(!g->on_device, SC_BAD_INPUT, "sc_compliance_grad takes host grids");
        auto b = std::make_unique<Batch>();
        c.last.reset();  // the previous solve's hierarchy is not kept through this one
        SC_CK(cudaStreamSynchronize(c.stream));
        c.mem.peak = c.mem.now;
        grid_level0(c, *b, {*g}, true, opt->tile);
        int64_t nodes = b->node_count[0];
        require(!motions || capacity >= 6 * nodes, SC_BAD_INPUT, "motions buffer too small");
        DBuf<double> x;
        SolveStats st;
        double solve_ms = 0;
        solve_status = solve_batch(c, *b, *opt, x, st, solve_ms);
        const Level& L = b->levels[0];
        // C = f . u (FP64, deterministic per piece)
        DBuf<double> cc;
        cc.alloc(1, c.stream, &c.mem);
        seg_dot(c, L, b->loads.get(), x.get(), cc.get());
        double C = 0;
        cc.download(&C, 1);
        // the fused per-cell strain-energy gather, then dC/dk = -2 U / k
        const Grid0& G = b->grid;
        DBuf<double> energy, grad;
        energy.alloc(std::max<int64_t>(G.ncells, 1), c.stream, &c.mem);
        grid_cell_energy(c, *b, x.get(), energy.get());
        int64_t ncell = (int64_t)g->nx * g->ny * g->nz;
        grad.alloc(ncell, c.stream, &c.mem);
        grad.zero();
        k_grad<<<grid_for(G.ncells, 256), 256, 0, c.stream>>>(G.ncells, G.cell.get(), G.cell_flat.get(), energy.get(),
                                                               grad.get());
        SC_LAUNCH_CK();
        grad.download(dc_dk, ncell);
        if (motions) {
            DBuf<double> out;
            out.alloc(6 * nodes, c.stream, &c.mem);
            out.zero();
            k_scatter<<<grid_for(L.n, 256), 256, 0, c.stream>>>(L.n, L.piece.get(), b->node_start.get(),
                                                                 b->part_node.get(), x.get(), out.get());
            SC_LAUNCH_CK();
            out.download(motions, 6 * nodes);
        }
        SC_CK(cudaStreamSynchronize(c.stream));
        if (compliance) *compliance = C;
        fill_info(*b, 0, st, info, solve_ms, c.mem.peak);
        read_steps(c, *b, 0, info);
        c.last = std::move(b);
    });
    return s != SC_OK ? s : solve_status;
}

sc_status sc_grid_apply(sc_context* ctx, const sc_grid* g, int32_t precision, const double* xin, double* yout) {
    return sc_grid_apply_tile(ctx, g, precision, 0, xin, yout);
}

sc_status sc_grid_apply_tile(sc_context* ctx, const sc_grid* g, int32_t precision, int32_t tile, const double* xin,
                             double* yout) {
    if (!g || !xin || !yout) return SC_BAD_INPUT;
    return guarded(ctx, [&] {
        Context& c = ctx->c;
        check_grid(*g);
        sc_options o;
        sc_default_options(&o);
        o.tile = tile;
        check_options(o);
        Batch b;
        grid_level0(c, b, {*g}, false, tile);
        const Level& L = b.levels[0];
        int64_t n6 = 6 * L.n;
        DBuf<double> x, y;
        x.alloc(n6, c.stream, &c.mem);
        y.alloc(n6, c.stream, &c.mem);
        x.upload(xin, n6);
        if (b.grid.use_bricks) {  // the iterations' stencil: x into brick order, y back
            bricks_build(c, b);
            bricks_enter(c, b);
            DBuf<double> xb;
            xb.alloc(n6, c.stream, &c.mem);
            brick_permute<double>(c, b, x.get(), xb.get(), true);
            x = std::move(xb);
        }
        auto to_ref = [&](auto& v) {  // y from brick order into the reference's
            if (!b.grid.use_bricks) return;
            using V = typename std::remove_reference<decltype(*v.get())>::type;
            DBuf<V> o;
            o.alloc(n6, c.stream, &c.mem);
            brick_permute<V>(c, b, v.get(), o.get(), false);
            v = std::move(o);
        };
        if (precision == SC_MIXED) {
            DBuf<float> xf, yf;
            to_float(c, x, xf);
            yf.alloc(n6, c.stream, &c.mem);
            stencil_apply<float>(c, b, xf.get(), yf.get(), nullptr, nullptr);
            to_ref(yf);
            std::vector<float> h(n6);
            yf.download(h.data(), n6);
            SC_CK(cudaStreamSynchronize(c.stream));
            for (int64_t i = 0; i < n6; i++) yout[i] = h[i];
        } else {
            stencil_apply<double>(c, b, x.get(), y.get(), nullptr, nullptr);
            to_ref(y);
            y.download(yout, n6);
            SC_CK(cudaStreamSynchronize(c.stream));
        }
    });
}

sc_status sc_last_up(sc_context* ctx, int32_t level, int32_t* up, int64_t capacity) {
    if (!up) return SC_BAD_INPUT;
    return guarded(ctx, [&] {
        Context& c = ctx->c;
        require(c.last != nullptr, SC_BAD_INPUT, "no solve yet");
        require(level >= 0 && level + 1 < (int)c.last->levels.size(), SC_BAD_INPUT, "no such coarsening");
        const Level& L = c.last->levels[level];
        require(capacity >= L.n, SC_BAD_INPUT, "capacity below the level's parts");
        L.up.download(up, L.n);
        SC_CK(cudaStreamSynchronize(c.stream));
    });
}


sc_status sc_motions(sc_context* ctx, const sc_lattice* lat, const uint8_t* alive, const uint8_t* gone,
                     const double* loads, const sc_options* opt, double* motions, sc_solve_info* info) {
    if (!lat || !loads || !opt || !motions) return SC_BAD_INPUT;
    sc_status solve_status = SC_OK;
    sc_status s = guarded(ctx, [&] {
        Context& c = ctx->c;
        check_options(*opt);
        check_lattice(*lat);
        DBuf<double> out;
        out.alloc(6 * lat->n_nodes, c.stream, &c.mem);
        solve_status = lattice_motions(c, *lat, alive, gone, loads, *opt, out.get(), info);
        out.download(motions, 6 * lat->n_nodes);
        SC_CK(cudaStreamSynchronize(c.stream));
    });
    return s != SC_OK ? s : solve_status;
}

sc_status sc_used_standing(sc_context* ctx, const sc_lattice* lat, const sc_strength* str, const sc_options* opt,
                           double* used, sc_solve_info* info) {
    if (!lat || !str || !opt || !used) return SC_BAD_INPUT;
    sc_status solve_status = SC_OK;
    sc_status s = guarded(ctx, [&] {
        check_options(*opt);
        check_lattice(*lat);
        require(str->m && (lat->n_bonds == 0 || (str->ft && str->fc && str->fs)), SC_BAD_INPUT,
                "masses and strengths are required");
        solve_status = used_standing(ctx->c, *lat, *str, *opt, used, info);
    });
    return s != SC_OK ? s : solve_status;
}

sc_status sc_settle(sc_context* ctx, const sc_lattice* lat, const sc_strength* str, const sc_options* opt,
                    uint8_t* gone, sc_settle_info* out) {
    if (!lat || !str || !opt || !gone) return SC_BAD_INPUT;
    sc_status solve_status = SC_OK;
    sc_status s = guarded(ctx, [&] {
        check_options(*opt);
        check_lattice(*lat);
        require(str->m && (lat->n_bonds == 0 || (str->ft && str->fc && str->fs)), SC_BAD_INPUT,
                "masses and strengths are required");
        solve_status = settle(ctx->c, *lat, *str, *opt, gone, out);
    });
    return s != SC_OK ? s : solve_status;
}

sc_status sc_as_generated(sc_context* ctx, const sc_lattice* lat, const sc_strength* str, const sc_lattice* gen,
                          const sc_strength* gen_str, const sc_options* opt, double* ft, double* fc, double* fs) {
    if (!lat || !str || !gen || !gen_str || !opt || (lat->n_bonds > 0 && (!ft || !fc || !fs))) return SC_BAD_INPUT;
    sc_status solve_status = SC_OK;
    sc_status s = guarded(ctx, [&] {
        check_options(*opt);
        check_lattice(*lat);
        check_lattice(*gen);
        require(lat->n_bonds == 0 || (str->ft && str->fc && str->fs), SC_BAD_INPUT, "strengths are required");
        require(gen_str->m && (gen->n_bonds == 0 || (gen_str->ft && gen_str->fc && gen_str->fs)), SC_BAD_INPUT,
                "the generated lattice's masses and strengths are required");
        solve_status = as_generated(ctx->c, *lat, *str, *gen, *gen_str, *opt, ft, fc, fs);
    });
    return s != SC_OK ? s : solve_status;
}

sc_status sc_profile(sc_context* ctx, uint32_t mask) {
    return guarded(ctx, [&] {
        ctx->c.prof.reset();
        ctx->c.prof.mask = mask;
    });
}

sc_status sc_profile_read(sc_context* ctx, int32_t family, int64_t* launches, double* ms, double* bytes) {
    if (family < 0 || family >= SC_FAM_COUNT) return SC_BAD_INPUT;
    return guarded(ctx, [&] {
        ctx->c.prof.flush();
        if (launches) *launches = ctx->c.prof.launches[family];
        if (ms) *ms = ctx->c.prof.ms[family];
        if (bytes) *bytes = ctx->c.prof.bytes[family];
    });
}

int64_t sc_launches(void) { return g_launches.load(); }

sc_status sc_context_stream(sc_context* ctx, void** stream) {
    if (!ctx || !stream) return SC_BAD_INPUT;
    *stream = (void*)ctx->c.stream;
    return SC_OK;
}

}  // extern "C"
