// The callers of motions in the reference's statics crate, on the device: used_standing
// (statics/src/bodies.rs:550-554), each bond's used fraction of its strength with the
// structure standing, and settle (bodies.rs:511-541), rounds of solve -> break the
// overloaded beams -> drop what no longer reaches a held node, until nothing breaks.
// Each round's motions is the library's solve (lattice_motions); what happens around it
// -- which nodes still reach a held node (joined_to_held, bodies.rs:557-574), the bond
// forces of the motions (moved, bodies.rs:420-423, Bond::force, model.rs:115-119), their
// use of the bond's strength (Bond::used / Mat::used, model.rs:66-68, 123-129) and the
// breaking of whole beams -- runs in the kernels below.
#include <algorithm>
#include <array>
#include <cmath>
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "solver.cuh"

namespace sc {

namespace {

constexpr double GRAVITY = 9.81;  // statics/src/model.rs:38
constexpr int PER_BEAM = 4;       // bonds of one beam, consecutive (statics/src/lattice.rs:19)

struct BondsU {
    const int64_t *i, *j;
    const double *p, *n, *a, *d, *e, *g, *ft, *fc, *fs;
};

// the nodes joined to a held node through alive bonds: reach grows from the held nodes
// one bond at a time (a bond-parallel sweep; only ever sets flags, so sweeps can race)
__global__ void k_reach_init(int64_t n, const uint8_t* __restrict__ held, uint8_t* __restrict__ reach) {
    int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (v < n) reach[v] = held[v];
}
__global__ void k_reach_sweep(int64_t nb, const int64_t* __restrict__ bi, const int64_t* __restrict__ bj,
                              const uint8_t* __restrict__ alive, uint8_t* reach, int32_t* __restrict__ changed) {
    int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (b >= nb || !alive[b]) return;
    const int64_t i = bi[b], j = bj[b];
    const uint8_t ri = reach[i], rj = reach[j];
    if (ri != rj) {
        reach[i] = 1;
        reach[j] = 1;
        *changed = 1;
    }
}
__global__ void k_gone_update(int64_t n, const uint8_t* __restrict__ reach, uint8_t* __restrict__ gone) {
    int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (v < n && !reach[v]) gone[v] = 1;
}

__device__ __forceinline__ double fmax_r(double a, double b) { return fmax(a, b); }

// each bond's force from the motions u (6 per node) and its use of its strength; zero for
// a dead bond or one with a gone end (bodies.rs:407-417, 544-546)
__global__ void k_bond_used(int64_t nb, BondsU B, const double* __restrict__ x, const double* __restrict__ u,
                            const uint8_t* __restrict__ alive, const uint8_t* __restrict__ gone,
                            double* __restrict__ used) {
    int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const int64_t i = B.i[b], j = B.j[b];
    double f[3] = {0.0, 0.0, 0.0};
    if (alive[b] && !gone[i] && !gone[j]) {
        // at(v) = translation of v + rotation of v x (bond point - node position)
        double at[2][3];
        for (int s = 0; s < 2; s++) {
            const int64_t v = s ? j : i;
            const double r0 = B.p[3 * b] - x[3 * v], r1 = B.p[3 * b + 1] - x[3 * v + 1],
                         r2 = B.p[3 * b + 2] - x[3 * v + 2];
            const double* w = u + 6 * v + 3;
            at[s][0] = u[6 * v] + (w[1] * r2 - w[2] * r1);
            at[s][1] = u[6 * v + 1] + (w[2] * r0 - w[0] * r2);
            at[s][2] = u[6 * v + 2] + (w[0] * r1 - w[1] * r0);
        }
        const double dl[3] = {at[1][0] - at[0][0], at[1][1] - at[0][1], at[1][2] - at[0][2]};
        const double* n = B.n + 3 * b;
        const double along = dl[0] * n[0] + dl[1] * n[1] + dl[2] * n[2];
        const double k = B.a[b] / B.d[b];
        for (int q = 0; q < 3; q++) f[q] = n[q] * (B.e[b] * k * along) + (dl[q] - n[q] * along) * (B.g[b] * k);
    }
    const double inv = 1.0 / B.a[b];
    const double t[3] = {f[0] * inv, f[1] * inv, f[2] * inv};
    const double* n = B.n + 3 * b;
    const double sigma = t[0] * n[0] + t[1] * n[1] + t[2] * n[2];
    const double tau2 = fmax_r(t[0] * t[0] + t[1] * t[1] + t[2] * t[2] - sigma * sigma, 0.0);
    const double r = sqrt(sigma * sigma / 4.0 + tau2);
    const double s1 = sigma / 2.0 + r, s3 = sigma / 2.0 - r;
    used[b] = fmax_r(fmax_r(s1 / B.ft[b], -s3 / B.fc[b]), (s1 - s3) / (2.0 * B.fs[b]));
}

// a beam with any bond over its strength (alive, both ends standing) breaks whole
__global__ void k_break_beams(int64_t nbeams, const double* __restrict__ used, const int64_t* __restrict__ bi,
                              const int64_t* __restrict__ bj, const uint8_t* __restrict__ gone,
                              uint8_t* __restrict__ alive, int32_t* __restrict__ broke) {
    int64_t beam = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (beam >= nbeams) return;
    bool any = false;
    for (int q = 0; q < PER_BEAM; q++) {
        const int64_t b = PER_BEAM * beam + q;
        any = any || (alive[b] && !gone[bi[b]] && !gone[bj[b]] && used[b] > 1.0);
    }
    if (any) {
        for (int q = 0; q < PER_BEAM; q++) alive[PER_BEAM * beam + q] = 0;
        *broke = 1;
    }
}

// the lattice's node positions, held flags and bonds (with strengths) on the device
struct DeviceLattice {
    int64_t n = 0, nb = 0;
    DBuf<double> x, p, nrm, a, d, e, g, ft, fc, fs;
    DBuf<int64_t> bi, bj;
    DBuf<uint8_t> held;
    void load(Context& c, const sc_lattice& L, const sc_strength& S) {
        cudaStream_t st = c.stream;
        n = L.n_nodes;
        nb = L.n_bonds;
        auto up = [&](auto& buf, const auto* src, int64_t count) {
            buf.alloc(std::max<int64_t>(count, 1), st, &c.mem);
            if (count) buf.upload(src, count);
        };
        up(x, L.x, 3 * n);
        up(held, L.held, n);
        up(bi, L.bond_i, nb);
        up(bj, L.bond_j, nb);
        up(p, L.bond_p, 3 * nb);
        up(nrm, L.bond_n, 3 * nb);
        up(a, L.bond_a, nb);
        up(d, L.bond_d, nb);
        up(e, L.bond_e, nb);
        up(g, L.bond_g, nb);
        up(ft, S.ft, nb);
        up(fc, S.fc, nb);
        up(fs, S.fs, nb);
    }
    BondsU view() const {
        return BondsU{bi.get(), bj.get(), p.get(), nrm.get(), a.get(), d.get(), e.get(), g.get(), ft.get(), fc.get(),
                      fs.get()};
    }
};

// gone |= not joined to a held node through alive bonds (bodies.rs:557-574)
void drop_unheld(Context& c, const DeviceLattice& D, const uint8_t* alive, uint8_t* gone) {
    cudaStream_t st = c.stream;
    DBuf<uint8_t> reach;
    reach.alloc(std::max<int64_t>(D.n, 1), st, &c.mem);
    DBuf<int32_t> changed;
    changed.alloc(1, st, &c.mem);
    k_reach_init<<<grid_for(D.n, 256), 256, 0, st>>>(D.n, D.held.get(), reach.get());
    SC_LAUNCH_CK();
    int32_t* flag = c.pinned_i32();
    for (int64_t sweep = 0; sweep <= D.n && D.nb > 0; sweep += 8) {
        changed.zero();
        for (int s = 0; s < 8; s++) {  // eight sweeps between looks at the flag
            k_reach_sweep<<<grid_for(D.nb, 256), 256, 0, st>>>(D.nb, D.bi.get(), D.bj.get(), alive, reach.get(),
                                                               changed.get());
            SC_LAUNCH_CK();
        }
        SC_CK(cudaMemcpyAsync(flag, changed.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        SC_CK(cudaStreamSynchronize(st));
        if (!*flag) break;
    }
    k_gone_update<<<grid_for(D.n, 256), 256, 0, st>>>(D.n, reach.get(), gone);
    SC_LAUNCH_CK();
}

// forces under the weights and their use of the bonds' strengths, for the given alive /
// gone flags (device); the solve's status
sc_status round_used(Context& c, const sc_lattice& L, const DeviceLattice& D, const std::vector<double>& weights,
                     const uint8_t* alive_d, const uint8_t* gone_d, const sc_options& opt, double* used_d,
                     sc_solve_info* info, double& work) {
    cudaStream_t st = c.stream;
    std::vector<uint8_t> alive_h(std::max<int64_t>(D.nb, 1)), gone_h(D.n);
    if (D.nb) SC_CK(cudaMemcpyAsync(alive_h.data(), alive_d, D.nb, cudaMemcpyDeviceToHost, st));
    SC_CK(cudaMemcpyAsync(gone_h.data(), gone_d, D.n, cudaMemcpyDeviceToHost, st));
    SC_CK(cudaStreamSynchronize(st));
    DBuf<double> u;
    u.alloc(6 * D.n, st, &c.mem);
    sc_solve_info local{};
    sc_solve_info* inf = info ? info : &local;
    sc_status s = lattice_motions(c, L, alive_h.data(), gone_h.data(), weights.data(), opt, u.get(), inf);
    work += inf->work;
    if (D.nb > 0) {
        k_bond_used<<<grid_for(D.nb, 256), 256, 0, st>>>(D.nb, D.view(), D.x.get(), u.get(), alive_d, gone_d, used_d);
        SC_LAUNCH_CK();
    }
    return s;
}

std::vector<double> weights_of(const sc_lattice& L, const sc_strength& S) {
    std::vector<double> w(6 * L.n_nodes, 0.0);  // Node::m * GRAVITY down y (bodies.rs:408)
    for (int64_t v = 0; v < L.n_nodes; v++) w[6 * v + 1] = -S.m[v] * GRAVITY;
    return w;
}

}  // namespace

sc_status used_standing(Context& c, const sc_lattice& L, const sc_strength& S, const sc_options& opt, double* used,
                        sc_solve_info* info) {
    cudaStream_t st = c.stream;
    DeviceLattice D;
    D.load(c, L, S);
    DBuf<uint8_t> alive, gone;
    alive.alloc(std::max<int64_t>(D.nb, 1), st, &c.mem);
    SC_CK(cudaMemsetAsync(alive.get(), 1, std::max<int64_t>(D.nb, 1), st));
    gone.alloc(D.n, st, &c.mem);
    gone.zero();
    drop_unheld(c, D, alive.get(), gone.get());
    DBuf<double> u;
    u.alloc(std::max<int64_t>(D.nb, 1), st, &c.mem);
    double work = 0;
    sc_status s = round_used(c, L, D, weights_of(L, S), alive.get(), gone.get(), opt, u.get(), info, work);
    if (D.nb) u.download(used, D.nb);
    SC_CK(cudaStreamSynchronize(st));
    return s;
}

sc_status settle(Context& c, const sc_lattice& L, const sc_strength& S, const sc_options& opt, uint8_t* gone_out,
                 sc_settle_info* out) {
    cudaStream_t st = c.stream;
    DeviceLattice D;
    D.load(c, L, S);
    const std::vector<double> w = weights_of(L, S);
    DBuf<uint8_t> alive, gone;
    alive.alloc(std::max<int64_t>(D.nb, 1), st, &c.mem);
    SC_CK(cudaMemsetAsync(alive.get(), 1, std::max<int64_t>(D.nb, 1), st));
    gone.alloc(D.n, st, &c.mem);
    gone.zero();
    DBuf<double> used;
    used.alloc(std::max<int64_t>(D.nb, 1), st, &c.mem);
    DBuf<int32_t> broke;
    broke.alloc(1, st, &c.mem);
    int32_t* flag = c.pinned_i32();
    double work = 0;
    int64_t rounds = 0;
    sc_status worst = SC_OK;
    // every round breaks at least one beam or ends, so at most n_bonds / 4 + 1 rounds
    for (;;) {
        rounds += 1;
        drop_unheld(c, D, alive.get(), gone.get());
        sc_status s = round_used(c, L, D, w, alive.get(), gone.get(), opt, used.get(), nullptr, work);
        worst = std::max(worst, s);
        broke.zero();
        const int64_t nbeams = D.nb / PER_BEAM;
        if (nbeams > 0) {
            k_break_beams<<<grid_for(nbeams, 256), 256, 0, st>>>(nbeams, used.get(), D.bi.get(), D.bj.get(),
                                                                 gone.get(), alive.get(), broke.get());
            SC_LAUNCH_CK();
        }
        SC_CK(cudaMemcpyAsync(flag, broke.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        SC_CK(cudaStreamSynchronize(st));
        if (!*flag) break;
    }
    gone.download(gone_out, D.n);
    SC_CK(cudaStreamSynchronize(st));
    double free = 0.0, fell = 0.0;
    for (int64_t v = 0; v < D.n; v++) {
        if (!L.held[v]) free += S.m[v];
        if (gone_out[v]) fell += S.m[v];
    }
    if (out) {
        out->fell = free > 0.0 ? fell / free : 0.0;
        out->rounds = rounds;
        out->work = work;
        out->status = worst;
    }
    return worst;
}


// statics::bodies::as_generated (bodies.rs:611-625): for every beam of `generated` (its
// bonds keyed by the cells their two ends lie between, the lesser end first), the most
// of its strength any of its bonds uses standing; each bond of `lattice` on the same beam
// made max(MARGIN * that, 1) times as strong (Mat::stronger, model.rs:71-73), the others
// unchanged. The used fractions are the device's (used_standing); the matching is host
// work, as the reference's is: both bond lists keyed and sorted, then merged.
sc_status as_generated(Context& c, const sc_lattice& L, const sc_strength& S, const sc_lattice& G,
                       const sc_strength& GS, const sc_options& opt, double* ft, double* fc, double* fs) {
    constexpr double MARGIN = 2.0;  // bodies.rs:605
    std::vector<double> used((size_t)std::max<int64_t>(G.n_bonds, 1));
    sc_solve_info info;
    sc_status s = used_standing(c, G, GS, opt, used.data(), &info);
    using Key = std::array<int64_t, 12>;
    auto key_of = [](const sc_lattice& l, int64_t b) {
        const int64_t* i = l.around + 6 * l.bond_i[b];
        const int64_t* j = l.around + 6 * l.bond_j[b];
        Key k;
        const bool swap = !std::lexicographical_compare(i, i + 6, j, j + 6);  // i < j keeps the order
        const int64_t* a = swap ? j : i;
        const int64_t* z = swap ? i : j;
        std::copy(a, a + 6, k.begin());
        std::copy(z, z + 6, k.begin() + 6);
        return k;
    };
    // the generated beams' need: the most any of their bonds uses (f64::max, NaN ignored)
    std::vector<std::pair<Key, double>> need((size_t)G.n_bonds);
    for (int64_t b = 0; b < G.n_bonds; b++) need[b] = {key_of(G, b), used[b]};
    std::stable_sort(need.begin(), need.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
    std::vector<std::pair<Key, double>> beams;
    for (auto& kv : need) {
        if (beams.empty() || beams.back().first != kv.first)
            beams.push_back({kv.first, std::fmax(0.0, kv.second)});
        else
            beams.back().second = std::fmax(beams.back().second, kv.second);
    }
    for (int64_t b = 0; b < L.n_bonds; b++) {
        const Key k = key_of(L, b);
        auto it = std::lower_bound(beams.begin(), beams.end(), k,
                                   [](const auto& x, const Key& y) { return x.first < y; });
        const double by = (it != beams.end() && it->first == k) ? std::fmax(it->second * MARGIN, 1.0) : 1.0;
        ft[b] = S.ft[b] * by;
        fc[b] = S.fc[b] * by;
        fs[b] = S.fs[b] * by;
    }
    return s;
}

}  // namespace sc
