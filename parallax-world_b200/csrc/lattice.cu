// Level 0 of a general lattice (any `Lattice`: the reference's level 0 or a gathered
// coarser level) assembled on the device from its bonds, as Level::new does
// (statics/src/bodies.rs:126-164): parts are the nodes neither held nor gone, in node
// order; every live bond (alive, neither end gone) adds T_i' S T_i to each free end's
// own block and -T_i' S T_j to the pair, S = Bond::stiffness (statics/src/model.rs:139-149),
// T_v = [I | -[p - x_v]x]. Contributions to one block are summed in bond order (a stable
// sort keeps it), so the assembly is deterministic.
#include <cub/cub.cuh>

#include "kernels.cuh"

namespace sc {

namespace {

struct BondsD {
    const int64_t* bi;
    const int64_t* bj;
    const double* p;
    const double* n;
    const double* a;
    const double* d;
    const double* e;
    const double* g;
    const double* x;  // node centres
};

__global__ void k_part_flags(int64_t nn, const uint8_t* __restrict__ held, const uint8_t* __restrict__ gone,
                             int64_t* __restrict__ isp) {
    int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (v >= nn) return;
    isp[v] = (!held[v] && !(gone && gone[v])) ? 1 : 0;
}

__global__ void k_part_of(int64_t nn, const int64_t* __restrict__ isp, const int64_t* __restrict__ before,
                          int32_t* __restrict__ part, int32_t* __restrict__ part_node) {
    int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (v >= nn) return;
    if (isp[v]) {
        part[v] = (int32_t)before[v];
        part_node[before[v]] = (int32_t)v;
    } else {
        part[v] = -1;
    }
}

__global__ void k_part_geom(int64_t np_, const int32_t* __restrict__ part_node, const double* __restrict__ x,
                            const int64_t* __restrict__ around, const double* __restrict__ loads,
                            double* __restrict__ centre, int64_t* __restrict__ site, double* __restrict__ rhs,
                            int32_t* __restrict__ piece) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= np_) return;
    int64_t v = part_node[k];
    for (int q = 0; q < 3; q++) {
        centre[3 * k + q] = x[3 * v + q];
        site[3 * k + q] = around[6 * v + q];
    }
    for (int q = 0; q < 6; q++) rhs[6 * k + q] = loads[6 * v + q];
    piece[k] = 0;
}

__device__ __forceinline__ bool live(int64_t b, const uint8_t* alive, const uint8_t* gone, const int64_t* bi,
                                     const int64_t* bj) {
    if (alive && !alive[b]) return false;
    if (gone && (gone[bi[b]] || gone[bj[b]])) return false;
    return true;
}

// entries per bond: ii, jj (free ends), ij and ji (both free); plus one diagonal per part
__global__ void k_bond_count(int64_t nb, BondsD B, const uint8_t* __restrict__ alive, const uint8_t* __restrict__ gone,
                             const int32_t* __restrict__ part, int64_t* __restrict__ cnt) {
    int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (b >= nb) return;
    int c = 0;
    if (live(b, alive, gone, B.bi, B.bj)) {
        int32_t i = part[B.bi[b]], j = part[B.bj[b]];
        c = (i >= 0) + (j >= 0) + 2 * (i >= 0 && j >= 0);
    }
    cnt[b] = c;
}

// kind: 0 own of i, 1 own of j, 2 (i,j), 3 (j,i)
__global__ void k_bond_fill(int64_t nb, BondsD B, const uint8_t* __restrict__ alive, const uint8_t* __restrict__ gone,
                            const int32_t* __restrict__ part, const int64_t* __restrict__ off,
                            uint64_t* __restrict__ keys, int64_t* __restrict__ ref) {
    int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (b >= nb) return;
    if (!live(b, alive, gone, B.bi, B.bj)) return;
    int32_t i = part[B.bi[b]], j = part[B.bj[b]];
    int64_t o = off[b];
    auto put = [&](int32_t r, int32_t c, int kind) {
        keys[o] = ((uint64_t)(uint32_t)r << 32) | (uint32_t)c;
        ref[o] = 4 * b + kind;
        o++;
    };
    if (i >= 0) put(i, i, 0);
    if (j >= 0) put(j, j, 1);
    if (i >= 0 && j >= 0) {
        put(i, j, 2);
        put(j, i, 3);
    }
}

__global__ void k_diag_fill(int64_t np_, int64_t base, uint64_t* __restrict__ keys, int64_t* __restrict__ ref) {
    int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= np_) return;
    keys[base + k] = ((uint64_t)(uint32_t)k << 32) | (uint32_t)k;
    ref[base + k] = -1;
}

// T_a' S T_b for a bond (bodies.rs:141-149): a, b the node centres of its two sides
__device__ void through(const BondsD& B, int64_t b, int64_t va, int64_t vb, double* out) {
    double n[3] = {B.n[3 * b], B.n[3 * b + 1], B.n[3 * b + 2]};
    double k = B.a[b] / B.d[b];
    double s[3][3];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) {
            double nn = n[r] * n[c];
            s[r][c] = B.e[b] * k * nn + B.g[b] * k * ((r == c ? 1.0 : 0.0) - nn);
        }
    auto T = [&](int64_t v, double t[3][6]) {
        double r0 = B.p[3 * b] - B.x[3 * v], r1 = B.p[3 * b + 1] - B.x[3 * v + 1], r2 = B.p[3 * b + 2] - B.x[3 * v + 2];
        double m[3][6] = {{1, 0, 0, 0, r2, -r1}, {0, 1, 0, -r2, 0, r0}, {0, 0, 1, r1, -r0, 0}};
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 6; j++) t[i][j] = m[i][j];
    };
    double ta[3][6], tb[3][6];
    T(va, ta);
    T(vb, tb);
    double sb[3][6];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 6; c++) {
            double acc = 0.0;
            for (int q = 0; q < 3; q++) acc += s[r][q] * tb[q][c];
            sb[r][c] = acc;
        }
    for (int r = 0; r < 6; r++)
        for (int c = 0; c < 6; c++) {
            double acc = 0.0;
            for (int q = 0; q < 3; q++) acc += ta[q][r] * sb[q][c];
            out[6 * r + c] = acc;
        }
}

// one thread per stored block: sum its contributions in bond order
__global__ void k_block_sum(int64_t nblk, const int64_t* __restrict__ seg, const int64_t* __restrict__ ref, BondsD B,
                            double* __restrict__ val) {
    int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= nblk) return;
    double acc[36];
    for (int i = 0; i < 36; i++) acc[i] = 0.0;
    double t[36];
    for (int64_t e = seg[q]; e < seg[q + 1]; e++) {
        int64_t rf = ref[e];
        if (rf < 0) continue;
        int64_t b = rf >> 2;
        int kind = (int)(rf & 3);
        int64_t vi = B.bi[b], vj = B.bj[b];
        if (kind == 0) {
            through(B, b, vi, vi, t);
            for (int i = 0; i < 36; i++) acc[i] += t[i];
        } else if (kind == 1) {
            through(B, b, vj, vj, t);
            for (int i = 0; i < 36; i++) acc[i] += t[i];
        } else {
            // the pair block is of (lesser part, greater part); the other is its transpose
            through(B, b, kind == 2 ? vi : vj, kind == 2 ? vj : vi, t);
            for (int i = 0; i < 36; i++) acc[i] -= t[i];
        }
    }
    for (int i = 0; i < 36; i++) val[36 * q + i] = acc[i];
}

// make pairs exactly symmetric: block (r, c) with r > c becomes the transpose of (c, r)
__global__ void k_symmetrize(int64_t n, const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                             double* __restrict__ val) {
    int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= n) return;
    for (int64_t e = rowptr[r]; e < rowptr[r + 1]; e++) {
        int32_t c = col[e];
        if (c >= (int32_t)r) break;
        int64_t f = lower_bound_i32(col, rowptr[c], rowptr[c + 1], (int32_t)r);
        for (int i = 0; i < 6; i++)
            for (int j = 0; j < 6; j++) val[36 * e + 6 * i + j] = val[36 * f + 6 * j + i];
    }
}

__global__ void k_unpack2(int64_t m, const uint64_t* __restrict__ keys, int32_t* __restrict__ col,
                          int32_t* __restrict__ row) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= m) return;
    col[i] = (int32_t)(keys[i] & 0xffffffffu);
    row[i] = (int32_t)(keys[i] >> 32);
}

__global__ void k_seg_starts(int64_t m, const uint64_t* __restrict__ keys, int64_t* __restrict__ flag) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= m) return;
    flag[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}
__global__ void k_seg_write(int64_t m, const uint64_t* __restrict__ keys, const int64_t* __restrict__ flag,
                            const int64_t* __restrict__ idx, int64_t* __restrict__ seg, uint64_t* __restrict__ ukeys) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= m) return;
    if (flag[i]) {
        seg[idx[i]] = i;
        ukeys[idx[i]] = keys[i];
    }
}
__global__ void k_rowptr(int64_t m, const int32_t* __restrict__ rows, int64_t nrows, int64_t* __restrict__ rowptr) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i > m) return;
    int32_t prev = i == 0 ? -1 : rows[i - 1];
    int32_t cur = i == m ? (int32_t)nrows : rows[i];
    for (int32_t c = prev + 1; c <= cur; c++) rowptr[c] = i;
}

int bits_for2(int64_t v) {
    int b = 1;
    while (b < 63 && (int64_t(1) << b) <= v) b++;
    return b;
}

}  // namespace

void lattice_level0(Context& ctx, Batch& b, const sc_lattice& Lt, const uint8_t* alive_h, const uint8_t* gone_h,
                    const double* loads_h) {
    cudaStream_t st = ctx.stream;
    MemStats* ms = &ctx.mem;
    int64_t nn = Lt.n_nodes, nb = Lt.n_bonds;
    b.npieces = 1;
    b.base_level = Lt.level;
    auto up = [&](auto* host, size_t count, auto& buf) {
        buf.alloc(std::max<size_t>(count, 1), st, ms);
        if (host) buf.upload(host, count);
    };
    DBuf<double> x, p, n, a, d, e, g, loads;
    DBuf<int64_t> bi, bj, around;
    DBuf<uint8_t> held, alive, gone;
    up(Lt.x, 3 * nn, x);
    up(Lt.bond_p, 3 * nb, p);
    up(Lt.bond_n, 3 * nb, n);
    up(Lt.bond_a, nb, a);
    up(Lt.bond_d, nb, d);
    up(Lt.bond_e, nb, e);
    up(Lt.bond_g, nb, g);
    up(Lt.bond_i, nb, bi);
    up(Lt.bond_j, nb, bj);
    up(Lt.around, 6 * nn, around);
    up(Lt.held, nn, held);
    up(loads_h, 6 * nn, loads);
    if (alive_h) up(alive_h, nb, alive);
    if (gone_h) up(gone_h, nn, gone);
    const uint8_t* al = alive_h ? alive.get() : nullptr;
    const uint8_t* gn = gone_h ? gone.get() : nullptr;
    BondsD B{bi.get(), bj.get(), p.get(), n.get(), a.get(), d.get(), e.get(), g.get(), x.get()};
    // parts
    DBuf<int64_t> isp, before;
    isp.alloc(nn + 1, st, ms);
    before.alloc(nn + 1, st, ms);
    SC_CK(cudaMemsetAsync(isp.get() + nn, 0, sizeof(int64_t), st));
    k_part_flags<<<grid_for(nn, 256), 256, 0, st>>>(nn, held.get(), gn, isp.get());
    SC_LAUNCH_CK();
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, isp.get(), before.get(), nn + 1, st);
    cub::DeviceScan::ExclusiveSum(ctx.cub_scratch(tb), tb, isp.get(), before.get(), nn + 1, st);
    int64_t nparts = 0;
    SC_CK(cudaMemcpyAsync(&nparts, before.get() + nn, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    SC_CK(cudaStreamSynchronize(st));
    require(nparts > 0, SC_BAD_INPUT, "no free node");
    require(nparts < INT32_MAX, SC_BAD_INPUT, "lattice too large");
    b.node_count = {nn};
    std::vector<int64_t> ns = {0, nn};
    b.node_start.alloc(2, st, ms);
    b.node_start.upload(ns.data(), 2);
    DBuf<int32_t> part;
    part.alloc(nn, st, ms);
    b.part_node.alloc(nparts, st, ms);
    k_part_of<<<grid_for(nn, 256), 256, 0, st>>>(nn, isp.get(), before.get(), part.get(), b.part_node.get());
    SC_LAUNCH_CK();
    Level& L = b.levels.emplace_back();
    L.n = nparts;
    L.pstart = {0, nparts};
    L.pstart_d.alloc(2, st, ms);
    L.pstart_d.upload(L.pstart.data(), 2);
    L.centre.alloc(3 * nparts, st, ms);
    L.site.alloc(3 * nparts, st, ms);
    L.piece.alloc(nparts, st, ms);
    b.loads.alloc(6 * nparts, st, ms);
    k_part_geom<<<grid_for(nparts, 256), 256, 0, st>>>(nparts, b.part_node.get(), x.get(), around.get(), loads.get(),
                                                       L.centre.get(), L.site.get(), b.loads.get(), L.piece.get());
    SC_LAUNCH_CK();
    // block entries
    DBuf<int64_t> cnt, off;
    cnt.alloc(nb + 1, st, ms);
    off.alloc(nb + 1, st, ms);
    SC_CK(cudaMemsetAsync(cnt.get() + nb, 0, sizeof(int64_t), st));
    if (nb > 0) {
        k_bond_count<<<grid_for(nb, 256), 256, 0, st>>>(nb, B, al, gn, part.get(), cnt.get());
        SC_LAUNCH_CK();
    }
    cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.get(), off.get(), nb + 1, st);
    cub::DeviceScan::ExclusiveSum(ctx.cub_scratch(tb), tb, cnt.get(), off.get(), nb + 1, st);
    int64_t m = 0;
    SC_CK(cudaMemcpyAsync(&m, off.get() + nb, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    SC_CK(cudaStreamSynchronize(st));
    int64_t tot = m + nparts;
    DBuf<uint64_t> keys, keys_s;
    DBuf<int64_t> ref, ref_s;
    keys.alloc(tot, st, ms);
    ref.alloc(tot, st, ms);
    if (nb > 0) {
        k_bond_fill<<<grid_for(nb, 256), 256, 0, st>>>(nb, B, al, gn, part.get(), off.get(), keys.get(), ref.get());
        SC_LAUNCH_CK();
    }
    k_diag_fill<<<grid_for(nparts, 256), 256, 0, st>>>(nparts, m, keys.get(), ref.get());
    SC_LAUNCH_CK();
    keys_s.alloc(tot, st, ms);
    ref_s.alloc(tot, st, ms);
    int end_bit = 32 + bits_for2(nparts);
    cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.get(), keys_s.get(), ref.get(), ref_s.get(), tot, 0, end_bit, st);
    cub::DeviceRadixSort::SortPairs(ctx.cub_scratch(tb), tb, keys.get(), keys_s.get(), ref.get(), ref_s.get(), tot, 0,
                                    end_bit, st);
    keys.release();
    ref.release();
    DBuf<int64_t> flag, idx;
    flag.alloc(tot + 1, st, ms);
    idx.alloc(tot + 1, st, ms);
    SC_CK(cudaMemsetAsync(flag.get() + tot, 0, sizeof(int64_t), st));
    k_seg_starts<<<grid_for(tot, 256), 256, 0, st>>>(tot, keys_s.get(), flag.get());
    SC_LAUNCH_CK();
    cub::DeviceScan::ExclusiveSum(nullptr, tb, flag.get(), idx.get(), tot + 1, st);
    cub::DeviceScan::ExclusiveSum(ctx.cub_scratch(tb), tb, flag.get(), idx.get(), tot + 1, st);
    int64_t nblk = 0;
    SC_CK(cudaMemcpyAsync(&nblk, idx.get() + tot, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    SC_CK(cudaStreamSynchronize(st));
    DBuf<int64_t> seg;
    seg.alloc(nblk + 1, st, ms);
    DBuf<uint64_t> ukeys;
    ukeys.alloc(nblk, st, ms);
    k_seg_write<<<grid_for(tot, 256), 256, 0, st>>>(tot, keys_s.get(), flag.get(), idx.get(), seg.get(), ukeys.get());
    SC_LAUNCH_CK();
    SC_CK(cudaMemcpyAsync(seg.get() + nblk, &tot, sizeof(int64_t), cudaMemcpyHostToDevice, st));
    L.nnzb = nblk;
    L.col.alloc(nblk, st, ms);
    DBuf<int32_t> rows;
    rows.alloc(nblk, st, ms);
    k_unpack2<<<grid_for(nblk, 256), 256, 0, st>>>(nblk, ukeys.get(), L.col.get(), rows.get());
    SC_LAUNCH_CK();
    L.rowptr.alloc(nparts + 1, st, ms);
    k_rowptr<<<grid_for(nblk + 1, 256), 256, 0, st>>>(nblk, rows.get(), nparts, L.rowptr.get());
    SC_LAUNCH_CK();
    L.val.alloc(36 * nblk, st, ms);
    k_block_sum<<<grid_for(nblk, 64), 64, 0, st>>>(nblk, seg.get(), ref_s.get(), B, L.val.get());
    SC_LAUNCH_CK();
    k_symmetrize<<<grid_for(nparts, 128), 128, 0, st>>>(nparts, L.rowptr.get(), L.col.get(), L.val.get());
    SC_LAUNCH_CK();
    L.matrix_free = false;
    SC_CK(cudaStreamSynchronize(st));
}

}  // namespace sc
