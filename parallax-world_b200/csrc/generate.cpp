// Seeded synthetic voxel pieces: the structures the solver is measured on.
//
// Occupancy is 3D value noise of period 8 (lattice values every 8 cells, trilinear
// between them) thresholded at 0.5; the bottom z layer is fully occupied and held (the
// support), and only the 6-connected component that touches it is kept. Each cell's
// stiffness k is drawn from its own stream: uniform in [0.5, 2.0], or lognormal
// (mu 0, sigma 0.5, Box-Muller) clipped to [0.1, 10]. Cells are laid out x slowest,
// z fastest: the order in which the reference's `solids` visits sites
// (statics/src/lattice.rs:87-102), so a cell's flat index is ((x*ny)+y)*nz+z.
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/statics_cuda.h"

namespace {

uint64_t splitmix64(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// One 64-bit draw per (seed, stream, i, j, k).
uint64_t draw(uint64_t seed, uint64_t stream, int64_t i, int64_t j, int64_t k) {
    uint64_t h = splitmix64(seed ^ (stream * 0xD1B54A32D192ED03ull));
    h = splitmix64(h ^ (uint64_t)i);
    h = splitmix64(h ^ (uint64_t)j);
    h = splitmix64(h ^ (uint64_t)k);
    return h;
}

double unit_draw(uint64_t h) { return (double)(h >> 11) * 0x1.0p-53; }

constexpr int PERIOD = 8;

}  // namespace

extern "C" sc_status sc_generate_piece(int32_t nx, int32_t ny, int32_t nz, uint64_t seed, int32_t k_dist,
                                       uint8_t* state, float* k) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || !state || !k) return SC_BAD_INPUT;
    const size_t n = (size_t)nx * ny * nz;
    auto at = [&](int x, int y, int z) { return ((size_t)x * ny + y) * nz + z; };
    // Lattice values on the period-8 grid, one extra point past each far edge.
    const int lx = nx / PERIOD + 2, ly = ny / PERIOD + 2, lz = nz / PERIOD + 2;
    std::vector<double> lat((size_t)lx * ly * lz);
    for (int i = 0; i < lx; i++)
        for (int j = 0; j < ly; j++)
            for (int q = 0; q < lz; q++) lat[((size_t)i * ly + j) * lz + q] = unit_draw(draw(seed, 0, i, j, q));
    std::vector<uint8_t> occ(n, 0);
    for (int x = 0; x < nx; x++)
        for (int y = 0; y < ny; y++)
            for (int z = 0; z < nz; z++) {
                double f[3] = {(x + 0.5) / PERIOD, (y + 0.5) / PERIOD, (z + 0.5) / PERIOD};
                int i0[3];
                double t[3];
                for (int a = 0; a < 3; a++) {
                    i0[a] = (int)std::floor(f[a]);
                    t[a] = f[a] - i0[a];
                }
                double v = 0.0;
                for (int c = 0; c < 8; c++) {
                    int di = c >> 2 & 1, dj = c >> 1 & 1, dk = c & 1;
                    double w = (di ? t[0] : 1 - t[0]) * (dj ? t[1] : 1 - t[1]) * (dk ? t[2] : 1 - t[2]);
                    v += w * lat[((size_t)(i0[0] + di) * ly + (i0[1] + dj)) * lz + (i0[2] + dk)];
                }
                occ[at(x, y, z)] = (z == 0 || v > 0.5) ? 1 : 0;
            }
    // Keep what a 6-connected chain joins to the support layer.
    std::vector<uint8_t> keep(n, 0);
    std::vector<size_t> stack;
    for (int x = 0; x < nx; x++)
        for (int y = 0; y < ny; y++) {
            size_t c = at(x, y, 0);
            keep[c] = 1;
            stack.push_back(c);
        }
    while (!stack.empty()) {
        size_t c = stack.back();
        stack.pop_back();
        int z = (int)(c % nz), y = (int)(c / nz % ny), x = (int)(c / ((size_t)nz * ny));
        const int d[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
        for (auto& o : d) {
            int a = x + o[0], b = y + o[1], e = z + o[2];
            if (a < 0 || b < 0 || e < 0 || a >= nx || b >= ny || e >= nz) continue;
            size_t q = at(a, b, e);
            if (occ[q] && !keep[q]) {
                keep[q] = 1;
                stack.push_back(q);
            }
        }
    }
    for (int x = 0; x < nx; x++)
        for (int y = 0; y < ny; y++)
            for (int z = 0; z < nz; z++) {
                size_t c = at(x, y, z);
                state[c] = keep[c] ? (z == 0 ? SC_CELL_HELD : SC_CELL_FREE) : SC_CELL_EMPTY;
                double kv;
                if (k_dist == SC_K_LOGNORMAL) {
                    double u1 = ((double)(draw(seed, 1, x, y, z) >> 11) + 1.0) * 0x1.0p-53;
                    double u2 = unit_draw(draw(seed, 2, x, y, z));
                    double g = std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
                    kv = std::exp(0.5 * g);
                    kv = kv < 0.1 ? 0.1 : (kv > 10.0 ? 10.0 : kv);
                } else {
                    kv = 0.5 + 1.5 * unit_draw(draw(seed, 1, x, y, z));
                }
                k[c] = keep[c] ? (float)kv : 0.0f;
            }
    return SC_OK;
}
