// ORACLE — test infrastructure only, never part of the product.
//
// The benchmark's seeded synthetic voxel pieces, made on the host without the product
// library, so that the CPU reference arm and the CPU tests build their inputs from the
// checker's side alone. The definition (the benchmark's own; the reference has none):
//
//   * occupancy: value noise of period 8 -- one value per lattice point (i, j, q) of
//     the period-8 grid, SplitMix64 of (seed, stream 0, i, j, q) mapped to [0, 1) by
//     its top 53 bits, read trilinearly at the cell centre ((x+0.5)/8, (y+0.5)/8,
//     (z+0.5)/8); a cell is filled when the value is above 0.5, and the bottom z layer
//     is always filled;
//   * support: the bottom layer is held, and only what a 6-connected chain of filled
//     cells joins to it is kept;
//   * stiffness: its own stream per cell: uniform 0.5 + 1.5 u (stream 1), or
//     exp(0.5 g) clipped to [0.1, 10] with g a Box-Muller normal of streams 1 and 2.
//
// Cells are stored x slowest, z fastest (flat index ((x*ny)+y)*nz+z), the order in
// which the reference's `solids` visits sites (statics/src/lattice.rs:87-102).
// tests/test_oracle_generator.py checks that these pieces equal the library's
// sc_generate_piece byte for byte.
#include <cmath>
#include <cstdint>
#include <deque>
#include <vector>

namespace {

uint64_t mix(uint64_t x) {  // SplitMix64's output function of x + golden gamma
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

uint64_t hash4(uint64_t seed, uint64_t stream, int64_t i, int64_t j, int64_t q) {
    uint64_t h = mix(seed ^ (stream * 0xD1B54A32D192ED03ull));
    for (int64_t v : {i, j, q}) h = mix(h ^ (uint64_t)v);
    return h;
}

double to_unit(uint64_t h) { return std::ldexp((double)(h >> 11), -53); }

}  // namespace

extern "C" int or_generate_piece(int nx, int ny, int nz, uint64_t seed, int k_dist, uint8_t* state, float* k) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || !state || !k) return 4;
    const int64_t n = (int64_t)nx * ny * nz;
    auto flat = [&](int64_t x, int64_t y, int64_t z) { return (x * ny + y) * nz + z; };
    const int P = 8;
    const int gx = nx / P + 2, gy = ny / P + 2, gz = nz / P + 2;
    auto lattice = [&](int i, int j, int q) { return to_unit(hash4(seed, 0, i, j, q)); };
    std::vector<double> g((size_t)gx * gy * gz);
    for (int i = 0; i < gx; i++)
        for (int j = 0; j < gy; j++)
            for (int q = 0; q < gz; q++) g[((size_t)i * gy + j) * gz + q] = lattice(i, j, q);
    std::vector<uint8_t> filled(n);
    for (int x = 0; x < nx; x++)
        for (int y = 0; y < ny; y++)
            for (int z = 0; z < nz; z++) {
                const double u[3] = {(x + 0.5) / P, (y + 0.5) / P, (z + 0.5) / P};
                int b[3];
                double f[3];
                for (int a = 0; a < 3; a++) {
                    b[a] = (int)std::floor(u[a]);
                    f[a] = u[a] - b[a];
                }
                // the eight corners in the order (di, dj, dq) = 000, 001, ..., 111
                double v = 0.0;
                for (int corner = 0; corner < 8; corner++) {
                    const int di = (corner >> 2) & 1, dj = (corner >> 1) & 1, dq = corner & 1;
                    const double w = (di ? f[0] : 1 - f[0]) * (dj ? f[1] : 1 - f[1]) * (dq ? f[2] : 1 - f[2]);
                    v += w * g[((size_t)(b[0] + di) * gy + (b[1] + dj)) * gz + (b[2] + dq)];
                }
                filled[flat(x, y, z)] = (z == 0 || v > 0.5) ? 1 : 0;
            }
    // what a 6-connected chain joins to the support (a breadth-first walk; which cells
    // are reached does not depend on the walk's order)
    std::vector<uint8_t> kept(n, 0);
    std::deque<int64_t> todo;
    for (int x = 0; x < nx; x++)
        for (int y = 0; y < ny; y++) {
            kept[flat(x, y, 0)] = 1;
            todo.push_back(flat(x, y, 0));
        }
    while (!todo.empty()) {
        const int64_t c = todo.front();
        todo.pop_front();
        const int64_t z = c % nz, y = c / nz % ny, x = c / ((int64_t)nz * ny);
        const int64_t nb[6][3] = {{x - 1, y, z}, {x + 1, y, z}, {x, y - 1, z}, {x, y + 1, z}, {x, y, z - 1}, {x, y, z + 1}};
        for (auto& o : nb) {
            if (o[0] < 0 || o[1] < 0 || o[2] < 0 || o[0] >= nx || o[1] >= ny || o[2] >= nz) continue;
            const int64_t q = flat(o[0], o[1], o[2]);
            if (filled[q] && !kept[q]) {
                kept[q] = 1;
                todo.push_back(q);
            }
        }
    }
    for (int x = 0; x < nx; x++)
        for (int y = 0; y < ny; y++)
            for (int z = 0; z < nz; z++) {
                const int64_t c = flat(x, y, z);
                state[c] = kept[c] ? (z == 0 ? 2 : 1) : 0;  // held, free, empty
                double kv;
                if (k_dist == 1) {
                    const double u1 = std::ldexp((double)(hash4(seed, 1, x, y, z) >> 11) + 1.0, -53);
                    const double u2 = to_unit(hash4(seed, 2, x, y, z));
                    const double normal = std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
                    kv = std::fmin(std::fmax(std::exp(0.5 * normal), 0.1), 10.0);
                } else {
                    kv = 0.5 + 1.5 * to_unit(hash4(seed, 1, x, y, z));
                }
                k[c] = kept[c] ? (float)kv : 0.0f;
            }
    return 0;
}
