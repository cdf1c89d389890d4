// Row-by-row block-sparse products for the Galerkin triple product (statics/src/bodies.rs:
// 252-282) on levels whose pieces have at most ROWS_MAX_WIDTH coarse parts: C = op(A) B,
// each row i keeping only the columns [lo_i, hi_i). Every row's pattern is a bitmap of
// its window in shared memory and its values are summed in shared memory, one thread
// block per row, so no candidate list is expanded, sorted or stored. The contributions
// to a block are added in A's entry order, as the sorted-candidate product adds them, so
// both give the same bits.
#pragma once
#include "solver.cuh"
#include "level0_blocks.cuh"

namespace sc {

constexpr int64_t ROWS_MAX_WIDTH = 65536;  // window width the shared-memory bitmap covers

enum RowProdMode { ROWS_PLAIN = 0, ROWS_K0 = 1, ROWS_TRANSPOSED = 2 };

struct RowArgs {
    // A: rows, the B row of each entry and its block. PLAIN: block e of aval; K0: the
    // cell-template block of level 0 (k0); TRANSPOSED: block aent[e] of aval, transposed.
    const int64_t* arow;
    const int32_t* acol;
    const int64_t* aent;
    const double* aval;
    K0View k0;
    int64_t annz;
    // B
    const int64_t* brow;
    const int32_t* bcol;
    const double* bval;
    // each row's window [lo, hi) of output columns (empty when hi <= lo)
    const int32_t* lo;
    const int32_t* hi;
};

// Pattern (rowptr, sorted columns) and values of C; cands = the products summed.
void row_products(Context& ctx, int mode, const RowArgs& a, int64_t nrows, int64_t max_width, DBuf<int64_t>& crow,
                  DBuf<int32_t>& ccol, DBuf<double>& cval, int64_t& cnnz, int64_t& cands);

// windows of K P: row k of a continuing piece keeps columns from its P row's first
// column to its piece's last coarse part; a stopped row (up < 0) none
void kp_windows(Context& ctx, int64_t n, const int32_t* up, const int64_t* prow, const int32_t* pcol,
                const int32_t* piece, const int64_t* cpstart, int32_t* lo, int32_t* hi);
// windows of the upper P'KP: row c keeps columns from c to its piece's last coarse part
void upper_windows(Context& ctx, int64_t nc, const int32_t* cpiece, const int64_t* cpstart, int32_t* lo, int32_t* hi);

}  // namespace sc
