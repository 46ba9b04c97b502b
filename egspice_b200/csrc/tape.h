// Host-side symbolic analysis for the lane tapes: the BTF + AMD column order
// (ESPice src/solver/order.zig) and the lead lane's threshold-pivoted
// Gilbert-Peierls factor (src/solver/sparse_lu.zig factor/factorPass), frozen
// into the pivot tape every lane replays (src/solver/kernels/lane.zig
// LaneTab/buildTab). This is the reference's `ownTape` step
// (src/analysis/gpu/lanes.zig:590-603), which also runs on the host there.
#pragma once

#include <cstdint>
#include <vector>

namespace espl {

constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr double kPivotTol = 1e-3;          // direct.zig:33
constexpr double kRepivotFillCap = 3.0;     // direct.zig:36
constexpr double kGrowthLimit = 1e-12;      // direct.zig:54
constexpr uint32_t kVoidBit = 1, kScaledBit = 2;  // kernels/lane.zig:41,44

// Column order q (q[k] = column factored at step k). False on
// OutOfWorkspace, with the reference's slab size 48 n + 8 nnz + 64 words.
bool order_columns(uint32_t n, const uint32_t* col_ptr, const uint32_t* row_idx, std::vector<uint32_t>& q);

// Strictly-lower plus strictly-upper entries of an LU of the pattern under
// diagonal pivots in order q: twice the off-diagonal Cholesky count of A+A^T.
uint64_t diag_fill(uint32_t n, const uint32_t* col_ptr, const uint32_t* row_idx, const std::vector<uint32_t>& q);

// A frozen pivot tape: the factor's pattern and pivot sequence.
struct Tape {
    uint32_t n = 0, nnz = 0;
    std::vector<uint32_t> q, pinv, lp, li, up, ui, prow, flags, void_slots;
    std::vector<double> lx, ux, udiag;  // the lead lane's factor values
    bool sn_dfs = false;
    uint32_t panels = 0;
};

// The lead lane's full factor of `vals` on order q with the reference's
// fill caps (a first pass capped at 3 x diag_fill, then the diagonal
// pivots). False when the matrix is singular.
bool factor_tape(uint32_t n, const uint32_t* col_ptr, const uint32_t* row_idx, const double* vals,
                 const std::vector<uint32_t>& q, Tape& out);

// The replay as a flat program for the shared-memory LU chain: per column,
// the scatter of A's column, each U entry's take with the axpy of its L
// column, and the pivot with the division of the column's L entries, in the
// replay's order (kernels/lane.zig:56-125). Entries are (row << 16 | slot)
// words, so every index must be below 2^16; false (empty program) when one
// is not.
//   SCAT  hdr = 1 | cnt << 4, then cnt x (w row << 16 | A slot)
//   TAKE  hdr = 2 | cnt << 4, then (i << 16 | U slot), then cnt x (L row << 16 | L slot)
//   PIV   hdr = 3 | flags << 4 | cnt << 8, then k, then cnt x (L row << 16 | L slot)
//   VOID  hdr = 4, then k (after column k's scatter and takes: a void column)
//   END   0
enum LuOp : uint32_t { kOpEnd = 0, kOpScat = 1, kOpTake = 2, kOpPiv = 3, kOpVoid = 4 };
bool lu_program(const Tape& t, const uint32_t* col_ptr, std::vector<uint32_t>& prog);

// The same replay as fixed 16-byte records (4 words each) for the shared
// LU chain: a record's entries update distinct rows, so its loads issue
// together, and the next record's address is known before the current one
// is decoded. Entries are (row << 16 | slot) words as in lu_program.
//   SCAT  x = 1 | n << 4; y, z, w: n x (w row << 16 | A slot), n = 1..3
//   TAKE  x = 2 | n << 4 | i << 16; y = U slot; z, w: n x (L row << 16 | L slot), n = 0..2
//   AXPY  x = 3 | n << 4; y, z, w: the TAKE's further entries, n = 1..3
//   PIV   x = 4 | n << 4 | flags << 8 | last << 12 | k << 16; y, z, w: n x (L row << 16 | L slot)
//   DIV   x = 5 | n << 4 | last << 12; y, z, w: the pivot's further entries
//   VOID  x = 6 | k << 16 (a void column, after its scatter and takes)
//   END   x = 0, twice (the second one is read ahead and never run)
// `last` marks the final record of a pivot column (its checks run there).
enum LuRec : uint32_t { kRecEnd = 0, kRecScat = 1, kRecTake = 2, kRecAxpy = 3, kRecPiv = 4, kRecDiv = 5, kRecVoid = 6 };
bool lu_records(const Tape& t, const uint32_t* col_ptr, std::vector<uint32_t>& rec);

// The triangular solves (luSolve's two sweeps, kernels/lane.zig:130-157) as
// 16-byte records in the same style: the forward sweep by columns k = 0 ..
// n-1, then the back sweep by columns k = n-1 .. 0.
//   FWD   x = 1 | n << 4 | k << 16; y, z, w: n x (row << 16 | L slot): y[row] -= L y[k], n = 1..3
//   FWDC  x = 2 | n << 4: the column's further entries
//   BWD   x = 3 | n << 4 | k << 16; y[k] /= U_kk, then y, z, w: n x (row << 16 | U slot):
//         y[row] -= U y[k], n = 0..3
//   BWDC  x = 4 | n << 4
//   END   x = 0, twice
// A column without L entries has no FWD record; every column has a BWD one.
enum SolveRec : uint32_t { kSolEnd = 0, kSolFwd = 1, kSolFwdC = 2, kSolBwd = 3, kSolBwdC = 4 };
bool solve_records(const Tape& t, std::vector<uint32_t>& rec);

// The banded streaming replay: when the replay of every column k touches
// only work-vector rows within k - band .. k + band (a ladder's elimination
// walks its chain), the work vector fits a ring of w_ring rows and the L
// entries an axpy can read (those of the previous `band` columns) a ring of
// l_ring slots, both in shared memory. The program streams through shared
// memory in chunks that end on op boundaries (chunk_pc, chunk_e: the
// program word and scatter-entry offsets of each chunk, n_chunks + 1 each),
// with the A slot of every scatter entry in program order (scat_slot).
struct BandPlan {
    uint32_t band = 0, w_ring = 0, l_ring = 0, max_words = 0, max_entries = 0;
    std::vector<uint32_t> chunk_pc, chunk_e, scat_slot;
    // The solves stream the factor by column blocks: solve_col[c] .. solve_col[c + 1]
    // is block c (at most kSolveCols columns, kSolveEntries L and U entries);
    // rowof[j] is the row whose right-hand side starts pivot position j.
    std::vector<uint32_t> solve_col, rowof;
};
constexpr uint32_t kSolveCols = 32, kSolveEntries = 64;
// False when the template does not qualify (a void column, a band past
// max_band, an L ring past max_l_ring, or no program).
bool band_plan(const Tape& t, const std::vector<uint32_t>& prog, uint32_t max_band, uint32_t max_l_ring,
               uint32_t chunk_words, uint32_t chunk_entries, BandPlan& out);

// The level schedule of the row-oriented ("pull") triangular solves of a
// large template, run by a whole CTA per 32-lane tile (lane_levels.cuh).
// Forward: y_i -= sum_j L_ij y_j over row i of L, rows grouped by level
// (a row's level is one more than the highest level among the rows it reads);
// backward: y_j = (y_j - sum_k U_jk y_k) / U_jj over row j of U, levels
// counted from the last row. Rows of a level are independent. Row entries
// are (column, factor slot) pairs in ascending column order.
struct LevelPlan {
    std::vector<uint32_t> fl_ptr, fl_rows;   // forward levels: rows fl_rows[fl_ptr[v] .. fl_ptr[v + 1])
    std::vector<uint32_t> bl_ptr, bl_rows;   // backward levels
    std::vector<uint32_t> rl_ptr, rl_ent;    // L by rows: 2 words per entry (j, slot)
    std::vector<uint32_t> ru_ptr, ru_ent;    // U by rows: 2 words per entry (k, slot)
};
void level_plan(const Tape& t, LevelPlan& out);

// The refactor's columns by levels, for a CTA that factors independent
// columns at once: a column's level is one more than the highest level
// among the columns whose L it reads (the rows of its U entries), so the
// columns of a level read only finished columns and write only their own.
// Each level's columns are dealt to G groups (G the largest power of two
// not above the level's columns or max_groups), greedily by their work, the
// heaviest first; a group takes its columns in tape order.
//   lv_ptr[v] .. lv_ptr[v + 1]   level v's G + 1 group starts in gp
//   gp[lv_ptr[v] + g]            first entry of group g's columns in cols
//   ustream[4 p .. 4 p + 3]      U entry p's row i and its L column's
//                                bounds lp[i], lp[i + 1] (and a zero): the
//                                refactor reads them in sequence instead of
//                                as a chain of dependent loads
struct ColPlan {
    std::vector<uint32_t> lv_ptr, gp, cols, ustream;
};
void col_plan(const Tape& t, uint32_t max_groups, ColPlan& out);

// A sweep of the level schedule in streaming order, for solves that stage
// the factor through shared memory: the sweep's entries in the order the
// levels read them (level by level, row by row, a row's entries by
// column), cut into chunks of at most `chunk` entries and `max_rows` rows
// that end on a row and start on a multiple of four entries (padding
// entries, column 0 and slot kNone, fill the gaps). With skip_empty the
// rows without entries are left out (a forward row without L entries keeps
// its value). False when a row is longer than `chunk`.
//   col[e], slot[e]  column and factor slot of entry e (kNone: padding);
//                    a column that a row of the same chunk computes is
//                    kStreamLocal | that row's position in the chunk
//   ch[c]            first entry of chunk c (n_chunks + 1 values)
//   meta[mo[c] ..]   chunk c's plan, a multiple of four words: ns, nr, its
//                    entries (ch[c + 1] - ch[c]), 0; the copy of chunk
//                    c + ahead (first entry, entries, first plan word,
//                    plan words; zeros past the last chunk);
//                    ns segments (runs of rows of one level inside the
//                    chunk) of 3 words: first row, end row (of the chunk's
//                    rows), and its longest row's entries times two, plus 1
//                    when the segment ends its level; the nr rows' indices;
//                    nr + 1 entry offsets (from ch[c]) of the rows
//   max_meta         the longest chunk plan, words
constexpr uint32_t kStreamLocal = 0x80000000u;
struct StreamPlan {
    uint32_t entries = 0, n_chunks = 0, max_meta = 0;
    std::vector<uint32_t> col, slot, ch, meta, mo;
};
bool stream_plan(const std::vector<uint32_t>& lev_ptr, const std::vector<uint32_t>& rows,
                 const std::vector<uint32_t>& row_ptr, const std::vector<uint32_t>& ent, uint32_t chunk,
                 uint32_t max_rows, uint32_t ahead, bool skip_empty, StreamPlan& out);

}  // namespace espl
