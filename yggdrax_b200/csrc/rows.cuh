// Row sort shared by the traversal schedules: every row of a CSR list is
// sorted ascending and widened into the index dtype (the canonical row order
// of _result_to_interactions / _result_to_neighbors,
// _interactions_impl.py:3561-3837).  Kernels live in traverse.cu.
#pragma once
#include "common.cuh"

namespace ygx {

struct RowSortScratch {
  uint32_t* n_big;      // 64 words: long-row and class counters
  int32_t* big_rows;    // stride entries
  int32_t* class_rows;  // one list of stride rows per size class
  uint32_t* bitmaps;    // one bitmap over [0, universe) per long-row CTA
  int64_t stride;       // rows of both tables of a pass together
};

// One list's rows: row r has cnt[r] raw int32 values at raw + (roff ?
// roff[r] : off[r]) and is written, sorted, at vals + off[r] (values minus
// rbase[r] when rbase is given); far rows also write the target r - rbase[r]
// and lvl[r] for every entry into tgts / lvls.
struct RowTable {
  int64_t rows;
  const int64_t* off;
  const int32_t* cnt;
  const int32_t* lvl;
  int32_t* raw;
  const int64_t* roff;
  const int32_t* rbase;
  void* vals;
  void* tgts;
  void* lvls;
};

// Carves the scratch for a pass over a table of `total` rows and one of `L`
// rows whose values lie in [0, total).
RowSortScratch carve_row_sort(Arena& a, int64_t total, int64_t L);

// Sorts the rows of both tables in one pass (b.rows may be 0): one size
// classification, one launch per size class and one long-row launch for
// both, so the longest rows of either start first and the rest fill in
// around them.  Does not synchronize.
int row_sort_pass(const RowSortScratch& s, const RowTable& a, const RowTable& b, int index_bits,
                  int64_t universe, cudaStream_t stream);

}  // namespace ygx
