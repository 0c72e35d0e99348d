// Launch-shape knobs chosen by the autotuner (yggdrax_b200/autotune.py).
// One process-wide table; each knob has a fixed set of legal values, so a
// bad value is rejected here and never reaches a kernel launch.
#include "sort.cuh"

namespace ygx {

Tune g_tune;

namespace {
bool legal(int knob, int v) {
  switch (knob) {
    case YGX_TUNE_SORT_RANK: return v >= 0 && v <= 2;
    case YGX_TUNE_SORT_SKEW: return v >= 1 && v <= 256;
    case YGX_TUNE_WALK_BLOCKS: return v >= 2 && v <= 6;
    case YGX_TUNE_REFIT_WARPS: return v == 2 || v == 4 || v == 8;
    case YGX_TUNE_ROW_GRID: return v == 4 || v == 8 || v == 16 || v == 32;
    case YGX_TUNE_SORT_TILE: return v >= 0 && v < kSortTileShapes;
    case YGX_TUNE_SPIN_LIMIT: return v >= 0 && v <= kSpinLimitMax;
    case YGX_TUNE_TARGET_BUDGET: return v >= 1 && v <= 4096;
    case YGX_TUNE_SORT_BITS: return v == kSortRadixBits || v == kWideBits;
    default: return false;
  }
}
int* slot(int knob) {
  switch (knob) {
    case YGX_TUNE_SORT_RANK: return &g_tune.sort_rank_policy;
    case YGX_TUNE_SORT_SKEW: return &g_tune.sort_skew_q8;
    case YGX_TUNE_WALK_BLOCKS: return &g_tune.walk_blocks_per_sm;
    case YGX_TUNE_REFIT_WARPS: return &g_tune.refit_warps;
    case YGX_TUNE_ROW_GRID: return &g_tune.row_grid_per_sm;
    case YGX_TUNE_SORT_TILE: return &g_tune.sort_tile;
    case YGX_TUNE_SPIN_LIMIT: return &g_tune.spin_limit;
    case YGX_TUNE_TARGET_BUDGET: return &g_tune.target_budget;
    case YGX_TUNE_SORT_BITS: return &g_tune.sort_bits;
    default: return nullptr;
  }
}
}  // namespace

}  // namespace ygx

extern "C" {

int ygx_tune_set(int knob, int value) {
  if (!ygx::legal(knob, value)) return YGX_ERR_ARG;
  *ygx::slot(knob) = value;
  return YGX_OK;
}

int ygx_tune_get(int knob, int* value) {
  int* p = ygx::slot(knob);
  if (!p || !value) return YGX_ERR_ARG;
  *value = *p;
  return YGX_OK;
}

}  // extern "C"
