// Decision tree of the learned format selector (spops_select_format mode 2).
// Generated by sparseops_b200/selector.py from measured SpMV times; do not edit.
// Inputs: derived features log2_rows, log2_nnz, ave_nnz_row, cv_nnz_row, max_over_ave_row, gini_row, diag_close_ratio, dia_fill, log2_ndiags, nz_row_ratio, p_ratio_row.
// Fitted on 34 seeded matrices (NVIDIA B200); on the 17 held-out ones it picks the
// timed choice for 12 and its SpMV takes 1.038x the best on average (1.250x at worst).
#pragma once

namespace spops {

struct SelectorNode {
  int feature;      // derived feature index, -1 for a leaf
  double threshold; // go left when feature <= threshold
  int left, right;  // child nodes
  int format;       // spops_format_t of a leaf
};

constexpr int kSelectorNodes = 13;
constexpr SelectorNode kSelectorTree[kSelectorNodes] = {
    {3, 0.10046588256955147, 1, 2, -1},
    {-1, 0.0, -1, -1, 6},
    {5, 0.21198075264692307, 3, 10, -1},
    {8, 16.906989097595215, 4, 7, -1},
    {3, 0.28153955191373825, 5, 6, -1},
    {-1, 0.0, -1, -1, 4},
    {-1, 0.0, -1, -1, 4},
    {2, 48.96647262573242, 8, 9, -1},
    {-1, 0.0, -1, -1, 5},
    {-1, 0.0, -1, -1, 0},
    {1, 23.596771240234375, 11, 12, -1},
    {-1, 0.0, -1, -1, 0},
    {-1, 0.0, -1, -1, 5},
};

}  // namespace spops
