// Decision tree of the learned format selector (spops_select_format mode 2).
// Generated by sparseops_b200/selector.py from measured SpMV times; do not edit.
// Not fitted yet: a single leaf (CSR).
#pragma once

namespace spops {

struct SelectorNode {
  int feature;      // derived feature index, -1 for a leaf
  double threshold; // go left when feature <= threshold
  int left, right;  // child nodes
  int format;       // spops_format_t of a leaf
};

constexpr int kSelectorNodes = 1;
constexpr SelectorNode kSelectorTree[kSelectorNodes] = {
    {-1, 0.0, -1, -1, 0},
};

}  // namespace spops
