// The learned storage-format selector: a decision tree over derived structure
// features (csrc/selector_tree.h), fitted by sparseops_b200/selector.py on
// seeded matrices whose SpMV time was measured in every candidate format.
// The reference leaves the choice to a model outside its repository
// (src/sparse_features.cpp:1225 writes the features out for it).
#include <cmath>
#include <cstring>

#include "selector_tree.h"
#include "spops_internal.h"

namespace spops {

// the tree's inputs, in selector.py's DERIVED order
void derived_features(const spops_features_t& f, double* d) {
  const double rows = (double)f.rows, cols = (double)f.cols, nnz = (double)f.nnz, nd = (double)f.ndiags;
  const double ave = f.ave_nnz_row;
  const double mn = rows < cols ? rows : cols;
  d[0] = std::log2(rows + 1.0);
  d[1] = std::log2(nnz + 1.0);
  d[2] = ave;
  d[3] = f.std_nnz_row / (ave > 1e-12 ? ave : 1e-12);
  d[4] = (double)f.max_nnz_row / (ave > 1e-12 ? ave : 1e-12);
  d[5] = f.gini_row;
  d[6] = f.diag_close_ratio;
  d[7] = nd > 0 && mn > 0 ? nnz / (nd * mn) : 0.0;
  d[8] = std::log2(nd + 1.0);
  d[9] = f.nz_row_ratio;
  d[10] = f.p_ratio_row;
}

// the tree's choice and its spops_convert parameters; DIA only when the
// diagonals allow it (otherwise CSR)
void tree_select(const spops_features_t& f, spops_format_t* format, spops_format_params_t* params) {
  double d[11];
  derived_features(f, d);
  int k = 0;
  for (int steps = 0; steps < kSelectorNodes && kSelectorTree[k].feature >= 0; ++steps)
    k = d[kSelectorTree[k].feature] <= kSelectorTree[k].threshold ? kSelectorTree[k].left : kSelectorTree[k].right;
  int fmt = kSelectorTree[k].feature < 0 ? kSelectorTree[k].format : (int)SPOPS_FMT_CSR;
  std::memset(params, 0, sizeof(*params));
  const int64_t mn = f.rows < f.cols ? f.rows : f.cols;
  const bool dia_ok = f.ndiags > 0 && f.ndiags <= 10240 && (double)f.nnz >= 0.25 * (double)f.ndiags * (double)mn;
  switch (fmt) {
    case SPOPS_FMT_SELL_C_R:
      params->chunk = 32;
      params->alignment = 1;
      params->layout = SPOPS_COL_MAJOR;
      break;
    case SPOPS_FMT_SELL_C_SIGMA:
      params->chunk = 32;
      params->sigma = 4096;
      params->alignment = 1;
      params->layout = SPOPS_COL_MAJOR;
      break;
    case SPOPS_FMT_DIA:
      if (dia_ok) params->alignment = 1;
      else fmt = SPOPS_FMT_CSR;
      break;
    case SPOPS_FMT_CSR5:
      break;
    default:
      fmt = SPOPS_FMT_CSR;
  }
  *format = (spops_format_t)fmt;
}

}  // namespace spops

extern "C" spops_status_t spops_select_format_from_features(const spops_features_t* features, spops_format_t* format,
                                                           spops_format_params_t* params) {
  if (!features || !format || !params) return spops::fail(SPOPS_ERR_INVALID, "spops_select_format_from_features: null");
  spops::tree_select(*features, format, params);
  return SPOPS_OK;
}
