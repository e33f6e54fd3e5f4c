// Oracle harness, test infrastructure only: the reference's own feature
// extraction, MTX::MtxLoad + MTX::CalculateFeatures (src/sparse_features.cpp),
// compiled from its source into this translation unit with the class's data
// members readable, so that the oracle's restatement and the device features
// can be compared with what the reference itself computes from a Matrix
// Market file.  Every system header the reference uses is included first so
// that only the reference's own declarations see the access change.
#include <ctype.h>
#include <immintrin.h>
#include <limits.h>
#include <malloc.h>
#include <math.h>
#include <memory.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>
#include <time.h>

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iostream>
#include <limits>
#include <map>
#include <numeric>
#include <parallel/algorithm>
#include <queue>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>

#define private public
#include "sparse_features.cpp"
#undef private

// Features in the order of spops_features_t (32 values); returns 0 on success.
extern "C" int ref_features(const char* mtx_path, double* out) {
  MTX<int, double> m;
  if (!m.MtxLoad(mtx_path)) return -1;
  if (!m.CalculateFeatures()) return -2;
  double v[] = {(double)m.num_rows, (double)m.num_cols, (double)m.num_nnzs, (double)m.nnz_lower_,
                (double)m.nnz_upper_, (double)m.nnz_diagonal_, (double)m.complete_ndiags,
                (double)m.min_nnz_each_row_, (double)m.max_nnz_each_row_, (double)m.min_nnz_each_col_,
                (double)m.max_nnz_each_col_, m.nnz_ratio_, m.diag_close_ratio_, m.pattern_symm_, m.value_symm_,
                m.nz_row_ratio_, m.ave_nnz_each_row_, m.var_nnz_each_row_, m.standard_dev_row_, m.P_ratio_row_,
                m.Gini_row_, m.nz_col_ratio_, m.ave_nnz_each_col_, m.var_nnz_each_col_, m.standard_dev_col_,
                m.P_ratio_col_, m.Gini_col_, m.diagonal_dominant_ratio_, m.max_value_offdiag_,
                m.max_value_diagonal_, m.row_variability_, m.col_variability_};
  std::memcpy(out, v, sizeof(v));
  return 0;
}
