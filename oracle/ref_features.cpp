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

// Tile features (MTX::MtxLoad's tile counts, CalculateTilesFeatures via
// CalculateFeatures, and CalculateTilesExtraFeatures' distance_per_row_):
// scalars in the order of spops_tile_features_t (34 values), then the maps.
// tiles (num_blocks^2, row-major): nnz, uniq rows, uniq cols, max row nnz;
// ave and std row nnz.  Blocks (num_blocks each): RB nnz, RB max row nnz, CB
// nnz, CB max col nnz; RB ave / std, CB ave / std.
extern "C" int ref_tile_features(const char* mtx_path, double* sc, int64_t* tile_i, double* tile_d,
                                 int64_t* blk_i, double* blk_d) {
  MTX<int, double> m;
  if (!m.MtxLoad(mtx_path)) return -1;
  if (!m.CalculateFeatures()) return -2;
  if (!m.CalculateTilesExtraFeatures(mtx_path)) return -3;
  double v[] = {(double)m.t_num_blocks, (double)m.t_num_RB, (double)m.t_mod_RB, (double)m.t_num_CB,
                (double)m.t_mod_CB, (double)m.t_min_nnz_all_tiles_, (double)m.t_max_nnz_all_tiles_,
                (double)m.t_min_nnz_each_RB_, (double)m.t_max_nnz_each_RB_, (double)m.t_min_nnz_each_CB_,
                (double)m.t_max_nnz_each_CB_, m.t_nz_ratio_tiles_, m.t_ave_nnz_all_tiles, m.t_var_nnz_all_tiles,
                m.t_standard_dev_all_tiles, m.t_P_ratio_all_tiles_, m.t_Gini_all_tiles_, m.t_nz_ratio_RB_,
                m.t_ave_nnz_RB, m.t_var_nnz_RB, m.t_standard_dev_RB, m.t_P_ratio_RB_, m.t_Gini_RB_,
                m.t_nz_ratio_CB_, m.t_ave_nnz_CB, m.t_var_nnz_CB, m.t_standard_dev_CB, m.t_P_ratio_CB_,
                m.t_Gini_CB_, m.uniqR, m.uniqC, m.potReuseR, m.potReuseC, m.distance_per_row_};
  std::memcpy(sc, v, sizeof(v));
  const size_t B = (size_t)m.t_num_blocks, T = B * B;
  for (size_t i = 0; i < T; ++i) {
    tile_i[i] = m.nnz_by_Tiles_[i];
    tile_i[T + i] = m.uniq_RB[i];
    tile_i[2 * T + i] = m.uniq_CB[i];
    tile_i[3 * T + i] = m.max_rownnz_per_tile_[i];
    tile_d[i] = m.ave_rownnz_per_tile_[i];
    tile_d[T + i] = m.std_rownnz_per_tile_[i];
  }
  for (size_t i = 0; i < B; ++i) {
    blk_i[i] = m.nnz_by_RB_[i];
    blk_i[B + i] = m.max_rownnz_per_RB_[i];
    blk_i[2 * B + i] = m.nnz_by_CB_[i];
    blk_i[3 * B + i] = m.max_colnnz_per_CB_[i];
    blk_d[i] = m.ave_rownnz_per_RB_[i];
    blk_d[B + i] = m.std_rownnz_per_RB_[i];
    blk_d[2 * B + i] = m.ave_colnnz_per_CB_[i];
    blk_d[3 * B + i] = m.std_colnnz_per_CB_[i];
  }
  return 0;
}
