/* C++ drop-in for the SparseOps operator API (the reference's include/SpOps.h),
 * running on one B200 through the C ABI of ../sparseops_b200.h.
 *
 * A caller of the reference switches its include path to this directory and
 * links libsparseops_b200.so; the structs (include/sparse_format.h:49-295 of
 * the reference), their field names and the call signatures stay the same:
 *
 *   SpOps_csr / _coo / _ell / _sell / _sell_c_sigma / _sell_c_R / _dia / _bsr / _csr5
 *       (alpha, const FMT_Matrix<I,V>& A, const V* x, beta, V* y)    host x, y
 *   coo_to_csr, csr_to_coo, csr_to_ell, csr_to_sell, csr_to_sell_c_sigma,
 *   csr_to_sell_c_R, csr_to_dia, csr_to_bsr, csr_to_csr5             host structs out
 *   delete_host_matrix(...)
 *   minhash_signatures_flat, lsh_candidate_pairs_vector,
 *   hierarchical_clustering_v0_fast                                   LeSpGEMM preprocessing
 *   read_coo_matrix, read_csr_matrix                                  Matrix Market files
 *   LeSpGEMM<sortOutput>(A, B, C, kernel_flag), HashSpGEMMTopK(A, C, top_k)
 *                                                                     row-wise SpGEMM (include/spgemm.h)
 *   MTX<I,V>: MtxLoad, CalculateFeatures, FeaturesPrint, FeaturesWrite ...  features
 *   read_<fmt>_matrix, coo_to_ell, sum_csr_duplicates, csr_transpose, csr_reorder_rows,
 *   csr_to_binary_pattern, minhash_estimated_jaccard, delete_<fmt>_matrix,
 *   Le_*_thread_* (kept settings only)
 *   CSR_VlengthCluster, csr_to_vlength_cluster, LeSpGEMM_VLength, vlength_cluster2csr
 *
 * What differs, and why:
 *   - Work runs on the GPU.  By default (CacheMode::Pattern) the first
 *     SpOps_csr call on a CSR struct uploads it and keeps the device copy of
 *     its pattern (row_offset, col_index and the analysis) keyed by the
 *     struct's first array pointer; every call then re-reads A.values from
 *     the host, as the reference reads its arrays on every call, so values
 *     changed in place are always seen.  Other formats are uploaded on every
 *     call.  CacheMode::All (set_cache(true)) keeps whole device copies of
 *     every format and moves only x and y: after changing a struct's arrays
 *     in place, call spops_b200::invalidate(ptr) (delete_host_matrix does it
 *     for you).  CacheMode::Off (set_cache(false)) uploads everything on
 *     every call.  A CSR pattern changed in place (same pointers and sizes)
 *     still needs invalidate(ptr) under the default mode.
 *   - Conversions run on the device; the returned host structs hold the
 *     reference's layouts (row-major chunks, reorder, chunk_len, ...) and the
 *     device copy used by SpOps_<fmt> keeps the device-native layout.
 *   - Errors throw std::runtime_error with the library's message where the
 *     reference calls exit() or asserts.
 *   - CSR5 tiles are the device's (32 lanes x 16 entries): tile_ptr/tile_desc
 *     are filled from them; y agrees with the reference, tile arrays do not.
 *   - Host arrays come from posix_memalign and are released with free(), as
 *     the reference's delete_array does; pointer-per-chunk tables use new[].
 */
#ifndef SPOPS_B200_CXX_SPOPS_H
#define SPOPS_B200_CXX_SPOPS_H

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "../sparseops_b200.h"

/* Defaults as the reference ships them (include/general_config.h,
 * include/plat_config.h); a caller's own definitions win. */
#ifndef CHUNK_SIZE
#define CHUNK_SIZE 4
#endif
#ifndef SELL_SIGMA
#define SELL_SIGMA 16384
#endif
#ifndef MAX_DIAG_NUM
#define MAX_DIAG_NUM 10240
#endif
#ifndef BSR_BlockDimRow
#define BSR_BlockDimRow 16
#endif
#ifndef SIMD_WIDTH
#define SIMD_WIDTH 256
#endif
#ifndef KERNEL_FLAG
#define KERNEL_FLAG 1
#endif

typedef enum { RowMajor = 0, ColMajor = 1 } LeadingDimension;

/* ------------------------------------------------------------- structs */
template <typename IndexType>
struct Matrix_Features {
  typedef IndexType index_type;
  IndexType num_rows;
  IndexType num_cols;
  IndexType num_nnzs;
  double sparsity;
  IndexType* partition = nullptr;
  double time, gflops, gbytes;
  int tag;
  int kernel_flag;
};

template <typename IndexType, typename ValueType>
struct COO_Matrix : public Matrix_Features<IndexType> {
  typedef IndexType index_type;
  typedef ValueType value_type;
  IndexType* row_index;
  IndexType* col_index;
  ValueType* values;
};

template <typename IndexType, typename ValueType>
struct CSR_Matrix : public Matrix_Features<IndexType> {
  typedef IndexType index_type;
  typedef ValueType value_type;
  IndexType* row_offset;
  IndexType* col_index;
  ValueType* values;
};

template <typename IndexType, typename ValueType>
struct BSR_Matrix : public Matrix_Features<IndexType> {
  typedef IndexType index_type;
  typedef ValueType value_type;
  IndexType blockDim_r;
  IndexType blockDim_c;
  IndexType blockNNZ;
  IndexType mb;
  IndexType nb;
  IndexType nnzb;
  IndexType* row_ptr;
  IndexType* block_colindex;
  ValueType* block_data;  // blocks row-major inside
};

template <typename IndexType, typename UIndexType, typename ValueType>
struct CSR5_Matrix : public CSR_Matrix<IndexType, ValueType> {
  IndexType sigma;
  IndexType omega;
  IndexType bit_y_offset;
  IndexType bit_scansum_offset;
  IndexType num_packets;
  IndexType num_offsets;
  IndexType _p;  // tiles
  IndexType tail_partition_start;
  UIndexType* tile_ptr;   // [_p + 1]
  UIndexType* tile_desc;  // [_p * omega]
  IndexType* tile_desc_offset_ptr;
  IndexType* tile_desc_offset;
  ValueType* calibrator;
};

template <typename IndexType, typename ValueType>
struct DIA_Matrix : public Matrix_Features<IndexType> {
  typedef IndexType index_type;
  typedef ValueType value_type;
  IndexType stride;
  IndexType complete_ndiags;
  long int* diag_offsets;
  ValueType* diag_data;  // [complete_ndiags * stride]
};

template <typename IndexType, typename ValueType>
struct ELL_Matrix : public Matrix_Features<IndexType> {
  typedef IndexType index_type;
  typedef ValueType value_type;
  LeadingDimension ld;
  IndexType max_row_width;
  IndexType min_row_width;
  IndexType* col_index;  // [num_rows * max_row_width], -1 = padding
  ValueType* values;
};

template <typename IndexType, typename ValueType>
struct S_ELL_Matrix : public Matrix_Features<IndexType> {
  typedef IndexType index_type;
  typedef ValueType value_type;
  IndexType sliceWidth;
  IndexType chunk_num;
  IndexType alignment;
  IndexType* row_width;    // [chunk_num]
  IndexType** col_index;   // [chunk_num][sliceWidth * row_width[c]], row-major
  ValueType** values;
};

template <typename IndexType, typename ValueType>
struct SELL_C_Sigma_Matrix : public Matrix_Features<IndexType> {
  typedef IndexType index_type;
  typedef ValueType value_type;
  IndexType sliceWidth_Sigma;
  IndexType chunkWidth_C;
  IndexType sliceNum;
  IndexType chunkNum;
  IndexType validchunkNum;
  IndexType chunk_num_per_slice;
  IndexType alignment;
  IndexType* reorder;      // [num_rows]: stored row -> original row
  IndexType* chunk_len;    // [validchunkNum]
  IndexType** col_index;   // [validchunkNum][chunkWidth_C * chunk_len[c]], row-major
  ValueType** values;
};

template <typename IndexType, typename ValueType>
struct SELL_C_R_Matrix : public Matrix_Features<IndexType> {
  typedef IndexType index_type;
  typedef ValueType value_type;
  IndexType chunkWidth_C;
  IndexType validchunkNum;
  IndexType alignment;
  IndexType* reorder;
  IndexType* chunk_len;
  IndexType** col_index;
  ValueType** values;
};

template <typename IndexType, typename ValueType>
struct CandidatePair {
  IndexType i;
  IndexType j;
  ValueType score;
};

/* --------------------------------------------------------------- state */
namespace spops_b200 {
namespace detail {

struct Entry {
  spops_matrix_t h = nullptr;
  int64_t rows = 0, cols = 0, nnz = 0;
};

enum class CacheModeImpl { Off, Pattern, All };

struct State {
  std::mutex mu;
  int device = 0;
  CacheModeImpl cache = CacheModeImpl::Pattern;
  spops_context_t ctx = nullptr;
  std::unordered_map<const void*, Entry> handles;
};

// never destroyed: at process exit the CUDA runtime may already be gone
inline State& state() {
  static State* s = new State();
  return *s;
}

inline void check(spops_status_t s, const char* what) {
  if (s != SPOPS_OK) {
    const char* m = spops_last_error();
    throw std::runtime_error(std::string(what) + ": " + spops_status_string(s) + (m ? std::string(": ") + m : ""));
  }
}

inline spops_context_t ctx() {
  State& s = state();
  std::lock_guard<std::mutex> lk(s.mu);
  if (!s.ctx) check(spops_create(&s.ctx, s.device, nullptr), "spops_create");
  return s.ctx;
}

// the argument's own type, kept out of template argument deduction (so that
// size arguments given as int literals work with 64-bit index types)
template <typename T>
struct same {
  typedef T type;
};
template <typename T>
using same_t = typename same<T>::type;

template <typename I>
constexpr spops_index_t itype() {
  static_assert(std::is_integral<I>::value && (sizeof(I) == 4 || sizeof(I) == 8), "index type: 32- or 64-bit integer");
  return sizeof(I) == 4 ? SPOPS_INDEX_I32 : SPOPS_INDEX_I64;
}

template <typename V>
constexpr spops_value_t vtype() {
  static_assert(std::is_same<V, float>::value || std::is_same<V, double>::value, "value type: float or double");
  return std::is_same<V, float>::value ? SPOPS_VALUE_F32 : SPOPS_VALUE_F64;
}

template <typename T>
inline T* host_alloc(int64_t n) {
  void* p = nullptr;
  const size_t bytes = (size_t)(n > 0 ? n : 1) * sizeof(T);
  if (posix_memalign(&p, 64, bytes) != 0) throw std::bad_alloc();
  return static_cast<T*>(p);
}

inline void release(const void* key) {
  State& s = state();
  std::lock_guard<std::mutex> lk(s.mu);
  auto it = s.handles.find(key);
  if (it != s.handles.end()) {
    spops_matrix_destroy(it->second.h);
    s.handles.erase(it);
  }
}

// cached device handle for `key`, or nullptr (sizes must match)
inline spops_matrix_t find(const void* key, int64_t rows, int64_t cols, int64_t nnz) {
  State& s = state();
  std::lock_guard<std::mutex> lk(s.mu);
  auto it = s.handles.find(key);
  if (it == s.handles.end()) return nullptr;
  if (it->second.rows == rows && it->second.cols == cols && it->second.nnz == nnz) return it->second.h;
  spops_matrix_destroy(it->second.h);
  s.handles.erase(it);
  return nullptr;
}

inline void put(const void* key, spops_matrix_t h, int64_t rows, int64_t cols, int64_t nnz) {
  State& s = state();
  std::lock_guard<std::mutex> lk(s.mu);
  auto it = s.handles.find(key);
  if (it != s.handles.end() && it->second.h != h) spops_matrix_destroy(it->second.h);
  s.handles[key] = Entry{h, rows, cols, nnz};
}

// whole device copies of any format are kept between calls
inline bool caching() { return state().cache == CacheModeImpl::All; }
// CSR device copies are kept (their values re-read from the host per call
// unless caching() holds)
inline bool caching_csr() { return state().cache != CacheModeImpl::Off; }

// run y = alpha*A*x + beta*y with host vectors on handle h.  A handle this
// call created (fresh) is cached under `key` when `keep`, or destroyed; a
// handle found in the cache stays there.
inline void spmv_host(spops_matrix_t h, bool fresh, const void* key, double alpha, const void* x, double beta,
                      void* y, const char* what, int64_t rows, int64_t cols, int64_t nnz, bool keep) {
  spops_status_t s = spops_spmv_host(ctx(), alpha, h, x, beta, y);
  if (fresh) {
    if (keep) put(key, h, rows, cols, nnz); else spops_matrix_destroy(h);
  }
  check(s, what);
}

template <typename T>
inline T* fetch(spops_matrix_t h, spops_array_t which, int64_t* count) {
  const void* dp = nullptr;
  int64_t n = 0;
  int32_t eb = 0;
  check(spops_matrix_array(h, which, &dp, &n, &eb), "spops_matrix_array");
  if (n > 0 && eb != (int32_t)sizeof(T)) throw std::runtime_error("spops_b200: array element size mismatch");
  T* out = host_alloc<T>(n);
  if (n > 0) check(spops_matrix_download(ctx(), h, which, out, n), "spops_matrix_download");
  if (count) *count = n;
  return out;
}

inline spops_matrix_info_t info(spops_matrix_t h) {
  spops_matrix_info_t i;
  check(spops_matrix_info(h, &i), "spops_matrix_info");
  return i;
}

template <typename I, typename V>
inline spops_matrix_t upload_csr(const CSR_Matrix<I, V>& A) {
  spops_matrix_t h = nullptr;
  check(spops_csr_create(ctx(), &h, A.num_rows, A.num_cols, A.num_nnzs, A.row_offset, A.col_index, A.values,
                         itype<I>(), vtype<V>(), SPOPS_MEM_HOST),
        "spops_csr_create");
  return h;
}

// pattern-only handle: the value slot borrows the column array (never read)
template <typename I>
inline spops_matrix_t upload_pattern(const I* rowptr, const I* col, I n) {
  spops_matrix_t h = nullptr;
  const int64_t nnz = n > 0 ? (int64_t)rowptr[n] : 0;
  const int64_t cols = sizeof(I) == 4 ? (int64_t)INT32_MAX : ((int64_t)1 << 40);  // no column bound is needed
  check(spops_csr_create(ctx(), &h, n, cols, nnz, rowptr, col, col, itype<I>(),
                         sizeof(I) == 4 ? SPOPS_VALUE_F32 : SPOPS_VALUE_F64, SPOPS_MEM_HOST),
        "spops_csr_create");
  return h;
}

inline spops_matrix_t convert(spops_matrix_t csr, spops_format_t f, const spops_format_params_t& p) {
  spops_matrix_t out = nullptr;
  check(spops_convert(ctx(), csr, f, &p, &out), "spops_convert");
  return out;
}

template <typename I, typename V, typename M>
inline void set_features(M& m, int64_t rows, int64_t cols, int64_t nnz) {
  std::memset(static_cast<void*>(&m), 0, sizeof(M));
  m.num_rows = (I)rows;
  m.num_cols = (I)cols;
  m.num_nnzs = (I)nnz;
  m.sparsity = (rows > 0 && cols > 0) ? (double)nnz / ((double)rows * (double)cols) : 0.0;
}

// split concatenated row-major chunks into one host array per chunk
template <typename T, typename I>
inline T** split_chunks(const T* all, int64_t total, const I* len, int64_t nchunks, int64_t C) {
  int64_t need = 0;
  for (int64_t c = 0; c < nchunks; ++c) need += C * (int64_t)len[c];
  if (need != total) throw std::runtime_error("spops_b200: padded arrays do not match the chunk widths");
  T** out = new T*[(size_t)(nchunks > 0 ? nchunks : 1)];
  int64_t at = 0;
  for (int64_t c = 0; c < nchunks; ++c) {
    const int64_t m = C * (int64_t)len[c];
    out[c] = host_alloc<T>(m);
    if (m) std::memcpy(out[c], all + at, (size_t)m * sizeof(T));
    at += m;
  }
  return out;
}

template <typename T, typename I>
inline std::vector<T> join_chunks(T* const* parts, const I* len, int64_t nchunks, int64_t C) {
  std::vector<T> all;
  for (int64_t c = 0; c < nchunks; ++c) all.insert(all.end(), parts[c], parts[c] + C * (int64_t)len[c]);
  return all;
}

}  // namespace detail

/* Device used by the calls below (before the first call). */
inline void set_device(int device) { detail::state().device = device; }
/* What the SpOps_<fmt> calls keep on the device between calls:
 *   Off      nothing: every call uploads the struct (the reference's per-call read);
 *   Pattern  (default) CSR patterns and their analysis; A.values re-read from
 *            the host on every call; other formats uploaded on every call;
 *   All      whole device copies of every format; only x and y move.  Host
 *            arrays changed in place need invalidate(ptr). */
enum class CacheMode { Off, Pattern, All };
inline void set_cache_mode(CacheMode m) {
  detail::state().cache = m == CacheMode::Off ? detail::CacheModeImpl::Off
                          : m == CacheMode::All ? detail::CacheModeImpl::All
                                                : detail::CacheModeImpl::Pattern;
}
inline CacheMode cache_mode() {
  const detail::CacheModeImpl m = detail::state().cache;
  return m == detail::CacheModeImpl::Off ? CacheMode::Off
         : m == detail::CacheModeImpl::All ? CacheMode::All
                                           : CacheMode::Pattern;
}
/* set_cache(true): CacheMode::All; set_cache(false): CacheMode::Off. */
inline void set_cache(bool on) { set_cache_mode(on ? CacheMode::All : CacheMode::Off); }
/* Drop the device copy of the matrix whose first array is `key` (e.g.
 * A.row_offset, coo.row_index, sell.reorder) after changing it in place. */
inline void invalidate(const void* key) { detail::release(key); }

}  // namespace spops_b200

/* ---------------------------------------------------------------- SpMV */
template <typename IndexType, typename ValueType>
void SpOps_csr(const ValueType alpha, const CSR_Matrix<IndexType, ValueType>& A, const ValueType* x,
               const ValueType beta, ValueType* y) {
  namespace d = spops_b200::detail;
  spops_matrix_t h = d::caching_csr() ? d::find(A.row_offset, A.num_rows, A.num_cols, A.num_nnzs) : nullptr;
  const bool fresh = h == nullptr;
  if (!h) h = d::upload_csr(A);
  else if (!d::caching()) d::check(spops_csr_upload_values(d::ctx(), h, A.values), "spops_csr_upload_values");
  d::spmv_host(h, fresh, A.row_offset, alpha, x, beta, y, "SpOps_csr", A.num_rows, A.num_cols, A.num_nnzs,
               d::caching_csr());
}

template <typename IndexType, typename ValueType>
void SpOps_coo(const ValueType alpha, const COO_Matrix<IndexType, ValueType>& A, const ValueType* x,
               const ValueType beta, ValueType* y) {
  namespace d = spops_b200::detail;
  spops_matrix_t h = !d::caching() ? nullptr : d::find(A.row_index, A.num_rows, A.num_cols, A.num_nnzs);
  const bool fresh = h == nullptr;
  if (!h)
    d::check(spops_coo_create(d::ctx(), &h, A.num_rows, A.num_cols, A.num_nnzs, A.row_index, A.col_index, A.values,
                              d::itype<IndexType>(), d::vtype<ValueType>(), SPOPS_MEM_HOST),
             "spops_coo_create");
  d::spmv_host(h, fresh, A.row_index, alpha, x, beta, y, "SpOps_coo", A.num_rows, A.num_cols, A.num_nnzs,
               d::caching());
}

template <typename IndexType, typename ValueType>
void SpOps_ell(const ValueType alpha, const ELL_Matrix<IndexType, ValueType>& A, const ValueType* x,
               const ValueType beta, ValueType* y) {
  namespace d = spops_b200::detail;
  spops_matrix_t h = !d::caching() ? nullptr : d::find(A.col_index, A.num_rows, A.num_cols, A.num_nnzs);
  const bool fresh = h == nullptr;
  if (!h) {
    const IndexType w = A.max_row_width;
    d::check(spops_padded_create(d::ctx(), &h, SPOPS_FMT_ELL, A.num_rows, A.num_cols, A.num_nnzs,
                                 A.num_rows > 0 ? A.num_rows : 1, 0, 1,
                                 A.ld == ColMajor ? SPOPS_COL_MAJOR : SPOPS_ROW_MAJOR, nullptr, &w, 1, A.col_index,
                                 A.values, (int64_t)A.num_rows * w, d::itype<IndexType>(), d::vtype<ValueType>(),
                                 SPOPS_MEM_HOST),
             "spops_padded_create");
  }
  d::spmv_host(h, fresh, A.col_index, alpha, x, beta, y, "SpOps_ell", A.num_rows, A.num_cols, A.num_nnzs,
               d::caching());
}

template <typename IndexType, typename ValueType>
void SpOps_sell(const ValueType alpha, const S_ELL_Matrix<IndexType, ValueType>& A, const ValueType* x,
                const ValueType beta, ValueType* y) {
  namespace d = spops_b200::detail;
  spops_matrix_t h = !d::caching() ? nullptr : d::find(A.row_width, A.num_rows, A.num_cols, A.num_nnzs);
  const bool fresh = h == nullptr;
  if (!h) {
    const std::vector<IndexType> col = d::join_chunks(A.col_index, A.row_width, A.chunk_num, A.sliceWidth);
    const std::vector<ValueType> val = d::join_chunks(A.values, A.row_width, A.chunk_num, A.sliceWidth);
    d::check(spops_padded_create(d::ctx(), &h, SPOPS_FMT_SELL, A.num_rows, A.num_cols, A.num_nnzs, A.sliceWidth, 0,
                                 A.alignment, SPOPS_ROW_MAJOR, nullptr, A.row_width, A.chunk_num, col.data(),
                                 val.data(), (int64_t)col.size(), d::itype<IndexType>(), d::vtype<ValueType>(),
                                 SPOPS_MEM_HOST),
             "spops_padded_create");
  }
  d::spmv_host(h, fresh, A.row_width, alpha, x, beta, y, "SpOps_sell", A.num_rows, A.num_cols, A.num_nnzs,
               d::caching());
}

template <typename IndexType, typename ValueType>
void SpOps_sell_c_sigma(const ValueType alpha, const SELL_C_Sigma_Matrix<IndexType, ValueType>& A, const ValueType* x,
                        const ValueType beta, ValueType* y) {
  namespace d = spops_b200::detail;
  spops_matrix_t h = !d::caching() ? nullptr : d::find(A.reorder, A.num_rows, A.num_cols, A.num_nnzs);
  const bool fresh = h == nullptr;
  if (!h) {
    const std::vector<IndexType> col = d::join_chunks(A.col_index, A.chunk_len, A.validchunkNum, A.chunkWidth_C);
    const std::vector<ValueType> val = d::join_chunks(A.values, A.chunk_len, A.validchunkNum, A.chunkWidth_C);
    d::check(spops_padded_create(d::ctx(), &h, SPOPS_FMT_SELL_C_SIGMA, A.num_rows, A.num_cols, A.num_nnzs,
                                 A.chunkWidth_C, A.sliceWidth_Sigma, A.alignment, SPOPS_ROW_MAJOR, A.reorder,
                                 A.chunk_len, A.validchunkNum, col.data(), val.data(), (int64_t)col.size(),
                                 d::itype<IndexType>(), d::vtype<ValueType>(), SPOPS_MEM_HOST),
             "spops_padded_create");
  }
  d::spmv_host(h, fresh, A.reorder, alpha, x, beta, y, "SpOps_sell_c_sigma", A.num_rows, A.num_cols, A.num_nnzs,
               d::caching());
}

template <typename IndexType, typename ValueType>
void SpOps_sell_c_R(const ValueType alpha, const SELL_C_R_Matrix<IndexType, ValueType>& A, const ValueType* x,
                    const ValueType beta, ValueType* y) {
  namespace d = spops_b200::detail;
  spops_matrix_t h = !d::caching() ? nullptr : d::find(A.reorder, A.num_rows, A.num_cols, A.num_nnzs);
  const bool fresh = h == nullptr;
  if (!h) {
    const std::vector<IndexType> col = d::join_chunks(A.col_index, A.chunk_len, A.validchunkNum, A.chunkWidth_C);
    const std::vector<ValueType> val = d::join_chunks(A.values, A.chunk_len, A.validchunkNum, A.chunkWidth_C);
    d::check(spops_padded_create(d::ctx(), &h, SPOPS_FMT_SELL_C_R, A.num_rows, A.num_cols, A.num_nnzs,
                                 A.chunkWidth_C, A.num_rows, A.alignment, SPOPS_ROW_MAJOR, A.reorder, A.chunk_len,
                                 A.validchunkNum, col.data(), val.data(), (int64_t)col.size(), d::itype<IndexType>(),
                                 d::vtype<ValueType>(), SPOPS_MEM_HOST),
             "spops_padded_create");
  }
  d::spmv_host(h, fresh, A.reorder, alpha, x, beta, y, "SpOps_sell_c_R", A.num_rows, A.num_cols, A.num_nnzs,
               d::caching());
}

template <typename IndexType, typename ValueType>
void SpOps_dia(const ValueType alpha, const DIA_Matrix<IndexType, ValueType>& A, const ValueType* x,
               const ValueType beta, ValueType* y) {
  namespace d = spops_b200::detail;
  static_assert(sizeof(long int) == 8, "diag_offsets must be 64-bit");
  spops_matrix_t h = !d::caching() ? nullptr : d::find(A.diag_offsets, A.num_rows, A.num_cols, A.num_nnzs);
  const bool fresh = h == nullptr;
  if (!h)
    d::check(spops_dia_create(d::ctx(), &h, A.num_rows, A.num_cols, A.num_nnzs, A.complete_ndiags, A.stride,
                              reinterpret_cast<const int64_t*>(A.diag_offsets), A.diag_data, d::vtype<ValueType>(),
                              SPOPS_MEM_HOST),
             "spops_dia_create");
  d::spmv_host(h, fresh, A.diag_offsets, alpha, x, beta, y, "SpOps_dia", A.num_rows, A.num_cols, A.num_nnzs,
               d::caching());
}

template <typename IndexType, typename ValueType>
void SpOps_bsr(const ValueType alpha, const BSR_Matrix<IndexType, ValueType>& A, const ValueType* x,
               const ValueType beta, ValueType* y) {
  namespace d = spops_b200::detail;
  spops_matrix_t h = !d::caching() ? nullptr : d::find(A.row_ptr, A.num_rows, A.num_cols, A.num_nnzs);
  const bool fresh = h == nullptr;
  if (!h)
    d::check(spops_bsr_create(d::ctx(), &h, A.num_rows, A.num_cols, A.num_nnzs, A.blockDim_r, A.blockDim_c, A.nnzb,
                              A.row_ptr, A.block_colindex, A.block_data, d::itype<IndexType>(), d::vtype<ValueType>(),
                              SPOPS_MEM_HOST),
             "spops_bsr_create");
  d::spmv_host(h, fresh, A.row_ptr, alpha, x, beta, y, "SpOps_bsr", A.num_rows, A.num_cols, A.num_nnzs,
               d::caching());
}

template <typename IndexType, typename UIndexType, typename ValueType>
void SpOps_csr5(const ValueType alpha, const CSR5_Matrix<IndexType, UIndexType, ValueType>& A, const ValueType* x,
                const ValueType beta, ValueType* y) {
  namespace d = spops_b200::detail;
  spops_matrix_t h = !d::caching() ? nullptr : d::find(A.tile_ptr, A.num_rows, A.num_cols, A.num_nnzs);
  const bool fresh = h == nullptr;
  if (!h) {  // rebuild the device tiles from the CSR arrays the struct carries
    spops_matrix_t c = d::upload_csr(static_cast<const CSR_Matrix<IndexType, ValueType>&>(A));
    spops_format_params_t p;
    std::memset(&p, 0, sizeof(p));
    spops_status_t s = spops_convert(d::ctx(), c, SPOPS_FMT_CSR5, &p, &h);
    spops_matrix_destroy(c);
    d::check(s, "spops_convert");
  }
  d::spmv_host(h, fresh, A.tile_ptr, alpha, x, beta, y, "SpOps_csr5", A.num_rows, A.num_cols, A.num_nnzs,
               d::caching());
}

/* ---------------------------------------------------------- conversions */
template <class IndexType, class ValueType>
CSR_Matrix<IndexType, ValueType> coo_to_csr(const COO_Matrix<IndexType, ValueType>& coo, bool compact = false) {
  namespace d = spops_b200::detail;
  spops_matrix_t hc = nullptr, h = nullptr;
  d::check(spops_coo_create(d::ctx(), &hc, coo.num_rows, coo.num_cols, coo.num_nnzs, coo.row_index, coo.col_index,
                            coo.values, d::itype<IndexType>(), d::vtype<ValueType>(), SPOPS_MEM_HOST),
           "spops_coo_create");
  spops_status_t s = spops_coo_to_csr(d::ctx(), hc, compact ? 1 : 0, &h);
  spops_matrix_destroy(hc);
  d::check(s, "spops_coo_to_csr");
  const spops_matrix_info_t i = d::info(h);
  CSR_Matrix<IndexType, ValueType> csr;
  d::set_features<IndexType, ValueType>(csr, i.rows, i.cols, i.nnz);
  csr.row_offset = d::fetch<IndexType>(h, SPOPS_ARR_ROW, nullptr);
  csr.col_index = d::fetch<IndexType>(h, SPOPS_ARR_COL, nullptr);
  csr.values = d::fetch<ValueType>(h, SPOPS_ARR_VAL, nullptr);
  if (d::caching_csr()) d::put(csr.row_offset, h, i.rows, i.cols, i.nnz); else spops_matrix_destroy(h);
  return csr;
}

template <class IndexType, class ValueType>
COO_Matrix<IndexType, ValueType> csr_to_coo(const CSR_Matrix<IndexType, ValueType>& csr) {
  namespace d = spops_b200::detail;
  spops_matrix_t c = d::upload_csr(csr);
  spops_format_params_t p;
  std::memset(&p, 0, sizeof(p));
  spops_matrix_t h = nullptr;
  spops_status_t s = spops_convert(d::ctx(), c, SPOPS_FMT_COO, &p, &h);
  spops_matrix_destroy(c);
  d::check(s, "spops_convert");
  COO_Matrix<IndexType, ValueType> coo;
  d::set_features<IndexType, ValueType>(coo, csr.num_rows, csr.num_cols, csr.num_nnzs);
  coo.row_index = d::fetch<IndexType>(h, SPOPS_ARR_ROW, nullptr);
  coo.col_index = d::fetch<IndexType>(h, SPOPS_ARR_COL, nullptr);
  coo.values = d::fetch<ValueType>(h, SPOPS_ARR_VAL, nullptr);
  if (d::caching()) d::put(coo.row_index, h, csr.num_rows, csr.num_cols, csr.num_nnzs); else spops_matrix_destroy(h);
  return coo;
}

template <class IndexType, class ValueType>
ELL_Matrix<IndexType, ValueType> csr_to_ell(const CSR_Matrix<IndexType, ValueType>& csr,
                                            const LeadingDimension ld = RowMajor) {
  namespace d = spops_b200::detail;
  spops_matrix_t c = d::upload_csr(csr);
  spops_format_params_t p;
  std::memset(&p, 0, sizeof(p));
  p.layout = ld == ColMajor ? SPOPS_COL_MAJOR : SPOPS_ROW_MAJOR;
  spops_matrix_t h = nullptr;
  spops_status_t s = spops_convert(d::ctx(), c, SPOPS_FMT_ELL, &p, &h);
  spops_matrix_destroy(c);
  d::check(s, "spops_convert");
  const spops_matrix_info_t i = d::info(h);
  ELL_Matrix<IndexType, ValueType> ell;
  d::set_features<IndexType, ValueType>(ell, csr.num_rows, csr.num_cols, csr.num_nnzs);
  ell.ld = ld;
  ell.max_row_width = (IndexType)i.extra[0];
  ell.min_row_width = (IndexType)i.extra[1];
  ell.col_index = d::fetch<IndexType>(h, SPOPS_ARR_COL, nullptr);
  ell.values = d::fetch<ValueType>(h, SPOPS_ARR_VAL, nullptr);
  if (d::caching()) d::put(ell.col_index, h, csr.num_rows, csr.num_cols, csr.num_nnzs); else spops_matrix_destroy(h);
  return ell;
}

namespace spops_b200 {
namespace detail {
// padded SELL-type conversion: host arrays in the reference (row-major)
// layout from one conversion, the cached device copy column-major
inline void sell_pair(spops_matrix_t c, spops_format_t f, spops_format_params_t p, spops_matrix_t* host_side,
                      spops_matrix_t* dev_side) {
  p.layout = SPOPS_ROW_MAJOR;
  *host_side = convert(c, f, p);
  p.layout = SPOPS_COL_MAJOR;
  spops_status_t s = spops_convert(ctx(), c, f, &p, dev_side);
  if (s != SPOPS_OK) {
    spops_matrix_destroy(*host_side);
    check(s, "spops_convert");
  }
}
}  // namespace detail
}  // namespace spops_b200

template <class IndexType, class ValueType>
S_ELL_Matrix<IndexType, ValueType> csr_to_sell(const CSR_Matrix<IndexType, ValueType>& csr, FILE* fp_feature,
                                               const int chunkwidth = CHUNK_SIZE,
                                               const spops_b200::detail::same_t<IndexType> alignment =
                                                   (SIMD_WIDTH / 8 / sizeof(ValueType))) {
  namespace d = spops_b200::detail;
  (void)fp_feature;
  spops_matrix_t c = d::upload_csr(csr), hh = nullptr, hd = nullptr;
  spops_format_params_t p;
  std::memset(&p, 0, sizeof(p));
  p.chunk = chunkwidth;
  p.alignment = alignment;
  try {
    d::sell_pair(c, SPOPS_FMT_SELL, p, &hh, &hd);
  } catch (...) {
    spops_matrix_destroy(c);
    throw;
  }
  spops_matrix_destroy(c);
  const spops_matrix_info_t i = d::info(hh);
  S_ELL_Matrix<IndexType, ValueType> s;
  d::set_features<IndexType, ValueType>(s, csr.num_rows, csr.num_cols, csr.num_nnzs);
  s.sliceWidth = (IndexType)chunkwidth;
  s.chunk_num = (IndexType)i.extra[0];
  s.alignment = alignment;
  s.row_width = d::fetch<IndexType>(hh, SPOPS_ARR_CHUNK_LEN, nullptr);
  int64_t ncol = 0, nval = 0;
  IndexType* col = d::fetch<IndexType>(hh, SPOPS_ARR_COL, &ncol);
  ValueType* val = d::fetch<ValueType>(hh, SPOPS_ARR_VAL, &nval);
  s.col_index = d::split_chunks(col, ncol, s.row_width, s.chunk_num, chunkwidth);
  s.values = d::split_chunks(val, nval, s.row_width, s.chunk_num, chunkwidth);
  std::free(col);
  std::free(val);
  spops_matrix_destroy(hh);
  if (d::caching()) d::put(s.row_width, hd, csr.num_rows, csr.num_cols, csr.num_nnzs); else spops_matrix_destroy(hd);
  return s;
}

template <class IndexType, class ValueType>
SELL_C_Sigma_Matrix<IndexType, ValueType> csr_to_sell_c_sigma(
    const CSR_Matrix<IndexType, ValueType>& csr, FILE* fp_feature, const int slicewidth = SELL_SIGMA,
    const int chunkwidth = CHUNK_SIZE,
    const spops_b200::detail::same_t<IndexType> alignment = (SIMD_WIDTH / 8 / sizeof(ValueType))) {
  namespace d = spops_b200::detail;
  (void)fp_feature;
  spops_matrix_t c = d::upload_csr(csr), hh = nullptr, hd = nullptr;
  spops_format_params_t p;
  std::memset(&p, 0, sizeof(p));
  p.sigma = slicewidth;
  p.chunk = chunkwidth;
  p.alignment = alignment;
  try {
    d::sell_pair(c, SPOPS_FMT_SELL_C_SIGMA, p, &hh, &hd);
  } catch (...) {
    spops_matrix_destroy(c);
    throw;
  }
  spops_matrix_destroy(c);
  const spops_matrix_info_t i = d::info(hh);
  SELL_C_Sigma_Matrix<IndexType, ValueType> s;
  d::set_features<IndexType, ValueType>(s, csr.num_rows, csr.num_cols, csr.num_nnzs);
  s.sliceWidth_Sigma = (IndexType)slicewidth;
  s.chunkWidth_C = (IndexType)chunkwidth;
  s.sliceNum = (IndexType)i.extra[0];
  s.chunkNum = (IndexType)i.extra[1];
  s.validchunkNum = (IndexType)i.extra[2];
  s.chunk_num_per_slice = (IndexType)i.extra[3];
  s.alignment = alignment;
  s.reorder = d::fetch<IndexType>(hh, SPOPS_ARR_REORDER, nullptr);
  s.chunk_len = d::fetch<IndexType>(hh, SPOPS_ARR_CHUNK_LEN, nullptr);
  int64_t ncol = 0, nval = 0;
  IndexType* col = d::fetch<IndexType>(hh, SPOPS_ARR_COL, &ncol);
  ValueType* val = d::fetch<ValueType>(hh, SPOPS_ARR_VAL, &nval);
  s.col_index = d::split_chunks(col, ncol, s.chunk_len, s.validchunkNum, chunkwidth);
  s.values = d::split_chunks(val, nval, s.chunk_len, s.validchunkNum, chunkwidth);
  std::free(col);
  std::free(val);
  spops_matrix_destroy(hh);
  if (d::caching()) d::put(s.reorder, hd, csr.num_rows, csr.num_cols, csr.num_nnzs); else spops_matrix_destroy(hd);
  return s;
}

template <class IndexType, class ValueType>
SELL_C_R_Matrix<IndexType, ValueType> csr_to_sell_c_R(const CSR_Matrix<IndexType, ValueType>& csr, FILE* fp_feature,
                                                      const int chunkwidth = CHUNK_SIZE,
                                                      const spops_b200::detail::same_t<IndexType> alignment =
                                                          (SIMD_WIDTH / 8 / sizeof(ValueType))) {
  namespace d = spops_b200::detail;
  (void)fp_feature;
  spops_matrix_t c = d::upload_csr(csr), hh = nullptr, hd = nullptr;
  spops_format_params_t p;
  std::memset(&p, 0, sizeof(p));
  p.chunk = chunkwidth;
  p.alignment = alignment;
  try {
    d::sell_pair(c, SPOPS_FMT_SELL_C_R, p, &hh, &hd);
  } catch (...) {
    spops_matrix_destroy(c);
    throw;
  }
  spops_matrix_destroy(c);
  const spops_matrix_info_t i = d::info(hh);
  SELL_C_R_Matrix<IndexType, ValueType> s;
  d::set_features<IndexType, ValueType>(s, csr.num_rows, csr.num_cols, csr.num_nnzs);
  s.chunkWidth_C = (IndexType)chunkwidth;
  s.validchunkNum = (IndexType)i.extra[0];
  s.alignment = alignment;
  s.reorder = d::fetch<IndexType>(hh, SPOPS_ARR_REORDER, nullptr);
  s.chunk_len = d::fetch<IndexType>(hh, SPOPS_ARR_CHUNK_LEN, nullptr);
  int64_t ncol = 0, nval = 0;
  IndexType* col = d::fetch<IndexType>(hh, SPOPS_ARR_COL, &ncol);
  ValueType* val = d::fetch<ValueType>(hh, SPOPS_ARR_VAL, &nval);
  s.col_index = d::split_chunks(col, ncol, s.chunk_len, s.validchunkNum, chunkwidth);
  s.values = d::split_chunks(val, nval, s.chunk_len, s.validchunkNum, chunkwidth);
  std::free(col);
  std::free(val);
  spops_matrix_destroy(hh);
  if (d::caching()) d::put(s.reorder, hd, csr.num_rows, csr.num_cols, csr.num_nnzs); else spops_matrix_destroy(hd);
  return s;
}

template <class IndexType, class ValueType>
DIA_Matrix<IndexType, ValueType> csr_to_dia(const CSR_Matrix<IndexType, ValueType>& csr,
                                            const spops_b200::detail::same_t<IndexType> max_diags, FILE* fp_feature,
                                            const spops_b200::detail::same_t<IndexType> alignment =
                                                (SIMD_WIDTH / 8 / sizeof(ValueType))) {
  namespace d = spops_b200::detail;
  (void)fp_feature;
  spops_matrix_t c = d::upload_csr(csr), h = nullptr;
  spops_format_params_t p;
  std::memset(&p, 0, sizeof(p));
  p.max_diags = max_diags;
  p.alignment = alignment;
  spops_status_t s = spops_convert(d::ctx(), c, SPOPS_FMT_DIA, &p, &h);
  spops_matrix_destroy(c);
  d::check(s, "spops_convert");
  const spops_matrix_info_t i = d::info(h);
  DIA_Matrix<IndexType, ValueType> dia;
  d::set_features<IndexType, ValueType>(dia, csr.num_rows, csr.num_cols, csr.num_nnzs);
  dia.complete_ndiags = (IndexType)i.extra[0];
  dia.stride = (IndexType)i.extra[1];
  dia.diag_offsets = reinterpret_cast<long int*>(d::fetch<int64_t>(h, SPOPS_ARR_DIAG_OFFSETS, nullptr));
  dia.diag_data = d::fetch<ValueType>(h, SPOPS_ARR_VAL, nullptr);
  if (d::caching()) d::put(dia.diag_offsets, h, csr.num_rows, csr.num_cols, csr.num_nnzs); else spops_matrix_destroy(h);
  return dia;
}

template <class IndexType, class ValueType>
BSR_Matrix<IndexType, ValueType> csr_to_bsr(const CSR_Matrix<IndexType, ValueType>& csr,
                                            const spops_b200::detail::same_t<IndexType> blockDimRow = BSR_BlockDimRow,
                                            spops_b200::detail::same_t<IndexType> blockDimCol =
                                                (SIMD_WIDTH / 8 / sizeof(ValueType))) {
  namespace d = spops_b200::detail;
  spops_matrix_t c = d::upload_csr(csr), h = nullptr;
  spops_format_params_t p;
  std::memset(&p, 0, sizeof(p));
  p.block_rows = blockDimRow;
  p.block_cols = blockDimCol;
  spops_status_t s = spops_convert(d::ctx(), c, SPOPS_FMT_BSR, &p, &h);
  spops_matrix_destroy(c);
  d::check(s, "spops_convert");
  const spops_matrix_info_t i = d::info(h);
  BSR_Matrix<IndexType, ValueType> bsr;
  d::set_features<IndexType, ValueType>(bsr, csr.num_rows, csr.num_cols, csr.num_nnzs);
  bsr.mb = (IndexType)i.extra[0];
  bsr.nb = (IndexType)i.extra[1];
  bsr.nnzb = (IndexType)i.extra[2];
  bsr.blockDim_r = (IndexType)i.extra[3];
  bsr.blockDim_c = (IndexType)i.extra[4];
  bsr.blockNNZ = bsr.blockDim_r * bsr.blockDim_c;
  bsr.row_ptr = d::fetch<IndexType>(h, SPOPS_ARR_BLOCK_ROW_PTR, nullptr);
  bsr.block_colindex = d::fetch<IndexType>(h, SPOPS_ARR_BLOCK_COL, nullptr);
  bsr.block_data = d::fetch<ValueType>(h, SPOPS_ARR_VAL, nullptr);
  if (d::caching()) d::put(bsr.row_ptr, h, csr.num_rows, csr.num_cols, csr.num_nnzs); else spops_matrix_destroy(h);
  return bsr;
}

template <class IndexType, class UIndexType, class ValueType>
CSR5_Matrix<IndexType, UIndexType, ValueType> csr_to_csr5(const CSR_Matrix<IndexType, ValueType>& csr,
                                                          FILE* fp_feature) {
  namespace d = spops_b200::detail;
  static_assert(sizeof(UIndexType) == 4, "CSR5 tile words are 32-bit");
  (void)fp_feature;
  spops_matrix_t c = d::upload_csr(csr), h = nullptr;
  spops_format_params_t p;
  std::memset(&p, 0, sizeof(p));
  spops_status_t s = spops_convert(d::ctx(), c, SPOPS_FMT_CSR5, &p, &h);
  spops_matrix_destroy(c);
  d::check(s, "spops_convert");
  const spops_matrix_info_t i = d::info(h);
  CSR5_Matrix<IndexType, UIndexType, ValueType> m;
  std::memset(static_cast<void*>(&m), 0, sizeof(m));
  m.num_rows = csr.num_rows;
  m.num_cols = csr.num_cols;
  m.num_nnzs = csr.num_nnzs;
  m.sparsity = (csr.num_rows > 0 && csr.num_cols > 0)
                   ? (double)csr.num_nnzs / ((double)csr.num_rows * (double)csr.num_cols)
                   : 0.0;
  m.row_offset = d::host_alloc<IndexType>((int64_t)csr.num_rows + 1);
  m.col_index = d::host_alloc<IndexType>(csr.num_nnzs);
  m.values = d::host_alloc<ValueType>(csr.num_nnzs);
  std::memcpy(m.row_offset, csr.row_offset, ((size_t)csr.num_rows + 1) * sizeof(IndexType));
  std::memcpy(m.col_index, csr.col_index, (size_t)csr.num_nnzs * sizeof(IndexType));
  std::memcpy(m.values, csr.values, (size_t)csr.num_nnzs * sizeof(ValueType));
  m._p = (IndexType)i.extra[0];
  m.omega = (IndexType)i.extra[1];
  m.sigma = (IndexType)i.extra[2];
  m.tile_ptr = d::fetch<UIndexType>(h, SPOPS_ARR_TILE_PTR, nullptr);
  m.tile_desc = d::fetch<UIndexType>(h, SPOPS_ARR_TILE_DESC, nullptr);
  if (d::caching()) d::put(m.tile_ptr, h, csr.num_rows, csr.num_cols, csr.num_nnzs); else spops_matrix_destroy(h);
  return m;
}

/* ------------------------------------------------------------- delete */
namespace spops_b200 {
namespace detail {
template <typename T>
inline void free_array(T*& p) {
  std::free(p);
  p = nullptr;
}
template <typename T, typename I>
inline void free_chunks(T**& parts, I n) {
  if (parts) {
    for (I c = 0; c < n; ++c) std::free(parts[c]);
    delete[] parts;
  }
  parts = nullptr;
}
}  // namespace detail
}  // namespace spops_b200

template <typename I, typename V>
void delete_host_matrix(COO_Matrix<I, V>& m) {
  spops_b200::invalidate(m.row_index);
  spops_b200::detail::free_array(m.row_index);
  spops_b200::detail::free_array(m.col_index);
  spops_b200::detail::free_array(m.values);
}
template <typename I, typename V>
void delete_host_matrix(CSR_Matrix<I, V>& m) {
  spops_b200::invalidate(m.row_offset);
  spops_b200::detail::free_array(m.row_offset);
  spops_b200::detail::free_array(m.col_index);
  spops_b200::detail::free_array(m.values);
}
template <typename I, typename V>
void delete_host_matrix(ELL_Matrix<I, V>& m) {
  spops_b200::invalidate(m.col_index);
  spops_b200::detail::free_array(m.col_index);
  spops_b200::detail::free_array(m.values);
  m.max_row_width = m.min_row_width = 0;
}
template <typename I, typename V>
void delete_host_matrix(S_ELL_Matrix<I, V>& m) {
  spops_b200::invalidate(m.row_width);
  spops_b200::detail::free_chunks(m.col_index, m.chunk_num);
  spops_b200::detail::free_chunks(m.values, m.chunk_num);
  spops_b200::detail::free_array(m.row_width);
  m.chunk_num = 0;
}
template <typename I, typename V>
void delete_host_matrix(SELL_C_Sigma_Matrix<I, V>& m) {
  spops_b200::invalidate(m.reorder);
  spops_b200::detail::free_chunks(m.col_index, m.validchunkNum);
  spops_b200::detail::free_chunks(m.values, m.validchunkNum);
  spops_b200::detail::free_array(m.reorder);
  spops_b200::detail::free_array(m.chunk_len);
  m.validchunkNum = m.chunkNum = m.sliceNum = 0;
}
template <typename I, typename V>
void delete_host_matrix(SELL_C_R_Matrix<I, V>& m) {
  spops_b200::invalidate(m.reorder);
  spops_b200::detail::free_chunks(m.col_index, m.validchunkNum);
  spops_b200::detail::free_chunks(m.values, m.validchunkNum);
  spops_b200::detail::free_array(m.reorder);
  spops_b200::detail::free_array(m.chunk_len);
  m.validchunkNum = 0;
}
template <typename I, typename V>
void delete_host_matrix(DIA_Matrix<I, V>& m) {
  spops_b200::invalidate(m.diag_offsets);
  spops_b200::detail::free_array(m.diag_offsets);
  spops_b200::detail::free_array(m.diag_data);
}
template <typename I, typename V>
void delete_host_matrix(BSR_Matrix<I, V>& m) {
  spops_b200::invalidate(m.row_ptr);
  spops_b200::detail::free_array(m.row_ptr);
  spops_b200::detail::free_array(m.block_colindex);
  spops_b200::detail::free_array(m.block_data);
}
template <typename I, typename U, typename V>
void delete_host_matrix(CSR5_Matrix<I, U, V>& m) {
  spops_b200::invalidate(m.tile_ptr);
  spops_b200::detail::free_array(m.row_offset);
  spops_b200::detail::free_array(m.col_index);
  spops_b200::detail::free_array(m.values);
  spops_b200::detail::free_array(m.tile_ptr);
  spops_b200::detail::free_array(m.tile_desc);
  spops_b200::detail::free_array(m.tile_desc_offset_ptr);
  spops_b200::detail::free_array(m.tile_desc_offset);
  spops_b200::detail::free_array(m.calibrator);
}

/* ------------------------------------------------- LeSpGEMM preprocessing */
template <typename IndexType>
std::vector<uint64_t> minhash_signatures_flat(const IndexType* rowptr, const IndexType* col_index, IndexType num_rows,
                                              int k, uint64_t seed = 12345) {
  namespace d = spops_b200::detail;
  std::vector<uint64_t> sig((size_t)(num_rows > 0 ? num_rows : 0) * (size_t)(k > 0 ? k : 0));
  if (num_rows <= 0 || k <= 0) return sig;
  spops_matrix_t h = d::upload_pattern(rowptr, col_index, num_rows);
  spops_status_t s = spops_minhash_host(d::ctx(), h, k, seed, sig.data());
  spops_matrix_destroy(h);
  d::check(s, "spops_minhash_host");
  return sig;
}

template <typename IndexType, typename ValueType>
std::vector<CandidatePair<IndexType, ValueType>> lsh_candidate_pairs_vector(const IndexType* rowptr,
                                                                            const IndexType* col_index,
                                                                            IndexType num_rows, int k, int num_bands,
                                                                            uint64_t seed = 12345,
                                                                            bool constrain_large_buckets = true) {
  namespace d = spops_b200::detail;
  std::vector<CandidatePair<IndexType, ValueType>> out;
  if (num_rows <= 0) return out;
  spops_matrix_t h = d::upload_pattern(rowptr, col_index, num_rows);
  spops_pairs_t P = nullptr;
  spops_status_t s = spops_lsh_pairs(d::ctx(), h, k, num_bands, seed, constrain_large_buckets ? 1 : 0, &P);
  spops_matrix_destroy(h);
  d::check(s, "spops_lsh_pairs");
  int64_t n = 0;
  spops_pairs_count(P, &n);
  std::vector<int64_t> pi((size_t)n), pj((size_t)n);
  std::vector<double> ps((size_t)n);
  s = n ? spops_pairs_download(P, pi.data(), pj.data(), ps.data()) : SPOPS_OK;
  spops_pairs_destroy(P);
  d::check(s, "spops_pairs_download");
  out.resize((size_t)n);
  for (int64_t t = 0; t < n; ++t)
    out[(size_t)t] = CandidatePair<IndexType, ValueType>{(IndexType)pi[(size_t)t], (IndexType)pj[(size_t)t],
                                                         (ValueType)ps[(size_t)t]};
  return out;
}

template <typename IndexType, typename ValueType, typename PairLike>
inline void hierarchical_clustering_v0_fast(const IndexType* rowptr, const IndexType* colids, IndexType num_rows,
                                            const std::vector<PairLike>& pairs, IndexType cluster_size,
                                            std::vector<IndexType>& permutation_out,
                                            std::vector<IndexType>& offsets_out) {
  namespace d = spops_b200::detail;
  const int64_t n = num_rows > 0 ? num_rows : 0, nnz = n ? (int64_t)rowptr[n] : 0;
  std::vector<int64_t> rp((size_t)n + 1), ci((size_t)nnz), pi(pairs.size()), pj(pairs.size());
  std::vector<double> ps(pairs.size());
  for (int64_t r = 0; r <= n && n; ++r) rp[(size_t)r] = (int64_t)rowptr[r];
  for (int64_t e = 0; e < nnz; ++e) ci[(size_t)e] = (int64_t)colids[e];
  for (size_t t = 0; t < pairs.size(); ++t) {
    pi[t] = (int64_t)pairs[t].i;
    pj[t] = (int64_t)pairs[t].j;
    ps[t] = (double)pairs[t].score;
  }
  std::vector<int64_t> perm((size_t)n), offs((size_t)n + 1);
  int64_t ncl = 0;
  d::check(spops_hierarchical_clustering(rp.data(), ci.data(), n, pi.data(), pj.data(), ps.data(),
                                         (int64_t)pairs.size(), cluster_size, perm.data(), offs.data(), &ncl),
           "spops_hierarchical_clustering");
  permutation_out.assign(perm.begin(), perm.end());
  offsets_out.assign(offs.begin(), offs.begin() + ncl + 1);
}

/* ------------------------------------------------- Matrix Market files */
/* include/sparse_io.h:40 / :52: the file is read on the host and parsed on
 * the device (values as scanf("%lf") converts them); host structs out.  A
 * malformed file throws where the reference asserts or exits. */
template <class IndexType, class ValueType>
COO_Matrix<IndexType, ValueType> read_coo_matrix(const char* mm_filename) {
  namespace d = spops_b200::detail;
  spops_matrix_t h = nullptr;
  d::check(spops_mtx_read_coo(d::ctx(), mm_filename, d::itype<IndexType>(), d::vtype<ValueType>(), &h),
           "spops_mtx_read_coo");
  const spops_matrix_info_t i = d::info(h);
  COO_Matrix<IndexType, ValueType> coo;
  d::set_features<IndexType, ValueType>(coo, i.rows, i.cols, i.nnz);
  coo.row_index = d::fetch<IndexType>(h, SPOPS_ARR_ROW, nullptr);
  coo.col_index = d::fetch<IndexType>(h, SPOPS_ARR_COL, nullptr);
  coo.values = d::fetch<ValueType>(h, SPOPS_ARR_VAL, nullptr);
  spops_matrix_destroy(h);
  return coo;
}

template <class IndexType, class ValueType>
CSR_Matrix<IndexType, ValueType> read_csr_matrix(const char* mm_filename, bool compact = false) {
  namespace d = spops_b200::detail;
  spops_matrix_t h = nullptr;
  d::check(spops_mtx_read_csr(d::ctx(), mm_filename, d::itype<IndexType>(), d::vtype<ValueType>(), compact ? 1 : 0,
                              &h),
           "spops_mtx_read_csr");
  const spops_matrix_info_t i = d::info(h);
  CSR_Matrix<IndexType, ValueType> csr;
  d::set_features<IndexType, ValueType>(csr, i.rows, i.cols, i.nnz);
  csr.row_offset = d::fetch<IndexType>(h, SPOPS_ARR_ROW, nullptr);
  csr.col_index = d::fetch<IndexType>(h, SPOPS_ARR_COL, nullptr);
  csr.values = d::fetch<ValueType>(h, SPOPS_ARR_VAL, nullptr);
  if (d::caching_csr()) d::put(csr.row_offset, h, i.rows, i.cols, i.nnz); else spops_matrix_destroy(h);
  return csr;
}

/* ---------------------------------------------------- row-wise SpGEMM */
namespace spops_b200 {
namespace detail {
// a device result handle into a host CSR struct (arrays from posix_memalign)
template <typename I, typename V>
inline void take_csr(spops_matrix_t h, CSR_Matrix<I, V>& C) {
  const spops_matrix_info_t i = info(h);
  set_features<I, V>(C, i.rows, i.cols, i.nnz);
  C.row_offset = fetch<I>(h, SPOPS_ARR_ROW, nullptr);
  C.col_index = fetch<I>(h, SPOPS_ARR_COL, nullptr);
  C.values = fetch<V>(h, SPOPS_ARR_VAL, nullptr);
  spops_matrix_destroy(h);
}
}  // namespace detail
}  // namespace spops_b200

/* C = A * B row by row (include/spgemm.h:29, src/spgemm.cpp:683): every
 * structural entry kept, columns ascending; kernel_flag is recorded in C. */
template <bool sortOutput, typename IndexType, typename ValueType>
void LeSpGEMM(const CSR_Matrix<IndexType, ValueType>& A, const CSR_Matrix<IndexType, ValueType>& B,
              CSR_Matrix<IndexType, ValueType>& C, int kernel_flag) {
  namespace d = spops_b200::detail;
  spops_matrix_t a = d::upload_csr(A), b = d::upload_csr(B), c = nullptr;
  spops_status_t s = spops_spgemm_rowwise(d::ctx(), a, b, kernel_flag, sortOutput ? 1 : 0, &c, nullptr);
  spops_matrix_destroy(a);
  spops_matrix_destroy(b);
  d::check(s, "spops_spgemm_rowwise");
  d::take_csr<IndexType, ValueType>(c, C);
  C.kernel_flag = kernel_flag;
}

/* Top-k Jaccard similarities of A's rows (src/spgemm.cpp:708): per row, the
 * top_k other rows by similarity descending, then column ascending. */
template <typename IndexType, typename ValueType>
void HashSpGEMMTopK(const CSR_Matrix<IndexType, ValueType>& A, CSR_Matrix<IndexType, ValueType>& C,
                    IndexType top_k) {
  namespace d = spops_b200::detail;
  spops_matrix_t a = d::upload_csr(A), c = nullptr;
  spops_status_t s = spops_spgemm_topk(d::ctx(), a, (int64_t)top_k, &c);
  spops_matrix_destroy(a);
  d::check(s, "spops_spgemm_topk");
  d::take_csr<IndexType, ValueType>(c, C);
  C.kernel_flag = 0;
}

/* ----------------------------------------- more of the reference's API */
/* Per-format deletes (include/sparse_format.h:300-420): delete_host_matrix. */
template <class I, class V> void delete_coo_matrix(COO_Matrix<I, V>& m) { delete_host_matrix(m); }
template <class I, class V> void delete_csr_matrix(CSR_Matrix<I, V>& m) { delete_host_matrix(m); }
template <class I, class V> void delete_bsr_matrix(BSR_Matrix<I, V>& m) { delete_host_matrix(m); }
template <class I, class V> void delete_dia_matrix(DIA_Matrix<I, V>& m) { delete_host_matrix(m); }
template <class I, class V> void delete_ell_matrix(ELL_Matrix<I, V>& m) { delete_host_matrix(m); }
template <class I, class V> void delete_s_ell_matrix(S_ELL_Matrix<I, V>& m) { delete_host_matrix(m); }
template <class I, class V> void delete_s_ell_c_sigma_matrix(SELL_C_Sigma_Matrix<I, V>& m) { delete_host_matrix(m); }
template <class I, class V> void delete_s_ell_c_R_matrix(SELL_C_R_Matrix<I, V>& m) { delete_host_matrix(m); }
template <class I, class U, class V> void delete_csr5_matrix(CSR5_Matrix<I, U, V>& m) { delete_host_matrix(m); }

/* The reference's OpenMP thread controls (include/thread.h).  The work runs on
 * the GPU, so they only keep the caller's setting for its own queries. */
namespace spops_b200 {
namespace detail {
inline int& thread_setting() {
  static int n = 0;
  return n;
}
}  // namespace detail
}  // namespace spops_b200
inline int Le_get_core_num() {
  const unsigned c = std::thread::hardware_concurrency();
  return c ? (int)c : 1;
}
inline void Le_set_thread_num(const int thread_num) { spops_b200::detail::thread_setting() = thread_num; }
inline int Le_get_thread_num() {
  const int n = spops_b200::detail::thread_setting();
  return n > 0 ? n : Le_get_core_num();
}
inline int Le_get_thread_id() { return 0; }
inline void set_omp_schedule(int, int) {}

/* coo_to_ell (include/sparse_conversion.h:102): the rows keep the COO's
 * entry order, as through coo_to_csr. */
template <class IndexType, class ValueType>
ELL_Matrix<IndexType, ValueType> coo_to_ell(const COO_Matrix<IndexType, ValueType>& coo,
                                            const LeadingDimension ld = RowMajor) {
  CSR_Matrix<IndexType, ValueType> csr = coo_to_csr(coo, false);
  ELL_Matrix<IndexType, ValueType> ell = csr_to_ell(csr, ld);
  delete_host_matrix(csr);
  return ell;
}

/* Matrix Market files straight into a format (utils/sparse_io.cpp:225-390):
 * read_csr_matrix (or read_coo_matrix for ELL) and the conversion, on the
 * device; the reference's feature file argument is not written. */
template <class IndexType, class ValueType>
ELL_Matrix<IndexType, ValueType> read_ell_matrix(const char* mm_filename, LeadingDimension ld = RowMajor) {
  COO_Matrix<IndexType, ValueType> coo = read_coo_matrix<IndexType, ValueType>(mm_filename);
  ELL_Matrix<IndexType, ValueType> ell;
  if (coo.num_rows == 0) {
    std::memset(static_cast<void*>(&ell), 0, sizeof(ell));
    delete_host_matrix(coo);
    return ell;
  }
  ell = coo_to_ell(coo, ld);
  delete_host_matrix(coo);
  ell.kernel_flag = KERNEL_FLAG;
  return ell;
}
template <class IndexType, class ValueType>
DIA_Matrix<IndexType, ValueType> read_dia_matrix(const char* mm_filename,
                                                 const spops_b200::detail::same_t<IndexType> max_diags,
                                                 const spops_b200::detail::same_t<IndexType> alignment =
                                                     (SIMD_WIDTH / 8 / sizeof(ValueType))) {
  CSR_Matrix<IndexType, ValueType> csr = read_csr_matrix<IndexType, ValueType>(mm_filename);
  DIA_Matrix<IndexType, ValueType> m = csr_to_dia(csr, max_diags, nullptr, alignment);
  delete_host_matrix(csr);
  return m;
}
template <class IndexType, class ValueType>
S_ELL_Matrix<IndexType, ValueType> read_sell_matrix(const char* mm_filename, const int chunkwidth,
                                                    const spops_b200::detail::same_t<IndexType> alignment) {
  CSR_Matrix<IndexType, ValueType> csr = read_csr_matrix<IndexType, ValueType>(mm_filename);
  S_ELL_Matrix<IndexType, ValueType> m = csr_to_sell(csr, nullptr, chunkwidth, alignment);
  delete_host_matrix(csr);
  return m;
}
template <class IndexType, class ValueType>
SELL_C_Sigma_Matrix<IndexType, ValueType> read_sell_c_sigma_matrix(
    const char* mm_filename, const int slicewidth, const int chunkwidth,
    const spops_b200::detail::same_t<IndexType> alignment) {
  CSR_Matrix<IndexType, ValueType> csr = read_csr_matrix<IndexType, ValueType>(mm_filename);
  SELL_C_Sigma_Matrix<IndexType, ValueType> m = csr_to_sell_c_sigma(csr, nullptr, slicewidth, chunkwidth, alignment);
  delete_host_matrix(csr);
  return m;
}
template <class IndexType, class ValueType>
SELL_C_R_Matrix<IndexType, ValueType> read_sell_c_R_matrix(const char* mm_filename, const int chunkwidth,
                                                           const spops_b200::detail::same_t<IndexType> alignment) {
  CSR_Matrix<IndexType, ValueType> csr = read_csr_matrix<IndexType, ValueType>(mm_filename);
  SELL_C_R_Matrix<IndexType, ValueType> m = csr_to_sell_c_R(csr, nullptr, chunkwidth, alignment);
  delete_host_matrix(csr);
  return m;
}
template <class IndexType, class ValueType>
BSR_Matrix<IndexType, ValueType> read_bsr_matrix(const char* mm_filename,
                                                 const spops_b200::detail::same_t<IndexType> blockDimRow =
                                                     BSR_BlockDimRow,
                                                 const spops_b200::detail::same_t<IndexType> blockDimCol =
                                                     (SIMD_WIDTH / 8 / sizeof(ValueType))) {
  CSR_Matrix<IndexType, ValueType> csr = read_csr_matrix<IndexType, ValueType>(mm_filename);
  BSR_Matrix<IndexType, ValueType> m = csr_to_bsr(csr, blockDimRow, blockDimCol);
  delete_host_matrix(csr);
  return m;
}
template <class IndexType, class UIndexType, class ValueType>
CSR5_Matrix<IndexType, UIndexType, ValueType> read_csr5_matrix(const char* mm_filename) {
  CSR_Matrix<IndexType, ValueType> csr = read_csr_matrix<IndexType, ValueType>(mm_filename);
  CSR5_Matrix<IndexType, UIndexType, ValueType> m = csr_to_csr5<IndexType, UIndexType, ValueType>(csr, nullptr);
  delete_host_matrix(csr);
  return m;
}

/* sum_csr_duplicates (include/sparse_operation.h:21): duplicates of a row
 * summed, the row's columns in reverse order of first appearance, exact
 * zeros dropped, in place (row_ptr[num_rows] becomes the new count) -- the
 * device coo_to_csr's compact mode. */
template <class IndexType, class ValueType>
void sum_csr_duplicates(const IndexType num_rows, const IndexType num_cols, IndexType* row_ptr, IndexType* col_index,
                        ValueType* values) {
  const IndexType nnz = num_rows > 0 ? row_ptr[num_rows] : 0;
  COO_Matrix<IndexType, ValueType> coo;
  std::memset(static_cast<void*>(&coo), 0, sizeof(coo));
  coo.num_rows = num_rows;
  coo.num_cols = num_cols;
  coo.num_nnzs = nnz;
  std::vector<IndexType> rows((size_t)nnz);
  for (IndexType r = 0; r < num_rows; ++r)
    for (IndexType k = row_ptr[r]; k < row_ptr[r + 1]; ++k) rows[(size_t)k] = r;
  coo.row_index = rows.data();
  coo.col_index = col_index;
  coo.values = values;
  const spops_b200::CacheMode was = spops_b200::cache_mode();
  spops_b200::set_cache_mode(spops_b200::CacheMode::Off);  // the result is copied out, nothing to keep
  CSR_Matrix<IndexType, ValueType> c = coo_to_csr(coo, true);
  spops_b200::set_cache_mode(was);
  std::memcpy(row_ptr, c.row_offset, sizeof(IndexType) * ((size_t)num_rows + 1));
  std::memcpy(col_index, c.col_index, sizeof(IndexType) * (size_t)c.num_nnzs);
  std::memcpy(values, c.values, sizeof(ValueType) * (size_t)c.num_nnzs);
  delete_host_matrix(c);
}

/* csr_transpose (include/sparse_conversion.h:2067): the transpose with
 * duplicates summed and exact zeros dropped (csr_to_coo, index swap,
 * coo_to_csr compact), on the device. */
template <class IndexType, class ValueType>
CSR_Matrix<IndexType, ValueType> csr_transpose(const CSR_Matrix<IndexType, ValueType>& csr) {
  if (csr.num_nnzs == 0) {
    CSR_Matrix<IndexType, ValueType> t;
    std::memset(static_cast<void*>(&t), 0, sizeof(t));
    t.num_rows = csr.num_cols;
    t.num_cols = csr.num_rows;
    t.row_offset = spops_b200::detail::host_alloc<IndexType>((int64_t)csr.num_cols + 1);
    std::fill_n(t.row_offset, (size_t)csr.num_cols + 1, (IndexType)0);
    return t;
  }
  COO_Matrix<IndexType, ValueType> coo = csr_to_coo(csr);
  std::swap(coo.row_index, coo.col_index);
  std::swap(coo.num_rows, coo.num_cols);
  spops_b200::invalidate(coo.col_index);  // the cached COO handle no longer matches the struct
  spops_b200::invalidate(coo.row_index);
  CSR_Matrix<IndexType, ValueType> t = coo_to_csr(coo, true);
  delete_host_matrix(coo);
  return t;
}

/* csr_reorder_rows (include/sparse_conversion.h:1879-1998): row i of the
 * result is row row_permutation[i] of csr, gathered on the device. */
template <class IndexType, class ValueType>
CSR_Matrix<IndexType, ValueType> csr_reorder_rows(const CSR_Matrix<IndexType, ValueType>& csr,
                                                  const IndexType* row_permutation) {
  namespace d = spops_b200::detail;
  if (csr.num_nnzs == 0) {
    CSR_Matrix<IndexType, ValueType> r;
    std::memset(static_cast<void*>(&r), 0, sizeof(r));
    r.num_rows = csr.num_rows;
    r.num_cols = csr.num_cols;
    r.row_offset = d::host_alloc<IndexType>((int64_t)csr.num_rows + 1);
    std::fill_n(r.row_offset, (size_t)csr.num_rows + 1, (IndexType)0);
    return r;
  }
  spops_matrix_t a = d::upload_csr(csr), c = nullptr;
  spops_status_t s = spops_csr_reorder_rows(d::ctx(), a, row_permutation, &c);
  spops_matrix_destroy(a);
  d::check(s, "spops_csr_reorder_rows");
  CSR_Matrix<IndexType, ValueType> r;
  d::take_csr<IndexType, ValueType>(c, r);
  r.kernel_flag = 0;
  return r;
}
template <class IndexType, class ValueType>
CSR_Matrix<IndexType, ValueType> csr_reorder_rows(const CSR_Matrix<IndexType, ValueType>& csr,
                                                  const std::vector<IndexType>& row_permutation) {
  if (row_permutation.size() < (size_t)csr.num_rows)
    throw std::invalid_argument("row_permutation size must be >= matrix rows");
  return csr_reorder_rows(csr, row_permutation.data());
}

/* csr_to_binary_pattern (include/sparse_conversion.h:2121): the pattern with
 * every value 1. */
template <class IndexType, class ValueType>
CSR_Matrix<IndexType, ValueType> csr_to_binary_pattern(const CSR_Matrix<IndexType, ValueType>& csr) {
  namespace d = spops_b200::detail;
  CSR_Matrix<IndexType, ValueType> b;
  d::set_features<IndexType, ValueType>(b, csr.num_rows, csr.num_cols, csr.num_nnzs);
  b.kernel_flag = csr.kernel_flag;
  b.row_offset = d::host_alloc<IndexType>((int64_t)csr.num_rows + 1);
  std::memcpy(b.row_offset, csr.row_offset, sizeof(IndexType) * ((size_t)csr.num_rows + 1));
  b.col_index = d::host_alloc<IndexType>(csr.num_nnzs);
  b.values = d::host_alloc<ValueType>(csr.num_nnzs);
  if (csr.num_nnzs > 0) std::memcpy(b.col_index, csr.col_index, sizeof(IndexType) * (size_t)csr.num_nnzs);
  std::fill_n(b.values, (size_t)csr.num_nnzs, (ValueType)1);
  return b;
}

/* minhash_estimated_jaccard (include/spgemm_MinHashLSH.h:183-224): the share
 * of equal signature entries. */
inline double minhash_estimated_jaccard(const uint64_t* sig_a, const uint64_t* sig_b, int k) {
  if (k <= 0) return 0.0;
  int match = 0;
  for (int d = 0; d < k; ++d) match += sig_a[d] == sig_b[d];
  return (double)match / (double)k;
}
inline double minhash_estimated_jaccard(const std::vector<uint64_t>& sig_a, const std::vector<uint64_t>& sig_b) {
  if (sig_a.size() != sig_b.size() || sig_a.empty()) return 0.0;
  return minhash_estimated_jaccard(sig_a.data(), sig_b.data(), (int)sig_a.size());
}

/* ----------------------------------------------- clustered (VLength) form */
#ifndef CPU_L2CACHE_SIZE
#define CPU_L2CACHE_SIZE 67108864
#endif
#ifndef MIXED_L2_FRACTION
#define MIXED_L2_FRACTION 0.75
#endif

/* The reference's cluster struct (spgemm_cluster.h:108-143), same fields. */
template <typename IndexType, typename ValueType>
struct CSR_VlengthCluster : public Matrix_Features<IndexType> {
  typedef IndexType index_type;
  typedef ValueType value_type;
  IndexType csr_rows;
  IndexType rows;
  IndexType cols;
  IndexType nnzc;
  IndexType nnzv;
  IndexType max_cluster_sz;
  IndexType* cluster_sz;
  IndexType* rowptr;
  IndexType* colids;
  IndexType* rowptr_val;
  ValueType* values;
  int dense_cluster_count;
  char* acc_flag = NULL;
  IndexType* min_ccol = NULL;
  IndexType* max_ccol = NULL;
  double mixed_acc_setup_ms = 0.0;
  double mixed_acc_malloc_ms = 0.0;
  double mixed_acc_symbolic_ms = 0.0;
  double mixed_acc_dispatcher_ms = 0.0;
  double mixed_acc_numeric_ms = 0.0;
};

template <typename IndexType, typename ValueType>
void delete_vlength_cluster_matrix(CSR_VlengthCluster<IndexType, ValueType>& c) {
  std::free(c.cluster_sz);
  std::free(c.rowptr);
  std::free(c.colids);
  std::free(c.rowptr_val);
  std::free(c.values);
  c.cluster_sz = c.rowptr = c.colids = c.rowptr_val = nullptr;
  c.values = nullptr;
  c.csr_rows = c.rows = c.cols = c.nnzc = c.nnzv = 0;
}
template <typename IndexType, typename ValueType>
void delete_host_matrix(CSR_VlengthCluster<IndexType, ValueType>& c) { delete_vlength_cluster_matrix(c); }

namespace spops_b200 {
namespace detail {
// a clustered-form device handle into the caller's struct (arrays from
// posix_memalign, freed by delete_vlength_cluster_matrix)
template <typename I, typename V>
inline void take_vlcluster(spops_matrix_t h, CSR_VlengthCluster<I, V>& c) {
  const spops_matrix_info_t i = info(h);
  c.csr_rows = (I)i.rows;
  c.cols = (I)i.cols;
  c.nnzc = (I)i.nnz;
  c.rows = (I)i.extra[0];
  c.nnzv = (I)i.extra[1];
  c.max_cluster_sz = (I)i.extra[2];
  c.cluster_sz = fetch<I>(h, SPOPS_ARR_CLUSTER_SZ, nullptr);
  c.rowptr = fetch<I>(h, SPOPS_ARR_ROW, nullptr);
  c.colids = fetch<I>(h, SPOPS_ARR_COL, nullptr);
  c.rowptr_val = fetch<I>(h, SPOPS_ARR_ROWPTR_VAL, nullptr);
  c.values = fetch<V>(h, SPOPS_ARR_VAL, nullptr);
  c.dense_cluster_count = 0;
  c.num_rows = c.csr_rows;
  c.num_cols = c.cols;
  c.num_nnzs = c.nnzv;
  spops_matrix_destroy(h);
}
template <typename I, typename V>
inline spops_matrix_t upload_vlcluster(const CSR_VlengthCluster<I, V>& c) {
  spops_matrix_t h = nullptr;
  check(spops_vlcluster_create(ctx(), &h, c.csr_rows, c.rows, c.cols, c.nnzc, c.nnzv, c.cluster_sz, c.rowptr,
                               c.colids, c.rowptr_val, c.values, itype<I>(), vtype<V>(), SPOPS_MEM_HOST),
        "spops_vlcluster_create");
  return h;
}
}  // namespace detail
}  // namespace spops_b200

/* csr_to_vlength_cluster (sparse_conversion.h:1640-1765): cluster i is rows
 * offsets[i] .. offsets[i+1]; its columns ascending (the reference: hash-map
 * order). */
template <class IndexType, class ValueType>
CSR_VlengthCluster<IndexType, ValueType> csr_to_vlength_cluster(const CSR_Matrix<IndexType, ValueType>& csr,
                                                                const std::vector<IndexType>& offsets) {
  namespace d = spops_b200::detail;
  if (offsets.size() < 2) throw std::invalid_argument("offsets size must be >= 2");
  std::vector<int64_t> off(offsets.begin(), offsets.end());
  spops_matrix_t a = d::upload_csr(csr), h = nullptr;
  spops_status_t s = spops_csr_to_vlength_cluster(d::ctx(), a, off.data(), (int64_t)off.size() - 1, &h);
  spops_matrix_destroy(a);
  d::check(s, "spops_csr_to_vlength_cluster");
  CSR_VlengthCluster<IndexType, ValueType> c;
  std::memset(static_cast<void*>(&c), 0, sizeof(c));
  d::take_vlcluster<IndexType, ValueType>(h, c);
  return c;
}

/* vlength_cluster2csr (sparse_conversion.h:1777-1862): rows in cluster order,
 * exact zeros dropped. */
template <class IndexType, class ValueType>
CSR_Matrix<IndexType, ValueType> vlength_cluster2csr(const CSR_VlengthCluster<IndexType, ValueType>& cluster) {
  namespace d = spops_b200::detail;
  spops_matrix_t a = d::upload_vlcluster(cluster), h = nullptr;
  spops_status_t s = spops_vlength_cluster_to_csr(d::ctx(), a, &h);
  spops_matrix_destroy(a);
  d::check(s, "spops_vlength_cluster_to_csr");
  CSR_Matrix<IndexType, ValueType> csr;
  d::take_csr<IndexType, ValueType>(h, csr);
  csr.kernel_flag = 0;
  return csr;
}

/* LeSpGEMM_VLength (spgemm.h:175-180; src/spgemm.cpp:661-680): C = A * B
 * with A clustered; C in A's clusters (allocated here, columns ascending).
 * kernel_flag picks the reference kernel whose output rules C follows:
 *   3  mixed accumulator (spgemm_Vlength_mixed.cpp): dense clusters by the
 *      L2 rule; all-below-1e-12 columns dropped on the dense and sorted paths;
 *   2  array accumulator (spgemm_Vlength_array.cpp): every structural column
 *      kept, whatever sortOutput says;
 *   1 and any other value  hash accumulator (spgemm_Vlength_hash.cpp): no
 *      dense clusters; all-below-1e-12 columns dropped when sortOutput.
 * The device computes all three with the same hash/dense kernels; only the
 * dense budget and the drop rule differ.  The caller's acc_flag / min_ccol /
 * max_ccol, if any, are left untouched. */
template <bool sortOutput = true, typename IndexType, typename ValueType>
void LeSpGEMM_VLength(const CSR_VlengthCluster<IndexType, ValueType>& A_cluster,
                      const CSR_Matrix<IndexType, ValueType>& B, CSR_VlengthCluster<IndexType, ValueType>& C_cluster,
                      int kernel_flag = 1, double mixed_l2_fraction = -1.0) {
  namespace d = spops_b200::detail;
  const double frac = mixed_l2_fraction < 0 ? MIXED_L2_FRACTION : mixed_l2_fraction;
  // a negative budget makes no cluster dense (the hash and array kernels)
  const double budget = kernel_flag == 3 ? (double)CPU_L2CACHE_SIZE * frac : -1.0;
  const int32_t drop_sorted = (kernel_flag == 2) ? 0 : (sortOutput ? 1 : 0);
  spops_matrix_t a = d::upload_vlcluster(A_cluster), b = d::upload_csr(B), c = nullptr;
  spops_status_t s = spops_spgemm_vlength(d::ctx(), a, b, drop_sorted, budget, &c, nullptr);
  spops_matrix_destroy(a);
  spops_matrix_destroy(b);
  d::check(s, "spops_spgemm_vlength");
  d::take_vlcluster<IndexType, ValueType>(c, C_cluster);
  C_cluster.max_cluster_sz = A_cluster.max_cluster_sz;
}

/* ------------------------------------------------------------ features */
/* The reference's feature class (include/sparse_features.h:15-328,
 * src/sparse_features.cpp) with its public calls:
 *   MtxLoad(path)                 the Matrix Market file read on the device
 *                                 (read_csr_matrix, symmetric files expanded)
 *   CalculateFeatures()           structure and tile features on the device
 *                                 (spops_matrix_features, spops_matrix_tile_features)
 *   CalculateTilesFeatures(), CalculateTilesExtraFeatures(path)
 *                                 already computed by CalculateFeatures; true
 *   FeaturesPrint(), ExtraFeaturesPrint()   the reference's text
 *   FeaturesWrite(dir)            the .features file and the tile / RB / CB
 *                                 maps under dir/<name>/ (the reference writes
 *                                 under a fixed root); returns what the
 *                                 reference returns: false (EXIT_SUCCESS)
 *                                 when written, true when not
 *   ConvertToCSR(csr), getRowNum(), getColNum(), getTileSize(), getMatName()
 * Differences: a symmetric file's features are those of its expanded
 * matrix (the reference counts each off-diagonal entry twice too, and sets
 * the symmetry ratios to 1, which the expanded matrix gives); the GrX
 * features of CalculateTilesExtraFeatures, compiled out in the reference,
 * are not computed (printed as the reference's initial -1). */
template <typename IndexType, typename ValueType>
class MTX {
 public:
  explicit MTX(IndexType matID = 0) : matrixID_(matID) {
    std::printf("== MTX Features Extraction ==\n\n");
  }
  ~MTX() {
    if (h_) spops_matrix_destroy(h_);
  }
  MTX(const MTX&) = delete;
  MTX& operator=(const MTX&) = delete;
  IndexType getRowNum() { return (IndexType)f_.rows; }
  IndexType getColNum() { return (IndexType)f_.cols; }
  IndexType getTileSize() { return (IndexType)256; }
  std::string getMatName() { return matrixName_; }

  bool MtxLoad(const char* mat_path) {
    namespace d = spops_b200::detail;
    const auto t0 = std::chrono::steady_clock::now();
    if (h_) spops_matrix_destroy(h_);
    h_ = nullptr;
    d::check(spops_mtx_read_csr(d::ctx(), mat_path, d::itype<IndexType>(), d::vtype<ValueType>(), 0, &h_),
             "spops_mtx_read_csr");
    std::string name(mat_path);
    const size_t slash = name.find_last_of('/');
    if (slash != std::string::npos) name = name.substr(slash + 1);
    const size_t dot = name.find_last_of('.');
    matrixName_ = dot == std::string::npos ? name : name.substr(0, dot);
    const spops_matrix_info_t i = d::info(h_);
    f_.rows = i.rows;
    f_.cols = i.cols;
    f_.nnz = i.nnz;
    MtxLoad_time_ = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return true;
  }

  bool CalculateFeatures() {
    namespace d = spops_b200::detail;
    if (!h_) throw std::runtime_error("spops_b200: MTX::CalculateFeatures before MtxLoad");
    const auto t0 = std::chrono::steady_clock::now();
    d::check(spops_matrix_features(d::ctx(), h_, &f_), "spops_matrix_features");
    const size_t B = 256, T = B * B;
    tile_i_.assign(4 * T, 0);
    tile_d_.assign(2 * T, 0.0);
    blk_i_.assign(4 * B, 0);
    blk_d_.assign(4 * B, 0.0);
    spops_tile_maps_t m{};
    m.tile_nnz = tile_i_.data();
    m.tile_rows = tile_i_.data() + T;
    m.tile_cols = tile_i_.data() + 2 * T;
    m.tile_max_row_nnz = tile_i_.data() + 3 * T;
    m.tile_ave_row_nnz = tile_d_.data();
    m.tile_std_row_nnz = tile_d_.data() + T;
    m.rb_nnz = blk_i_.data();
    m.rb_max_row_nnz = blk_i_.data() + B;
    m.cb_nnz = blk_i_.data() + 2 * B;
    m.cb_max_col_nnz = blk_i_.data() + 3 * B;
    m.rb_ave_row_nnz = blk_d_.data();
    m.rb_std_row_nnz = blk_d_.data() + B;
    m.cb_ave_col_nnz = blk_d_.data() + 2 * B;
    m.cb_std_col_nnz = blk_d_.data() + 3 * B;
    d::check(spops_matrix_tile_features(d::ctx(), h_, (int64_t)B, &t_, &m), "spops_matrix_tile_features");
    is_symmetric_ = f_.pattern_symm == 1.0 && f_.value_symm == 1.0;
    computed_ = true;
    CalculateFeatures_time_ =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return true;
  }
  bool CalculateTilesFeatures() { return computed_ || CalculateFeatures(); }
  bool CalculateTilesExtraFeatures(const char*) { return computed_ || CalculateFeatures(); }

  bool ConvertToCSR(CSR_Matrix<IndexType, ValueType>& csr) {
    namespace d = spops_b200::detail;
    if (!h_) return false;
    const auto t0 = std::chrono::steady_clock::now();
    const spops_matrix_info_t i = d::info(h_);
    d::set_features<IndexType, ValueType>(csr, i.rows, i.cols, i.nnz);
    csr.row_offset = d::fetch<IndexType>(h_, SPOPS_ARR_ROW, nullptr);
    csr.col_index = d::fetch<IndexType>(h_, SPOPS_ARR_COL, nullptr);
    csr.values = d::fetch<ValueType>(h_, SPOPS_ARR_VAL, nullptr);
    ConvertToCSR_time_ = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return true;
  }

  void FeaturesPrint() {
    std::printf("[%lld]  %scounting by %d-bit Index, %d-bit Value\n", (long long)matrixID_, matrixName_.c_str(),
                (int)(8 * sizeof(IndexType)), (int)(8 * sizeof(ValueType)));
    std::printf("is_symmetric %d\npattern_symm %g%%\nvalue_symm   %g%%\n\n", is_symmetric_ ? 1 : 0,
                f_.pattern_symm * 100, f_.value_symm * 100);
    std::printf("num_rows   = %lld\nnum_cols   = %lld\nnnz_mtx    = %lld\nreal_nnz   = %lld\n", (long long)f_.rows,
                (long long)f_.cols, (long long)f_.nnz, (long long)f_.nnz);
    std::printf("nnz_ratio  = %g%%\nnum_of_diags  = %lld\nnnz_closed2diag_ratio = %g%%\n\n", f_.nnz_ratio * 100,
                (long long)f_.ndiags, f_.diag_close_ratio * 100);
    std::printf("nnz_lower    : %lld\nnnz_upper    : %lld\nnnz_diagonal : %lld\n\n", (long long)f_.nnz_lower,
                (long long)f_.nnz_upper, (long long)f_.nnz_diagonal);
    std::printf("NoneZero_Row_Ratio      : %g%%\nmin_nnz_each_row        : %lld\nmax_nnz_each_row        : %lld\n",
                f_.nz_row_ratio * 100, (long long)f_.min_nnz_row, (long long)f_.max_nnz_row);
    std::printf("ave_nnz_each_row        : %g\nvar_nnz_each_row        : %g\nstandard_dev_row        : %g\n",
                f_.ave_nnz_row, f_.var_nnz_row, f_.std_nnz_row);
    std::printf("P-ratio_row             : %g\nGini_coeff_row          : %g\n\n", f_.p_ratio_row, f_.gini_row);
    std::printf("NoneZero_Col_Ratio      : %g%%\nmin_nnz_each_col        : %lld\nmax_nnz_each_col        : %lld\n",
                f_.nz_col_ratio * 100, (long long)f_.min_nnz_col, (long long)f_.max_nnz_col);
    std::printf("ave_nnz_each_col        : %g\nvar_nnz_each_col        : %g\nstandard_dev_col        : %g\n",
                f_.ave_nnz_col, f_.var_nnz_col, f_.std_nnz_col);
    std::printf("P-ratio_col             : %g\nGini_coeff_col          : %g\n\n", f_.p_ratio_col, f_.gini_col);
    std::printf("diagonal_dominant_ratio : %g%%\n\n", f_.diagonal_dominant_ratio * 100);
    std::printf("max_value_offdiag  = %g\nmax_value_diagonal = %g\nrow_variability    = %g\n"
                "col_variability    = %g\n\n",
                f_.max_value_offdiag, f_.max_value_diagonal, f_.row_variability, f_.col_variability);
    std::printf("==========   Tile Features   ==========\nNumber of Tiles  : %lld\nTile inner size  : %lld * %lld\n",
                (long long)t_.num_blocks, (long long)t_.rows_per_block, (long long)t_.cols_per_block);
    std::printf("t_ave_nnz_tiles     : %g\nt_ave_nnz_RB        : %g\nt_ave_nnz_CB        : %g\n\n", t_.ave_nnz_tile,
                t_.ave_nnz_rb, t_.ave_nnz_cb);
    std::printf("t_var_nnz_tiles     : %g\nt_var_nnz_RB        : %g\nt_var_nnz_CB        : %g\n\n", t_.var_nnz_tile,
                t_.var_nnz_rb, t_.var_nnz_cb);
    std::printf("t_stand_dev_tiles     : %g\nt_stand_dev_RB        : %g\nt_stand_dev_CB        : %g\n\n",
                t_.std_nnz_tile, t_.std_nnz_rb, t_.std_nnz_cb);
    std::printf("min_nnz_each_tiles       : %lld\nmax_nnz_each_tiles       : %lld\n", (long long)t_.min_nnz_tile,
                (long long)t_.max_nnz_tile);
    std::printf("min_nnz_each_RB          : %lld\nmax_nnz_each_RB          : %lld\n", (long long)t_.min_nnz_rb,
                (long long)t_.max_nnz_rb);
    std::printf("min_nnz_each_CB          : %lld\nmax_nnz_each_CB          : %lld\n\n", (long long)t_.min_nnz_cb,
                (long long)t_.max_nnz_cb);
    std::printf("Gini_nnz_tiles     : %g\nGini_nnz_RB        : %g\nGini_nnz_CB        : %g\n\n", t_.gini_tiles,
                t_.gini_rb, t_.gini_cb);
    std::printf("P-ratio_tiles      : %g\nP-ratio_RB         : %g\nP-ratio_CB         : %g\n\n", t_.p_ratio_tiles,
                t_.p_ratio_rb, t_.p_ratio_cb);
    std::printf("NE_ratio_tiles_     : %g\nNE_ratio_RB         : %g\nNE_ratio_CB         : %g\n\n",
                t_.nz_ratio_tiles, t_.nz_ratio_rb, t_.nz_ratio_cb);
  }

  void ExtraFeaturesPrint() {
    std::printf("==========   Tile Extra Features   ==========\n");
    std::printf("uniq_R         = %g\nuniq_C         = %g\n\n", t_.uniq_r, t_.uniq_c);
    std::printf("GrX_uniqR      = %g\nGrX_uniqC      = %g\n\n", -1.0, -1.0);
    std::printf("potReuseR      = %g\npotReuseC      = %g\n\n", t_.pot_reuse_r, t_.pot_reuse_c);
    std::printf("GrX_potReuseR  = %g\nGrX_potReuseC  = %g\n\n", -1.0, -1.0);
    std::printf("ave_distance_= %g\n\n", t_.distance_per_row);
  }

  bool FeaturesWrite(const char* file_path) {
    if (!computed_) return true;
    const std::string dir = std::string(file_path ? file_path : ".") + "/" + matrixName_;
    std::error_code ec;
    std::filesystem::create_directories(dir, ec);
    if (ec) return true;
    const size_t B = 256, T = B * B;
    auto put_i = [&](const char* suffix, const int64_t* a, size_t n) {
      FILE* f = std::fopen((dir + "/" + matrixName_ + suffix).c_str(), "w");
      if (!f) return false;
      for (size_t i = 0; i < n; ++i) std::fprintf(f, "%lld\n", (long long)a[i]);
      std::fclose(f);
      return true;
    };
    auto put_d = [&](const char* suffix, const double* a, size_t n) {
      FILE* f = std::fopen((dir + "/" + matrixName_ + suffix).c_str(), "w");
      if (!f) return false;
      for (size_t i = 0; i < n; ++i) std::fprintf(f, "%g\n", a[i]);
      std::fclose(f);
      return true;
    };
    bool ok = put_d(".ave", tile_d_.data(), T) && put_i(".max", tile_i_.data() + 3 * T, T) &&
              put_i(".nnz", tile_i_.data(), T) && put_d(".std", tile_d_.data() + T, T) &&
              put_i(".RBmax", blk_i_.data() + B, B) && put_i(".RBnnz", blk_i_.data(), B) &&
              put_d(".RBave", blk_d_.data(), B) && put_d(".RBstd", blk_d_.data() + B, B) &&
              put_i(".CBmax", blk_i_.data() + 3 * B, B) && put_i(".CBnnz", blk_i_.data() + 2 * B, B) &&
              put_d(".CBave", blk_d_.data() + 2 * B, B) && put_d(".CBstd", blk_d_.data() + 3 * B, B);
    FILE* f = ok ? std::fopen((dir + "/" + matrixName_ + ".features").c_str(), "w") : nullptr;
    if (!f) return true;
    std::fprintf(f, "[%lld]: %s\n", (long long)matrixID_, matrixName_.c_str());
    std::fprintf(f, "num_rows %lld\nnum_cols %lld\nnum_nnz %lld\n", (long long)f_.rows, (long long)f_.cols,
                 (long long)f_.nnz);
    std::fprintf(f, "nnz_ratio %g\nnnz_on_maindiag_ratio %g\nnnz_row_distance_ratio %g\n", f_.nnz_ratio,
                 f_.diag_close_ratio, t_.distance_per_row / (double)f_.cols);
    std::fprintf(f, "nz_row_ratio %g\nmax_nnz_each_row %lld\nave_nnz_each_row %g\nstandard_dev_row %g\n",
                 f_.nz_row_ratio, (long long)f_.max_nnz_row, f_.ave_nnz_row, f_.std_nnz_row);
    std::fprintf(f, "P-ratio_row %g\nGini_coeff_row %g\n", f_.p_ratio_row, f_.gini_row);
    std::fprintf(f, "nz_col_ratio %g\nmax_nnz_each_col %lld\nave_nnz_each_col %g\nstandard_dev_col %g\n",
                 f_.nz_col_ratio, (long long)f_.max_nnz_col, f_.ave_nnz_col, f_.std_nnz_col);
    std::fprintf(f, "P-ratio_col %g\nGini_coeff_col %g\n", f_.p_ratio_col, f_.gini_col);
    std::fprintf(f, "nz_tiles_ratio %g\nmax_nnz_each_tiles %lld\nave_nnz_each_tiles %g\nstandard_dev_tiles %g\n",
                 t_.nz_ratio_tiles, (long long)t_.max_nnz_tile, t_.ave_nnz_tile, t_.std_nnz_tile);
    std::fprintf(f, "P-ratio_tiles %g\nGini_coeff_tiles %g\n", t_.p_ratio_tiles, t_.gini_tiles);
    std::fprintf(f, "nz_ratio_RB %g\nmax_nnz_each_RB %lld\nave_nnz_each_RB %g\nstandard_dev_RB %g\n",
                 t_.nz_ratio_rb, (long long)t_.max_nnz_rb, t_.ave_nnz_rb, t_.std_nnz_rb);
    std::fprintf(f, "P-ratio_RB %g\nGini_coeff_RB %g\n", t_.p_ratio_rb, t_.gini_rb);
    std::fprintf(f, "nz_ratio_CB %g\nmax_nnz_each_CB %lld\nave_nnz_each_CB %g\nstandard_dev_CB %g\n",
                 t_.nz_ratio_cb, (long long)t_.max_nnz_cb, t_.ave_nnz_cb, t_.std_nnz_cb);
    std::fprintf(f, "P-ratio_CB %g\nGini_coeff_CB %g\n", t_.p_ratio_cb, t_.gini_cb);
    std::fprintf(f, "uniq_R %g\nuniq_C %g\npotReuseR %g\npotReuseC %g\n", t_.uniq_r, t_.uniq_c, t_.pot_reuse_r,
                 t_.pot_reuse_c);
    std::fclose(f);
    return false;
  }

  // the computed values, by the C ABI's names
  const spops_features_t& features() const { return f_; }
  const spops_tile_features_t& tile_features() const { return t_; }

  double MtxLoad_time_ = 0.0;
  double CalculateFeatures_time_ = 0.0;
  double ConvertToCSR_time_ = 0.0;

 private:
  IndexType matrixID_ = 0;
  std::string matrixName_;
  spops_matrix_t h_ = nullptr;
  spops_features_t f_{};
  spops_tile_features_t t_{};
  std::vector<int64_t> tile_i_, blk_i_;
  std::vector<double> tile_d_, blk_d_;
  bool is_symmetric_ = false, computed_ = false;
};

#endif /* SPOPS_B200_CXX_SPOPS_H */
