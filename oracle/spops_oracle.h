/* CPU restatement of the SparseOps hot-path algorithms: the ORACLE.
 *
 * Test infrastructure only.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load this library, and only as the checker or
 * the timed CPU baseline; the product library never links or calls it.
 *
 * Each function restates one reference algorithm in plain sequential code and
 * cites the reference file:line it follows.  It is pinned against the
 * reference itself (oracle/_ref, compiled from the reference sources) through
 * the golden fixtures under tests/golden/ (tests/test_oracle_golden.py).
 */
#ifndef SPOPS_ORACLE_H
#define SPOPS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* y = alpha*A*x + beta*y, one sequential sum per row in stored order
 * (src/spmv_csr.cpp:74-91).  alpha==1 && beta==0 stores the sum. */
void orc_spmv_csr_f64_i32(int64_t nr, const int32_t* rp, const int32_t* ci, const double* v,
                          double alpha, const double* x, double beta, double* y);
void orc_spmv_csr_f64_i64(int64_t nr, const int64_t* rp, const int64_t* ci, const double* v,
                          double alpha, const double* x, double beta, double* y);
/* FP32 inputs, FP64 accumulation: the exact-as-possible reference for FP32. */
void orc_spmv_csr_f32_i32(int64_t nr, const int32_t* rp, const int32_t* ci, const float* v,
                          double alpha, const float* x, double beta, const float* y_in, double* y);
/* sum_j |a_ij * x_j| per row: the denominator of the componentwise error. */
void orc_absdot_csr_f64_i32(int64_t nr, const int32_t* rp, const int32_t* ci, const double* v,
                            const double* x, double* out);
/* Multi-RHS: Y[:,c] = alpha*A*X[:,c] + beta*Y[:,c]; X, Y row-major [n x k]. */
void orc_spmm_csr_f64_i32(int64_t nr, const int32_t* rp, const int32_t* ci, const double* v,
                          int64_t k, double alpha, const double* X, double beta, double* Y);

/* SELL-C-sigma row order and chunk lengths (include/sparse_conversion.h:344-425). */
void orc_sell_c_sigma_layout(int64_t nr, const int32_t* rp, int64_t sigma, int64_t C, int64_t align,
                             int32_t* reorder, int32_t* chunk_len);
/* S-ELL chunk widths (include/sparse_conversion.h:265-306). */
void orc_sell_row_width(int64_t nr, const int32_t* rp, int64_t C, int64_t align, int32_t* width);
/* DIA diagonal offsets in first-appearance order (include/sparse_conversion.h:619-762).
 * Returns the number of diagonals (writes at most max_out). */
int64_t orc_dia_offsets(int64_t nr, int64_t nc, const int32_t* rp, const int32_t* ci, int64_t max_out,
                        int64_t* offsets);
/* BSR block structure (include/sparse_conversion.h:776-885).  Returns nnzb;
 * block_col is written only when non-null (size it with a first call). */
int64_t orc_bsr_structure(int64_t nr, int64_t nc, const int32_t* rp, const int32_t* ci, int64_t br,
                          int64_t bc, int32_t* row_ptr, int32_t* block_col);

/* MinHash signatures, row-major [n x k] (include/spgemm_MinHashLSH.h:119-180). */
void orc_minhash(const int64_t* rp, const int64_t* ci, int64_t n, int32_t k, uint64_t seed, uint64_t* sig);
/* LSH candidate pairs (include/spgemm_MinHashLSH.h:427-605), as a handle. */
void* orc_lsh_pairs(const uint64_t* sig, int64_t n, int32_t k, int32_t bands, int32_t constrain);
int64_t orc_pairs_count(void* h);
void orc_pairs_copy(void* h, int64_t* i, int64_t* j, double* score);
void orc_pairs_free(void* h);
/* Hierarchical clustering (include/spgemm_utility.h:742-915).  perm[n],
 * offsets[nclusters+1] (size it n+1); returns nclusters. */
int64_t orc_hc(const int64_t* rp, const int64_t* ci, int64_t n, const int64_t* pi, const int64_t* pj,
               const double* ps, int64_t np, int64_t cluster_size, int64_t* perm, int64_t* offsets);

/* Cluster-wise C = A*B as the kernel-3 pipeline defines the result
 * (src/spgemm_Vlength_mixed.cpp, include/sparse_conversion.h:1777-1862):
 * handle with the final CSR in original row order, columns ascending. */
void* orc_spgemm(int64_t a_rows, const int64_t* arp, const int64_t* aci, const double* av, int64_t b_rows,
                 int64_t b_cols, const int64_t* brp, const int64_t* bci, const double* bv, const int64_t* perm,
                 const int64_t* offsets, int64_t nclusters, int32_t sort_output, double l2_budget_bytes);
/* Row-wise C = A*B (src/spgemm.cpp:44-235): every structural entry kept,
 * columns ascending. */
void* orc_spgemm_rowwise(int64_t a_rows, const int64_t* arp, const int64_t* aci, const double* av, int64_t b_rows,
                         const int64_t* brp, const int64_t* bci, const double* bv);
/* HashSpGEMMTopK (src/spgemm.cpp:708-842): top_k Jaccard-similar rows per
 * row, (similarity descending, column ascending); f32: float arithmetic. */
void* orc_spgemm_topk(int64_t n, const int64_t* arp, const int64_t* aci, int64_t ncols, int64_t top_k, int32_t f32);
/* [rows, nnz, dense_clusters, flops] */
void orc_csr_info(void* h, int64_t* out);
void orc_csr_copy(void* h, int64_t* rp, int64_t* ci, double* v, double* absv);
void orc_csr_free(void* h);
/* 2 * sum of intermediate products (src/spgemm.cpp:24-42). */
int64_t orc_spgemm_flop(int64_t a_rows, const int64_t* arp, const int64_t* aci, int64_t b_rows,
                        const int64_t* brp);

/* COO -> CSR (include/sparse_conversion.h:37-99), with compact != 0 the
 * duplicate summation of include/sparse_operation.h:21-69.  Output arrays
 * sized nnz (rp: n + 1); returns the output entry count. */
int64_t orc_coo_to_csr_f64(int64_t n, int64_t nnz, const int64_t* ri, const int64_t* ci, const double* v,
                           int32_t compact, int64_t* rp, int64_t* oc, double* ov);
int64_t orc_coo_to_csr_f32(int64_t n, int64_t nnz, const int64_t* ri, const int64_t* ci, const float* v,
                           int32_t compact, int64_t* rp, int64_t* oc, float* ov);

/* Structure features (src/sparse_features.cpp:643-775 with MtxLoad's counts,
 * :336-478) of a general CSR matrix, in spops_features_t order (32 values). */
void orc_features(int64_t n, int64_t nc, const int64_t* rp, const int64_t* ci, const double* v, double* out);
void orc_tile_features(int64_t n, int64_t nc, const int64_t* rp, const int64_t* ci, int64_t B, double* sc,
                       int64_t* tile_i, double* tile_d, int64_t* blk_i, double* blk_d);

/* y = A^T g by scatter (the value the reference's csr_transpose + SpOps_csr
 * gives, include/sparse_conversion.h:2066-2108), FP64. */
void orc_spmv_t_csr_f64_i32(int64_t nr, int64_t nc, const int32_t* rp, const int32_t* ci, const double* v,
                            const double* g, double* y);
/* out[k] = g[row(k)] * x[col(k)] on A's pattern. */
void orc_sddmm_csr_f64_i32(int64_t nr, const int32_t* rp, const int32_t* ci, const double* g, const double* x,
                           double* out);

#ifdef __cplusplus
}
#endif
#endif
