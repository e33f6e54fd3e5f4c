// C entry points over the reference SparseOps library, compiled from the
// reference's own sources by oracle/Makefile into oracle/_ref/.
//
// Test infrastructure only.  This harness is the CHECKER used to (1) pin the
// CPU restatement in oracle/spops_oracle.cpp against the reference itself,
// (2) write the golden fixtures under tests/golden/, and (3) time the
// reference's own OpenMP kernels for bench.py's reference arm.  It is never
// linked into, or called by, the product library.
//
// Every function calls the reference's public API unchanged:
//   SpOps_<fmt>                       src/spmv_<fmt>.cpp (e.g. spmv_csr.cpp:165)
//   csr_to_<fmt>                      include/sparse_conversion.h:152-934
//   minhash_signatures_flat           include/spgemm_MinHashLSH.h:119
//   lsh_candidate_pairs_vector        include/spgemm_MinHashLSH.h:777
//   hierarchical_clustering_v0_fast   include/spgemm_utility.h:742
//   csr_reorder_rows / csr_to_vlength_cluster / vlength_cluster2csr
//                                     include/sparse_conversion.h:1640-1999
//   LeSpGEMM_VLength (kernel 3)       src/spgemm.cpp:661
//   csr_transpose                     include/sparse_conversion.h:2066
#include "SpOps.h"
#include "spgemm_MinHashLSH.h"
#include "spgemm_utility.h"

#include <cstdint>
#include <chrono>
#include <cstring>
#include <vector>

typedef long long ll;

namespace {

template <typename I, typename V>
CSR_Matrix<I, V> wrap_csr(I nr, I nc, I nnz, const I* rp, const I* ci, const V* v, int flag) {
  CSR_Matrix<I, V> A;
  std::memset(static_cast<void*>(&A), 0, sizeof(A));
  A.num_rows = nr;
  A.num_cols = nc;
  A.num_nnzs = nnz;
  A.row_offset = const_cast<I*>(rp);
  A.col_index = const_cast<I*>(ci);
  A.values = const_cast<V*>(v);
  A.partition = nullptr;
  A.kernel_flag = flag;
  return A;
}

// nnz-balanced thread partition, computed once per handle exactly as the
// reference's own test routine does for kernel_flag 2
// (utils/test_spmv_csr.cpp:60-65).
template <typename I>
I* make_partition(const I* rp, I nr) {
  const I t = Le_get_thread_num();
  I* part = new_array<I>(t + 1);
  balanced_partition_row_by_nnz(rp, nr, t, part);
  return part;
}

enum Kind { K_CSR = 1, K_SELLCS, K_SELLCR, K_SELL, K_ELL, K_DIA, K_BSR, K_COO };

struct FmtHandle {
  int kind = 0;
  int flag = 1;
  CSR_Matrix<int, double> csr{};
  SELL_C_Sigma_Matrix<int, double> scs{};
  SELL_C_R_Matrix<int, double> scr{};
  S_ELL_Matrix<int, double> sell{};
  ELL_Matrix<int, double> ell{};
  DIA_Matrix<int, double> dia{};
  BSR_Matrix<int, double> bsr{};
  COO_Matrix<int, double> coo{};
};

}  // namespace

extern "C" {

void ref_set_threads(int n) { Le_set_thread_num(n); }
int ref_get_threads(void) { return Le_get_thread_num(); }
int ref_num_procs(void) { return Le_get_core_num(); }

// ---------------------------------------------------------------- CSR SpMV
void ref_spmv_csr_f64(int nr, int nc, int nnz, const int* rp, const int* ci, const double* v,
                      double alpha, const double* x, double beta, double* y, int flag) {
  CSR_Matrix<int, double> A = wrap_csr<int, double>(nr, nc, nnz, rp, ci, v, flag);
  if (flag == 2) A.partition = make_partition(rp, nr);
  SpOps_csr<int, double>(alpha, A, x, beta, y);
  if (A.partition) delete_array(A.partition);
}

void ref_spmv_csr_f32(int nr, int nc, int nnz, const int* rp, const int* ci, const float* v,
                      float alpha, const float* x, float beta, float* y, int flag) {
  CSR_Matrix<int, float> A = wrap_csr<int, float>(nr, nc, nnz, rp, ci, v, flag);
  if (flag == 2) A.partition = make_partition(rp, nr);
  SpOps_csr<int, float>(alpha, A, x, beta, y);
  if (A.partition) delete_array(A.partition);
}

void ref_spmv_csr_f64_i64(ll nr, ll nc, ll nnz, const ll* rp, const ll* ci, const double* v,
                          double alpha, const double* x, double beta, double* y, int flag) {
  CSR_Matrix<long long, double> A = wrap_csr<long long, double>(nr, nc, nnz, rp, ci, v, flag);
  if (flag == 2) A.partition = make_partition<long long>(rp, nr);
  SpOps_csr<long long, double>(alpha, A, x, beta, y);
  if (A.partition) delete_array(A.partition);
}

// ------------------------------------------------ format handles (i32, f64)
// A handle owns the reference-built struct; info/copy expose its arrays and
// spmv runs the reference's own SpOps_<fmt> on it.
void* ref_fmt_build(int kind, int nr, int nc, int nnz, const int* rp, const int* ci,
                    const double* v, ll p0, ll p1, ll p2, int flag) {
  FmtHandle* h = new FmtHandle();
  h->kind = kind;
  h->flag = flag;
  CSR_Matrix<int, double> A = wrap_csr<int, double>(nr, nc, nnz, rp, ci, v, flag);
  switch (kind) {
    case K_CSR:
      h->csr = A;
      if (flag == 2) h->csr.partition = make_partition(rp, nr);
      break;
    case K_SELLCS:  // p0 = sigma, p1 = C, p2 = alignment
      h->scs = csr_to_sell_c_sigma<int, double>(A, nullptr, (int)p0, (int)p1, (int)p2);
      h->scs.kernel_flag = (flag == 2) ? 1 : flag;
      h->scs.partition = nullptr;
      break;
    case K_SELLCR:  // p1 = C, p2 = alignment
      h->scr = csr_to_sell_c_R<int, double>(A, nullptr, (int)p1, (int)p2);
      h->scr.kernel_flag = (flag == 2) ? 1 : flag;
      h->scr.partition = nullptr;
      break;
    case K_SELL:  // p1 = C, p2 = alignment
      h->sell = csr_to_sell<int, double>(A, nullptr, (int)p1, (int)p2);
      h->sell.kernel_flag = (flag == 2) ? 1 : flag;
      h->sell.partition = nullptr;
      break;
    case K_ELL:  // p0 = leading dimension (0 row-major, 1 col-major)
      h->ell = csr_to_ell<int, double>(A, p0 ? ColMajor : RowMajor);
      h->ell.kernel_flag = (flag == 2) ? 1 : flag;
      h->ell.partition = nullptr;
      break;
    case K_DIA:  // p0 = max diagonals, p2 = alignment
      h->dia = csr_to_dia<int, double>(A, (int)p0, nullptr, (int)p2);
      h->dia.kernel_flag = flag;
      h->dia.partition = nullptr;
      break;
    case K_BSR:  // p0 = block rows, p1 = block cols
      h->bsr = csr_to_bsr<int, double>(A, (int)p0, (int)p1);
      h->bsr.kernel_flag = (flag == 2) ? 1 : flag;
      h->bsr.partition = nullptr;
      break;
    case K_COO:
      h->coo = csr_to_coo<int, double>(A);
      h->coo.kernel_flag = (flag == 2) ? 1 : flag;
      h->coo.partition = nullptr;
      break;
    default:
      delete h;
      return nullptr;
  }
  return h;
}

// Scalar fields of the built struct, format specific:
//  SELLCS: [sliceNum, chunkNum, validchunkNum, chunk_num_per_slice, alignment, total_elems]
//  SELLCR: [validchunkNum, alignment, total_elems]
//  SELL  : [chunk_num, alignment, total_elems]
//  ELL   : [max_row_width, ld]
//  DIA   : [complete_ndiags, stride]
//  BSR   : [mb, nb, nnzb, blockDim_r, blockDim_c]
void ref_fmt_info(void* vh, ll* out) {
  FmtHandle* h = static_cast<FmtHandle*>(vh);
  switch (h->kind) {
    case K_SELLCS: {
      ll tot = 0;
      for (int c = 0; c < h->scs.validchunkNum; ++c) tot += (ll)h->scs.chunk_len[c] * h->scs.chunkWidth_C;
      out[0] = h->scs.sliceNum; out[1] = h->scs.chunkNum; out[2] = h->scs.validchunkNum;
      out[3] = h->scs.chunk_num_per_slice; out[4] = h->scs.alignment; out[5] = tot;
      break;
    }
    case K_SELLCR: {
      ll tot = 0;
      for (int c = 0; c < h->scr.validchunkNum; ++c) tot += (ll)h->scr.chunk_len[c] * h->scr.chunkWidth_C;
      out[0] = h->scr.validchunkNum; out[1] = h->scr.alignment; out[2] = tot;
      break;
    }
    case K_SELL: {
      ll tot = 0;
      for (int c = 0; c < h->sell.chunk_num; ++c) tot += (ll)h->sell.row_width[c] * h->sell.sliceWidth;
      out[0] = h->sell.chunk_num; out[1] = h->sell.alignment; out[2] = tot;
      break;
    }
    case K_ELL: out[0] = h->ell.max_row_width; out[1] = (ll)h->ell.ld; break;
    case K_DIA: out[0] = h->dia.complete_ndiags; out[1] = h->dia.stride; break;
    case K_BSR:
      out[0] = h->bsr.mb; out[1] = h->bsr.nb; out[2] = h->bsr.nnzb;
      out[3] = h->bsr.blockDim_r; out[4] = h->bsr.blockDim_c;
      break;
    default: break;
  }
}

// Copy the built arrays out.  Per-chunk arrays are concatenated in chunk order.
//  SELLCS/SELLCR: a=reorder[i32 n], b=chunk_len[i32], c=col (flat i32), d=val (flat f64)
//  SELL         : a=row_width[i32], c=col, d=val
//  ELL          : c=col [n*w], d=val
//  DIA          : a=diag_offsets[i64], d=diag_data [ndiag*stride]
//  BSR          : a=row_ptr[mb+1], b=block_colindex[nnzb], d=block_data
//  COO          : a=row_index, b=col_index, d=values
void ref_fmt_copy(void* vh, void* a, void* b, void* c, void* d) {
  FmtHandle* h = static_cast<FmtHandle*>(vh);
  auto cat = [](int nch, const int* len, int C, int* const* col, double* const* val, int* oc, double* ov) {
    ll off = 0;
    for (int k = 0; k < nch; ++k) {
      ll m = (ll)len[k] * C;
      if (oc) std::memcpy(oc + off, col[k], m * sizeof(int));
      if (ov) std::memcpy(ov + off, val[k], m * sizeof(double));
      off += m;
    }
  };
  switch (h->kind) {
    case K_SELLCS:
      if (a) std::memcpy(a, h->scs.reorder, (size_t)h->scs.num_rows * sizeof(int));
      if (b) std::memcpy(b, h->scs.chunk_len, (size_t)h->scs.validchunkNum * sizeof(int));
      cat(h->scs.validchunkNum, h->scs.chunk_len, h->scs.chunkWidth_C, h->scs.col_index,
          h->scs.values, (int*)c, (double*)d);
      break;
    case K_SELLCR:
      if (a) std::memcpy(a, h->scr.reorder, (size_t)h->scr.num_rows * sizeof(int));
      if (b) std::memcpy(b, h->scr.chunk_len, (size_t)h->scr.validchunkNum * sizeof(int));
      cat(h->scr.validchunkNum, h->scr.chunk_len, h->scr.chunkWidth_C, h->scr.col_index,
          h->scr.values, (int*)c, (double*)d);
      break;
    case K_SELL:
      if (a) std::memcpy(a, h->sell.row_width, (size_t)h->sell.chunk_num * sizeof(int));
      cat(h->sell.chunk_num, h->sell.row_width, h->sell.sliceWidth, h->sell.col_index,
          h->sell.values, (int*)c, (double*)d);
      break;
    case K_ELL: {
      size_t m = (size_t)h->ell.num_rows * h->ell.max_row_width;
      if (c) std::memcpy(c, h->ell.col_index, m * sizeof(int));
      if (d) std::memcpy(d, h->ell.values, m * sizeof(double));
      break;
    }
    case K_DIA: {
      size_t m = (size_t)h->dia.complete_ndiags * h->dia.stride;
      if (a) std::memcpy(a, h->dia.diag_offsets, (size_t)h->dia.complete_ndiags * sizeof(long));
      if (d) std::memcpy(d, h->dia.diag_data, m * sizeof(double));
      break;
    }
    case K_BSR:
      if (a) std::memcpy(a, h->bsr.row_ptr, (size_t)(h->bsr.mb + 1) * sizeof(int));
      if (b) std::memcpy(b, h->bsr.block_colindex, (size_t)h->bsr.nnzb * sizeof(int));
      if (d) std::memcpy(d, h->bsr.block_data, (size_t)h->bsr.nnzb * h->bsr.blockNNZ * sizeof(double));
      break;
    case K_COO:
      if (a) std::memcpy(a, h->coo.row_index, (size_t)h->coo.num_nnzs * sizeof(int));
      if (b) std::memcpy(b, h->coo.col_index, (size_t)h->coo.num_nnzs * sizeof(int));
      if (d) std::memcpy(d, h->coo.values, (size_t)h->coo.num_nnzs * sizeof(double));
      break;
    default: break;
  }
}

void ref_fmt_spmv(void* vh, double alpha, const double* x, double beta, double* y) {
  FmtHandle* h = static_cast<FmtHandle*>(vh);
  switch (h->kind) {
    case K_CSR: SpOps_csr<int, double>(alpha, h->csr, x, beta, y); break;
    case K_SELLCS: SpOps_sell_c_sigma<int, double>(alpha, h->scs, x, beta, y); break;
    case K_SELLCR: SpOps_sell_c_R<int, double>(alpha, h->scr, x, beta, y); break;
    case K_SELL: SpOps_sell<int, double>(alpha, h->sell, x, beta, y); break;
    case K_ELL: SpOps_ell<int, double>(alpha, h->ell, x, beta, y); break;
    case K_DIA: SpOps_dia<int, double>(alpha, h->dia, x, beta, y); break;
    case K_BSR: SpOps_bsr<int, double>(alpha, h->bsr, x, beta, y); break;
    case K_COO: SpOps_coo<int, double>(alpha, h->coo, x, beta, y); break;
    default: break;
  }
}

void ref_fmt_free(void* vh) {
  FmtHandle* h = static_cast<FmtHandle*>(vh);
  switch (h->kind) {
    case K_CSR: if (h->csr.partition) delete_array(h->csr.partition); break;
    case K_SELLCS: delete_host_matrix(h->scs); break;
    case K_SELLCR: delete_host_matrix(h->scr); break;
    case K_SELL: delete_host_matrix(h->sell); break;
    case K_ELL: delete_host_matrix(h->ell); break;
    case K_DIA: delete_host_matrix(h->dia); break;
    case K_BSR: delete_host_matrix(h->bsr); break;
    case K_COO: delete_host_matrix(h->coo); break;
    default: break;
  }
  delete h;
}

// ---------------------------------------------------------- MinHash / LSH
void ref_minhash_flat(const ll* rp, const ll* ci, ll n, int k, unsigned long long seed,
                      unsigned long long* out) {
  std::vector<uint64_t> s = minhash_signatures_flat<long long>(rp, ci, n, k, seed);
  std::memcpy(out, s.data(), s.size() * sizeof(uint64_t));
}

struct PairsHandle {
  std::vector<CandidatePair<int64_t, double>> pairs;
};

void* ref_lsh_pairs(const ll* rp, const ll* ci, ll n, int k, int bands, unsigned long long seed,
                    int constrain) {
  PairsHandle* h = new PairsHandle();
  h->pairs = lsh_candidate_pairs_vector<int64_t, double>((const int64_t*)rp, (const int64_t*)ci,
                                                         (int64_t)n, k, bands, seed, constrain != 0);
  return h;
}
ll ref_pairs_count(void* vh) { return (ll) static_cast<PairsHandle*>(vh)->pairs.size(); }
void ref_pairs_copy(void* vh, ll* i, ll* j, double* s) {
  PairsHandle* h = static_cast<PairsHandle*>(vh);
  for (size_t t = 0; t < h->pairs.size(); ++t) {
    i[t] = h->pairs[t].i;
    j[t] = h->pairs[t].j;
    s[t] = h->pairs[t].score;
  }
}
void ref_pairs_free(void* vh) { delete static_cast<PairsHandle*>(vh); }

// HC on an explicit pair list (i < j, sorted, unique, as LSH emits).
// Returns the number of clusters; perm[n], offsets[nclusters+1] (caller sizes n+1).
ll ref_hc(const ll* rp, const ll* ci, ll n, const ll* pi, const ll* pj, const double* ps, ll np,
          ll cluster_size, ll* perm, ll* offsets) {
  std::vector<CandidatePair<int64_t, double>> pairs((size_t)np);
  for (ll t = 0; t < np; ++t) pairs[t] = {pi[t], pj[t], ps[t]};
  std::vector<int64_t> p, o;
  hierarchical_clustering_v0_fast<int64_t, double>((const int64_t*)rp, (const int64_t*)ci,
                                                   (int64_t)n, pairs, (int64_t)cluster_size, p, o);
  std::memcpy(perm, p.data(), p.size() * sizeof(ll));
  std::memcpy(offsets, o.data(), o.size() * sizeof(ll));
  return (ll)o.size() - 1;
}

// --------------------------------------------------------------- LeSpGEMM
struct CsrHandle {
  CSR_Matrix<int64_t, double> C{};
  ll dense_clusters = 0;
  ll clusters = 0;
  ll nnzc = 0;
};

// The test driver's correctness path (test/test_spgemm_hc_lsh.cpp:230-300):
// reorder A by perm, build the variable-length clusters, run kernel 3, turn
// the clusters back into CSR and restore the original row order.
void* ref_spgemm_kernel3(ll a_rows, ll a_cols, ll a_nnz, const ll* arp, const ll* aci,
                         const double* av, ll b_rows, ll b_cols, ll b_nnz, const ll* brp,
                         const ll* bci, const double* bv, const ll* perm, const ll* offsets,
                         ll nclusters, int sort_output, double l2_fraction) {
  CSR_Matrix<int64_t, double> A = wrap_csr<int64_t, double>(a_rows, a_cols, a_nnz, (const int64_t*)arp,
                                                            (const int64_t*)aci, av, 0);
  CSR_Matrix<int64_t, double> B = wrap_csr<int64_t, double>(b_rows, b_cols, b_nnz, (const int64_t*)brp,
                                                            (const int64_t*)bci, bv, 0);
  std::vector<int64_t> permutation(perm, perm + a_rows);
  std::vector<int64_t> offs(offsets, offsets + nclusters + 1);
  CSR_Matrix<int64_t, double> Ar = csr_reorder_rows<int64_t, double>(A, permutation);
  CSR_VlengthCluster<int64_t, double> Ac = csr_to_vlength_cluster<int64_t, double>(Ar, offs);
  delete_host_matrix(Ar);
  CSR_VlengthCluster<int64_t, double> Cc;
  Cc.acc_flag = new_array<char>(Ac.rows);
  Cc.min_ccol = new_array<int64_t>(Ac.rows);
  Cc.max_ccol = new_array<int64_t>(Ac.rows);
  if (sort_output)
    LeSpGEMM_VLength<true, int64_t, double>(Ac, B, Cc, 3, l2_fraction);
  else
    LeSpGEMM_VLength<false, int64_t, double>(Ac, B, Cc, 3, l2_fraction);
  CsrHandle* h = new CsrHandle();
  h->dense_clusters = Cc.dense_cluster_count;
  h->clusters = Cc.rows;
  h->nnzc = Cc.nnzc;
  CSR_Matrix<int64_t, double> Ccsr = vlength_cluster2csr<int64_t, double>(Cc);
  std::vector<int64_t> inv((size_t)a_rows);
  for (ll t = 0; t < a_rows; ++t) inv[(size_t)permutation[t]] = t;
  h->C = csr_reorder_rows<int64_t, double>(Ccsr, inv);
  delete_host_matrix(Ccsr);
  delete_array(Cc.acc_flag);
  delete_array(Cc.min_ccol);
  delete_array(Cc.max_ccol);
  Cc.acc_flag = nullptr;
  Cc.min_ccol = nullptr;
  Cc.max_ccol = nullptr;
  delete_vlength_cluster_matrix(Cc);
  delete_vlength_cluster_matrix(Ac);
  return h;
}

// Kernel-3 timing without the conversions: returns ms for `iters` calls of
// LeSpGEMM_VLength on prebuilt clusters (the reference's performance mode,
// test/test_spgemm_hc_lsh.cpp:150-180).
double ref_spgemm_kernel3_time(ll a_rows, ll a_cols, ll a_nnz, const ll* arp, const ll* aci,
                               const double* av, ll b_rows, ll b_cols, ll b_nnz, const ll* brp,
                               const ll* bci, const double* bv, const ll* perm, const ll* offsets,
                               ll nclusters, int iters, double l2_fraction);

// info: [rows, cols, nnz, dense_clusters, clusters, nnzc]
void ref_csr_info(void* vh, ll* out) {
  CsrHandle* h = static_cast<CsrHandle*>(vh);
  out[0] = h->C.num_rows; out[1] = h->C.num_cols; out[2] = h->C.num_nnzs;
  out[3] = h->dense_clusters; out[4] = h->clusters; out[5] = h->nnzc;
}
void ref_csr_copy(void* vh, ll* rp, ll* ci, double* v) {
  CsrHandle* h = static_cast<CsrHandle*>(vh);
  std::memcpy(rp, h->C.row_offset, (size_t)(h->C.num_rows + 1) * sizeof(ll));
  if (h->C.num_nnzs) {
    std::memcpy(ci, h->C.col_index, (size_t)h->C.num_nnzs * sizeof(ll));
    std::memcpy(v, h->C.values, (size_t)h->C.num_nnzs * sizeof(double));
  }
}
void ref_csr_free(void* vh) {
  CsrHandle* h = static_cast<CsrHandle*>(vh);
  delete_host_matrix(h->C);
  delete h;
}

// ------------------------------------------------------------ COO -> CSR
// The reference's coo_to_csr<int64_t, double> (include/sparse_conversion.h:37)
// on caller arrays; the result is read back through ref_csr_info / copy / free.
void* ref_coo_to_csr(ll nr, ll nc, ll nnz, const ll* ri, const ll* ci, const double* v, int compact) {
  COO_Matrix<int64_t, double> coo;
  std::memset(static_cast<void*>(&coo), 0, sizeof(coo));
  coo.num_rows = nr;
  coo.num_cols = nc;
  coo.num_nnzs = nnz;
  coo.row_index = const_cast<int64_t*>((const int64_t*)ri);
  coo.col_index = const_cast<int64_t*>((const int64_t*)ci);
  coo.values = const_cast<double*>(v);
  CsrHandle* h = new CsrHandle();
  h->C = coo_to_csr<int64_t, double>(coo, compact != 0);
  return h;
}

// --------------------------------------------------------------- transpose
void* ref_csr_transpose(ll nr, ll nc, ll nnz, const ll* rp, const ll* ci, const double* v) {
  CSR_Matrix<int64_t, double> A = wrap_csr<int64_t, double>(nr, nc, nnz, (const int64_t*)rp,
                                                            (const int64_t*)ci, v, 0);
  CsrHandle* h = new CsrHandle();
  h->C = csr_transpose<int64_t, double>(A);
  return h;
}

// ------------------------------------------------------- Matrix Market
// read_csr_matrix<long long, V>(path, compact) (utils/sparse_io.cpp:193), float
// values widened to double in the handle.
void* ref_read_csr(const char* path, int compact, int f32) {
  CsrHandle* h = new CsrHandle();
  if (f32) {
    CSR_Matrix<long long, float> C = read_csr_matrix<long long, float>(path, compact != 0);
    h->C.num_rows = C.num_rows;
    h->C.num_cols = C.num_cols;
    h->C.num_nnzs = C.num_nnzs;
    h->C.row_offset = new_array<int64_t>(C.num_rows + 1);
    h->C.col_index = new_array<int64_t>(C.num_nnzs > 0 ? C.num_nnzs : 1);
    h->C.values = new_array<double>(C.num_nnzs > 0 ? C.num_nnzs : 1);
    for (ll t = 0; t <= (ll)C.num_rows; ++t) h->C.row_offset[t] = C.row_offset ? C.row_offset[t] : 0;
    for (ll t = 0; t < (ll)C.num_nnzs; ++t) {
      h->C.col_index[t] = C.col_index[t];
      h->C.values[t] = (double)C.values[t];
    }
    delete_host_matrix(C);
  } else {
    CSR_Matrix<long long, double> C = read_csr_matrix<long long, double>(path, compact != 0);
    h->C.num_rows = C.num_rows;
    h->C.num_cols = C.num_cols;
    h->C.num_nnzs = C.num_nnzs;
    h->C.row_offset = new_array<int64_t>(C.num_rows + 1);
    h->C.col_index = new_array<int64_t>(C.num_nnzs > 0 ? C.num_nnzs : 1);
    h->C.values = new_array<double>(C.num_nnzs > 0 ? C.num_nnzs : 1);
    for (ll t = 0; t <= (ll)C.num_rows; ++t) h->C.row_offset[t] = C.row_offset ? C.row_offset[t] : 0;
    for (ll t = 0; t < (ll)C.num_nnzs; ++t) {
      h->C.col_index[t] = C.col_index[t];
      h->C.values[t] = C.values[t];
    }
    delete_host_matrix(C);
  }
  return h;
}

// ---------------------------------------------------- row-wise and top-k
// LeSpGEMM<sortOutput, int64_t, double>(A, B, C, kernel_flag) (src/spgemm.cpp:683).
void* ref_spgemm_rowwise(ll a_rows, ll a_cols, ll a_nnz, const ll* arp, const ll* aci, const double* av, ll b_rows,
                         ll b_cols, ll b_nnz, const ll* brp, const ll* bci, const double* bv, int kernel_flag,
                         int sort_output) {
  CSR_Matrix<int64_t, double> A = wrap_csr<int64_t, double>(a_rows, a_cols, a_nnz, (const int64_t*)arp,
                                                            (const int64_t*)aci, av, 0);
  CSR_Matrix<int64_t, double> B = wrap_csr<int64_t, double>(b_rows, b_cols, b_nnz, (const int64_t*)brp,
                                                            (const int64_t*)bci, bv, 0);
  CsrHandle* h = new CsrHandle();
  if (sort_output)
    LeSpGEMM<true, int64_t, double>(A, B, h->C, kernel_flag);
  else
    LeSpGEMM<false, int64_t, double>(A, B, h->C, kernel_flag);
  return h;
}

// HashSpGEMMTopK<int64_t, V>(A, C, top_k) (src/spgemm.cpp:708); float values
// are widened to double in the handle.
void* ref_spgemm_topk(ll nr, ll nc, ll nnz, const ll* rp, const ll* ci, ll top_k, int f32) {
  CsrHandle* h = new CsrHandle();
  if (f32) {
    std::vector<float> ones((size_t)(nnz > 0 ? nnz : 1), 1.0f);
    CSR_Matrix<int64_t, float> A = wrap_csr<int64_t, float>(nr, nc, nnz, (const int64_t*)rp, (const int64_t*)ci,
                                                            ones.data(), 0);
    CSR_Matrix<int64_t, float> C{};
    HashSpGEMMTopK<int64_t, float>(A, C, (int64_t)top_k);
    h->C.num_rows = C.num_rows;
    h->C.num_cols = C.num_cols;
    h->C.num_nnzs = C.num_nnzs;
    h->C.row_offset = new_array<int64_t>(C.num_rows + 1);
    std::memcpy(h->C.row_offset, C.row_offset, (size_t)(C.num_rows + 1) * sizeof(int64_t));
    h->C.col_index = new_array<int64_t>(C.num_nnzs > 0 ? C.num_nnzs : 1);
    h->C.values = new_array<double>(C.num_nnzs > 0 ? C.num_nnzs : 1);
    for (ll t = 0; t < (ll)C.num_nnzs; ++t) {
      h->C.col_index[t] = C.col_index[t];
      h->C.values[t] = (double)C.values[t];
    }
    delete_host_matrix(C);
  } else {
    std::vector<double> ones((size_t)(nnz > 0 ? nnz : 1), 1.0);
    CSR_Matrix<int64_t, double> A = wrap_csr<int64_t, double>(nr, nc, nnz, (const int64_t*)rp, (const int64_t*)ci,
                                                              ones.data(), 0);
    HashSpGEMMTopK<int64_t, double>(A, h->C, (int64_t)top_k);
  }
  return h;
}

// Mean ms over `iters` calls of LeSpGEMM<false, int64_t, double>(A, B, C,
// kernel_flag), or of HashSpGEMMTopK<int64_t, double>(A, C, top_k) when
// top_k >= 0 (B unused); the output is freed outside the timed region.
double ref_spgemm_rowwise_time(ll a_rows, ll a_cols, ll a_nnz, const ll* arp, const ll* aci, const double* av,
                               ll b_rows, ll b_cols, ll b_nnz, const ll* brp, const ll* bci, const double* bv,
                               int kernel_flag, ll top_k, int iters) {
  CSR_Matrix<int64_t, double> A = wrap_csr<int64_t, double>(a_rows, a_cols, a_nnz, (const int64_t*)arp,
                                                            (const int64_t*)aci, av, 0);
  CSR_Matrix<int64_t, double> B = wrap_csr<int64_t, double>(b_rows, b_cols, b_nnz, (const int64_t*)brp,
                                                            (const int64_t*)bci, bv, 0);
  double total = 0;
  for (int it = 0; it < iters; ++it) {
    CSR_Matrix<int64_t, double> C{};
    auto t0 = std::chrono::steady_clock::now();
    if (top_k >= 0)
      HashSpGEMMTopK<int64_t, double>(A, C, (int64_t)top_k);
    else
      LeSpGEMM<false, int64_t, double>(A, B, C, kernel_flag);
    total += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    delete_host_matrix(C);
  }
  return iters > 0 ? total / iters : 0.0;
}

}  // extern "C"

extern "C" double ref_spgemm_kernel3_time(ll a_rows, ll a_cols, ll a_nnz, const ll* arp,
                                          const ll* aci, const double* av, ll b_rows, ll b_cols,
                                          ll b_nnz, const ll* brp, const ll* bci, const double* bv,
                                          const ll* perm, const ll* offsets, ll nclusters, int iters,
                                          double l2_fraction) {
  CSR_Matrix<int64_t, double> A = wrap_csr<int64_t, double>(a_rows, a_cols, a_nnz, (const int64_t*)arp,
                                                            (const int64_t*)aci, av, 0);
  CSR_Matrix<int64_t, double> B = wrap_csr<int64_t, double>(b_rows, b_cols, b_nnz, (const int64_t*)brp,
                                                            (const int64_t*)bci, bv, 0);
  std::vector<int64_t> permutation(perm, perm + a_rows);
  std::vector<int64_t> offs(offsets, offsets + nclusters + 1);
  CSR_Matrix<int64_t, double> Ar = csr_reorder_rows<int64_t, double>(A, permutation);
  CSR_VlengthCluster<int64_t, double> Ac = csr_to_vlength_cluster<int64_t, double>(Ar, offs);
  delete_host_matrix(Ar);
  double total_ms = 0.0;
  for (int it = 0; it < iters; ++it) {
    CSR_VlengthCluster<int64_t, double> Cc;
    Cc.acc_flag = new_array<char>(Ac.rows);
    Cc.min_ccol = new_array<int64_t>(Ac.rows);
    Cc.max_ccol = new_array<int64_t>(Ac.rows);
    double t0 = omp_get_wtime();
    LeSpGEMM_VLength<false, int64_t, double>(Ac, B, Cc, 3, l2_fraction);
    double t1 = omp_get_wtime();
    total_ms += (t1 - t0) * 1e3;
    delete_array(Cc.acc_flag);
    delete_array(Cc.min_ccol);
    delete_array(Cc.max_ccol);
    Cc.acc_flag = nullptr;
    Cc.min_ccol = nullptr;
    Cc.max_ccol = nullptr;
    delete_vlength_cluster_matrix(Cc);
  }
  delete_vlength_cluster_matrix(Ac);
  return total_ms / (iters > 0 ? iters : 1);
}
