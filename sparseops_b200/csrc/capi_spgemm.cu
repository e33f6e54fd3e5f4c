// C ABI of the LeSpGEMM path: MinHash signatures, LSH candidate pairs,
// hierarchical clustering and the cluster-wise SpGEMM.
#include <chrono>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "spops_internal.h"

using namespace spops;

struct spops_pairs_s : spops::PairSet {
  spops::Context* ctx = nullptr;
};

namespace {

// The CSR pattern of A as int64 host arrays (for the host clustering), copied
// once per handle and kept on it: a handle's pattern never changes
// (spops_csr_set_values replaces values only).
spops_status_t host_pattern(Context* ctx, Matrix* A, const std::vector<int64_t>** rp_out,
                            const std::vector<int64_t>** ci_out) {
  *rp_out = &A->host_rp;
  *ci_out = &A->host_ci;
  if (A->host_rp.size() == (size_t)A->rows + 1) return SPOPS_OK;
  std::vector<int64_t> rp((size_t)A->rows + 1), ci((size_t)A->nnz);
  cudaStream_t st = ctx->stream;
  if (A->itype == SPOPS_INDEX_I64) {
    SPOPS_CUDA(cudaMemcpyAsync(rp.data(), A->row.p, rp.size() * 8, cudaMemcpyDeviceToHost, st));
    if (A->nnz) SPOPS_CUDA(cudaMemcpyAsync(ci.data(), A->col.p, ci.size() * 8, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
  } else {
    std::vector<int32_t> r32(rp.size()), c32(ci.size());
    SPOPS_CUDA(cudaMemcpyAsync(r32.data(), A->row.p, r32.size() * 4, cudaMemcpyDeviceToHost, st));
    if (A->nnz) SPOPS_CUDA(cudaMemcpyAsync(c32.data(), A->col.p, c32.size() * 4, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
    std::copy(r32.begin(), r32.end(), rp.begin());
    std::copy(c32.begin(), c32.end(), ci.begin());
  }
  A->host_rp.swap(rp);
  A->host_ci.swap(ci);
  return SPOPS_OK;
}

void put_stats(const SpgemmStats& s, spops_spgemm_stats_t* o) {
  if (!o) return;
  o->flops = s.flops;
  o->clusters = s.clusters;
  o->dense_clusters = s.dense_clusters;
  o->pairs = s.pairs;
  o->cluster_columns = s.cluster_columns;
  o->c_cluster_columns = s.c_cluster_columns;
  o->minhash_ms = s.minhash_ms;
  o->lsh_ms = s.lsh_ms;
  o->hc_ms = s.hc_ms;
  o->cluster_ms = s.cluster_ms;
  o->symbolic_ms = s.symbolic_ms;
  o->numeric_ms = s.numeric_ms;
  o->to_csr_ms = s.to_csr_ms;
}

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

extern "C" {

spops_status_t spops_minhash(spops_context_t ctx, spops_matrix_t A, int32_t k, uint64_t seed, void* sig) {
  if (!ctx || !A || (!sig && A->rows > 0)) return fail(SPOPS_ERR_INVALID, "spops_minhash: null argument");
  DeviceGuard g(ctx->device);
  return minhash_signatures(ctx, A, k, seed, static_cast<uint64_t*>(sig));
}

spops_status_t spops_minhash_host(spops_context_t ctx, spops_matrix_t A, int32_t k, uint64_t seed, void* sig_host) {
  if (!ctx || !A || (!sig_host && A->rows > 0)) return fail(SPOPS_ERR_INVALID, "spops_minhash_host: null argument");
  if (k <= 0) return fail(SPOPS_ERR_INVALID, "spops_minhash_host: k must be positive");
  DeviceGuard g(ctx->device);
  const size_t bytes = (size_t)std::max<int64_t>(A->rows, 1) * (size_t)k * 8;
  DevBuf sig;
  SPOPS_TRY(sig.alloc(bytes));
  spops_status_t s = minhash_signatures(ctx, A, k, seed, sig.as<uint64_t>());
  if (s == SPOPS_OK && A->rows > 0) {
    const cudaError_t e = cudaMemcpyAsync(sig_host, sig.p, (size_t)A->rows * (size_t)k * 8, cudaMemcpyDeviceToHost,
                                          ctx->stream);
    const cudaError_t e2 = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess || e2 != cudaSuccess)
      s = fail(SPOPS_ERR_CUDA, "spops_minhash_host: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
  }
  sig.release();
  return s;
}

spops_status_t spops_lsh_pairs_from_signatures(spops_context_t ctx, const void* sig, int64_t rows, int32_t k,
                                               int32_t bands, int32_t constrain, spops_pairs_t* out) {
  if (!ctx || !out || (!sig && rows > 0)) return fail(SPOPS_ERR_INVALID, "spops_lsh_pairs_from_signatures: null");
  DeviceGuard g(ctx->device);
  spops_pairs_s* P = new spops_pairs_s();
  P->ctx = ctx;
  spops_status_t s = lsh_pairs(ctx, static_cast<const uint64_t*>(sig), rows, k, bands, constrain != 0, P);
  if (s != SPOPS_OK) {
    P->release();
    delete P;
    return s;
  }
  *out = P;
  return SPOPS_OK;
}

spops_status_t spops_lsh_pairs(spops_context_t ctx, spops_matrix_t A, int32_t k, int32_t bands, uint64_t seed,
                               int32_t constrain, spops_pairs_t* out) {
  if (!ctx || !A || !out) return fail(SPOPS_ERR_INVALID, "spops_lsh_pairs: null argument");
  if (k <= 0) return fail(SPOPS_ERR_INVALID, "spops_lsh_pairs: k must be positive");
  DeviceGuard g(ctx->device);
  DevBuf sig;
  SPOPS_TRY(sig.alloc((size_t)std::max<int64_t>(A->rows, 1) * k * 8));
  spops_status_t s = minhash_signatures(ctx, A, k, seed, sig.as<uint64_t>());
  if (s == SPOPS_OK) s = spops_lsh_pairs_from_signatures(ctx, sig.p, A->rows, k, bands, constrain, out);
  SPOPS_CUDA(cudaStreamSynchronize(ctx->stream));
  sig.release();
  return s;
}

spops_status_t spops_pairs_count(spops_pairs_t P, int64_t* count) {
  if (!P || !count) return fail(SPOPS_ERR_INVALID, "spops_pairs_count: null argument");
  *count = P->count;
  return SPOPS_OK;
}

spops_status_t spops_pairs_arrays(spops_pairs_t P, const int64_t** i, const int64_t** j, const double** score) {
  if (!P) return fail(SPOPS_ERR_INVALID, "spops_pairs_arrays: null pairs");
  if (i) *i = P->pi.as<int64_t>();
  if (j) *j = P->pj.as<int64_t>();
  if (score) *score = P->score.as<double>();
  return SPOPS_OK;
}

spops_status_t spops_pairs_download(spops_pairs_t P, int64_t* i, int64_t* j, double* score) {
  if (!P) return fail(SPOPS_ERR_INVALID, "spops_pairs_download: null pairs");
  if (P->count == 0) return SPOPS_OK;
  DeviceGuard g(P->ctx->device);
  cudaStream_t st = P->ctx->stream;
  const size_t b = (size_t)P->count * 8;
  if (i) SPOPS_CUDA(cudaMemcpyAsync(i, P->pi.p, b, cudaMemcpyDeviceToHost, st));
  if (j) SPOPS_CUDA(cudaMemcpyAsync(j, P->pj.p, b, cudaMemcpyDeviceToHost, st));
  if (score) SPOPS_CUDA(cudaMemcpyAsync(score, P->score.p, b, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  return SPOPS_OK;
}

spops_status_t spops_pairs_destroy(spops_pairs_t P) {
  if (!P) return SPOPS_OK;
  DeviceGuard g(P->ctx->device);
  cudaStreamSynchronize(P->ctx->stream);
  P->release();
  delete P;
  return SPOPS_OK;
}

spops_status_t spops_hierarchical_clustering(const int64_t* row_ptr, const int64_t* col_index, int64_t rows,
                                             const int64_t* pi, const int64_t* pj, const double* score,
                                             int64_t npairs, int64_t cluster_size, int64_t* permutation,
                                             int64_t* offsets, int64_t* nclusters) {
  if (rows < 0 || npairs < 0 || (rows > 0 && (!row_ptr || !permutation || !offsets)) ||
      (npairs > 0 && (!pi || !pj || !score)) || !nclusters)
    return fail(SPOPS_ERR_INVALID, "spops_hierarchical_clustering: null argument");
  std::vector<int64_t> perm, offs;
  SPOPS_TRY(hierarchical_clustering(row_ptr, col_index, rows, pi, pj, score, npairs, cluster_size, perm, offs));
  std::memcpy(permutation, perm.data(), perm.size() * 8);
  std::memcpy(offsets, offs.data(), offs.size() * 8);
  *nclusters = (int64_t)offs.size() - 1;
  return SPOPS_OK;
}

spops_status_t spops_spgemm_clustered(spops_context_t ctx, spops_matrix_t A, spops_matrix_t B,
                                      const int64_t* permutation, const int64_t* offsets, int64_t nclusters,
                                      int32_t sort_output, double l2_budget_bytes, spops_matrix_t* C,
                                      spops_spgemm_stats_t* stats) {
  if (!ctx || !A || !B || !C || !offsets || (A->rows > 0 && !permutation))
    return fail(SPOPS_ERR_INVALID, "spops_spgemm_clustered: null argument");
  DeviceGuard g(ctx->device);
  SpgemmStats s;
  Matrix* out = nullptr;
  SPOPS_TRY(cluster_spgemm(ctx, A, B, permutation, offsets, nclusters, sort_output != 0, l2_budget_bytes, &out, &s));
  *C = static_cast<spops_matrix_s*>(out);
  put_stats(s, stats);
  return SPOPS_OK;
}

spops_status_t spops_spgemm_rowwise(spops_context_t ctx, spops_matrix_t A, spops_matrix_t B, int32_t kernel_flag,
                                    int32_t sort_output, spops_matrix_t* C, spops_spgemm_stats_t* stats) {
  if (!ctx || !A || !B || !C) return fail(SPOPS_ERR_INVALID, "spops_spgemm_rowwise: null argument");
  (void)kernel_flag;  // kernels 1-3 give the same entries; columns always ascending here
  DeviceGuard g(ctx->device);
  SpgemmStats s;
  Matrix* out = nullptr;
  SPOPS_TRY(rowwise_spgemm(ctx, A, B, sort_output != 0, &out, &s));
  *C = static_cast<spops_matrix_s*>(out);
  put_stats(s, stats);
  return SPOPS_OK;
}

spops_status_t spops_spgemm_topk(spops_context_t ctx, spops_matrix_t A, int64_t top_k, spops_matrix_t* C) {
  if (!ctx || !A || !C) return fail(SPOPS_ERR_INVALID, "spops_spgemm_topk: null argument");
  DeviceGuard g(ctx->device);
  Matrix* out = nullptr;
  SPOPS_TRY(topk_spgemm(ctx, A, top_k, &out));
  *C = static_cast<spops_matrix_s*>(out);
  return SPOPS_OK;
}

spops_status_t spops_spgemm_lsh(spops_context_t ctx, spops_matrix_t A, spops_matrix_t B, int32_t k, int32_t bands,
                                uint64_t seed, int64_t cluster_size, int32_t sort_output, double l2_budget_bytes,
                                spops_matrix_t* C, spops_spgemm_stats_t* stats) {
  if (!ctx || !A || !B || !C) return fail(SPOPS_ERR_INVALID, "spops_spgemm_lsh: null argument");
  DeviceGuard g(ctx->device);
  SpgemmStats s;
  auto t0 = std::chrono::steady_clock::now();
  PoolBuf sig(ctx);
  SPOPS_TRY(sig.alloc((size_t)std::max<int64_t>(A->rows, 1) * (size_t)std::max(k, 1) * 8));
  spops_status_t st = minhash_signatures(ctx, A, k, seed, sig.as<uint64_t>());
  if (st != SPOPS_OK) {
    sig.release();
    return st;
  }
  cudaStreamSynchronize(ctx->stream);
  s.minhash_ms = ms_since(t0);
  t0 = std::chrono::steady_clock::now();
  PairSet P;
  st = lsh_pairs(ctx, sig.as<uint64_t>(), A->rows, k, bands, true, &P);
  cudaStreamSynchronize(ctx->stream);
  sig.release();
  if (st != SPOPS_OK) return st;
  s.lsh_ms = ms_since(t0);
  s.pairs = P.count;
  t0 = std::chrono::steady_clock::now();
  const bool trace = std::getenv("SPOPS_TRACE") && std::getenv("SPOPS_TRACE")[0] == '1';
  auto lap = [&](const char* what) {
    if (trace) std::fprintf(stderr, "[spgemm_lsh] %-24s %9.3f ms\n", what, ms_since(t0));
  };
  std::vector<int64_t> pi((size_t)P.count), pj((size_t)P.count), perm, offs;
  std::vector<double> ps((size_t)P.count);
  const std::vector<int64_t>* rp = nullptr;
  const std::vector<int64_t>* ci = nullptr;
  st = host_pattern(ctx, A, &rp, &ci);
  lap("pattern to host");
  if (st == SPOPS_OK && P.count) {
    cudaMemcpy(pi.data(), P.pi.p, pi.size() * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(pj.data(), P.pj.p, pj.size() * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(ps.data(), P.score.p, ps.size() * 8, cudaMemcpyDeviceToHost);
  }
  P.release();
  lap("pairs to host");
  if (st == SPOPS_OK)
    st = hierarchical_clustering(rp->data(), ci->data(), A->rows, pi.data(), pj.data(), ps.data(), (int64_t)pi.size(),
                                 cluster_size, perm, offs);
  if (st != SPOPS_OK) return st;
  lap("clustering");
  s.hc_ms = ms_since(t0);
  Matrix* out = nullptr;
  SpgemmStats s2;
  SPOPS_TRY(cluster_spgemm(ctx, A, B, perm.data(), offs.data(), (int64_t)offs.size() - 1, sort_output != 0,
                           l2_budget_bytes, &out, &s2));
  s2.minhash_ms = s.minhash_ms;
  s2.lsh_ms = s.lsh_ms;
  s2.hc_ms = s.hc_ms;
  s2.pairs = s.pairs;
  *C = static_cast<spops_matrix_s*>(out);
  put_stats(s2, stats);
  return SPOPS_OK;
}

}  // extern "C"
