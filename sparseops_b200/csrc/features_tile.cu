// Tile features of a CSR matrix on the device (spops_matrix_tile_features).
//
// The reference's MTX class counts, while it reads a Matrix Market file
// (src/sparse_features.cpp:181-265), the entries of every tile of a
// num_blocks x num_blocks grid, every row block (RB) and column block (CB),
// and which rows and columns of a tile hold an entry; after the read it
// derives per-tile and per-block row statistics (:484-625) and summarises
// the tile, RB and CB counts in CalculateTilesFeatures (:783-846).  Here the
// same numbers come from a CSR handle:
//   * a pass over A's rows: a warp takes a row, histograms the column blocks
//     of its entries in shared memory, and every (row, column block) with
//     count c adds c to the tile's entries, 1 to its rows, c^2 to its sum of
//     squares and raises its maximum.  A CTA only covers rows of one row
//     block, so it accumulates that block's num_blocks tiles in shared memory
//     and adds them to the device arrays once (integer atomics: the result
//     does not depend on the order).  Row lengths give the RB maximum and sum
//     of squares, and (last - first column) / length the row distance of
//     CalculateTilesExtraFeatures (:943-965), summed per CTA in a fixed order;
//   * the same pass over the handle's transpose (rows of A^T are A's
//     columns): the columns of A per tile, the CB maximum and squares;
//   * the standard deviations from exact integer moments: over the R rows of
//     a block, sum (c - N/R)^2 = (R * S2 - N^2) / R, so they do not depend on
//     a summation order either;
//   * the count summaries (min, max, mean, squared deviations, P-ratio,
//     Gini) with the shared count statistics of features.cu, and the
//     reference's starting values applied to them on the host.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "spops_internal.h"

namespace spops {
namespace {

typedef unsigned long long ull;

constexpr int kMaxBlocks = 2048;
constexpr int kWarps = 8;
constexpr int64_t kRowsPerCta = 256;

inline unsigned grid_of(int64_t work, int threads = 256) {
  int64_t g = (work + threads - 1) / threads;
  return (unsigned)(g < 1 ? 1 : g);
}

// n items in B blocks: the first m blocks hold q + 1 items, the others q
struct Split {
  int64_t q, m, th;  // th = m * (q + 1): the first item of the short blocks
  double inv1, inv0;  // 1 / (q + 1), 1 / q (0 when q == 0)
  __host__ __device__ int64_t size(int64_t b) const { return b < m ? q + 1 : q; }
  __host__ __device__ int64_t start(int64_t b) const { return b < m ? b * (q + 1) : th + (b - m) * q; }
  // a / d for 0 <= a < 2^52 through a double reciprocal, corrected to the
  // exact quotient
  __device__ __forceinline__ static int64_t quot(int64_t a, int64_t d, double inv) {
    if (d <= 0) return 0;  // not reached for indices inside the matrix
    int64_t x = (int64_t)((double)a * inv);
    while (x > 0 && x * d > a) --x;
    while ((x + 1) * d <= a) ++x;
    return x;
  }
  __device__ __forceinline__ int block(int64_t i) const {
    return i < th ? (int)quot(i, q + 1, inv1) : (int)(m + quot(i - th, q, inv0));
  }
};

Split make_split(int64_t n, int64_t B) {
  Split s;
  s.q = n / B;
  s.m = n % B;
  s.th = s.m * (s.q + 1);
  s.inv1 = 1.0 / (double)(s.q + 1);
  s.inv0 = s.q ? 1.0 / (double)s.q : 0.0;
  return s;
}

struct PassOut {
  ull* nnz;      // [B*B] entries per tile (NULL: not counted)
  ull* s2;       // [B*B] sum over rows of (entries in the tile)^2
  ull* max;      // [B*B] largest row count in the tile
  ull* rows;     // [B*B] rows with an entry in the tile
  ull* blk_max;  // [B] longest row of the block
  ull* blk_s2;   // [B] sum of squared row lengths of the block
  double* dist;  // [grid] per-CTA sum of row distances (NULL: not needed)
};

// CTA blockIdx.x = b * cpb + k covers rows [start(b) + k * kRowsPerCta, ...)
// of row block b; tile (b, t) is stored at b * s_major + t * s_minor.
template <typename I>
__global__ void __launch_bounds__(kWarps * 32) tile_pass_kernel(const I* __restrict__ rp, const I* __restrict__ ci,
                                                              Split rs, Split cs, int B, int64_t cpb,
                                                              int64_t s_major, int64_t s_minor, PassOut o) {
  extern __shared__ __align__(16) unsigned char smem[];
  ull* acc_rows = reinterpret_cast<ull*>(smem);
  ull* acc_nnz = acc_rows + B;
  ull* acc_s2 = acc_nnz + B;
  double* wdist = reinterpret_cast<double*>(acc_s2 + B);
  ull* blk = reinterpret_cast<ull*>(wdist + kWarps);  // [0] max, [1] squares
  unsigned* acc_max = reinterpret_cast<unsigned*>(blk + 2);
  int* hist = reinterpret_cast<int*>(acc_max + B);
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int64_t b = blockIdx.x / cpb, k = blockIdx.x % cpb;
  const int64_t r_lo = rs.start(b) + k * kRowsPerCta;
  const int64_t r_hi = min(rs.start(b) + rs.size(b), r_lo + kRowsPerCta);
  for (int i = tid; i < kWarps * B; i += blockDim.x) hist[i] = 0;
  for (int i = tid; i < B; i += blockDim.x) {
    acc_rows[i] = 0;
    acc_nnz[i] = 0;
    acc_s2[i] = 0;
    acc_max[i] = 0;
  }
  if (tid < 2) blk[tid] = 0;
  __syncthreads();
  int* h = hist + w * B;
  double dist = 0.0;
  ull lmax = 0, ls2 = 0;
  for (int64_t r = r_lo + w; r < r_hi; r += kWarps) {
    const int64_t s = (int64_t)rp[r], e = (int64_t)rp[r + 1];
    for (int64_t j = s + lane; j < e; j += 32) atomicAdd(&h[cs.block((int64_t)ci[j])], 1);
    __syncwarp();
    // the first lane to take a block's count flushes it
    for (int64_t j = s + lane; j < e; j += 32) {
      const int t = cs.block((int64_t)ci[j]);
      const int c = atomicExch(&h[t], 0);
      if (c) {
        atomicAdd(&acc_rows[t], 1ULL);
        if (o.nnz) {
          atomicAdd(&acc_nnz[t], (ull)c);
          atomicAdd(&acc_s2[t], (ull)c * (ull)c);
          atomicMax(&acc_max[t], (unsigned)c);
        }
      }
    }
    __syncwarp();
    if (lane == 0) {
      const ull len = (ull)(e - s);
      lmax = max(lmax, len);
      ls2 += len * len;
      if (o.dist && len) dist += (double)((int64_t)ci[e - 1] - (int64_t)ci[s]) / (double)len;
    }
  }
  if (lane == 0) {
    if (lmax) atomicMax(&blk[0], lmax);
    if (ls2) atomicAdd(&blk[1], ls2);
    wdist[w] = dist;
  }
  __syncthreads();
  for (int t = tid; t < B; t += blockDim.x) {
    const ull nr = acc_rows[t];
    if (!nr) continue;
    const int64_t idx = b * s_major + (int64_t)t * s_minor;
    atomicAdd(&o.rows[idx], nr);
    if (o.nnz) {
      atomicAdd(&o.nnz[idx], acc_nnz[t]);
      atomicAdd(&o.s2[idx], acc_s2[t]);
      atomicMax(&o.max[idx], (ull)acc_max[t]);
    }
  }
  if (tid == 0) {
    if (blk[0]) atomicMax(&o.blk_max[b], blk[0]);
    if (blk[1]) atomicAdd(&o.blk_s2[b], blk[1]);
    if (o.dist) {
      double d = 0.0;
      for (int i = 0; i < kWarps; ++i) d += wdist[i];
      o.dist[blockIdx.x] = d;
    }
  }
}

// sum over R rows of (c - N/R)^2 = (R * S2 - N^2) / R, from exact integers
__device__ __forceinline__ double sq_dev(ull R, ull S2, ull N) {
  const unsigned __int128 x = (unsigned __int128)R * S2 - (unsigned __int128)N * N;
  const double hi = (double)(ull)(x >> 64), lo = (double)(ull)x;
  return (hi * 18446744073709551616.0 + lo) / (double)R;
}

// per tile (i = tr * B + tc): mean and population deviation of its rows'
// entry counts over the R rows of row block tr
__global__ void tile_finish_kernel(const ull* __restrict__ nnz, const ull* __restrict__ s2, Split rs, int B,
                                   int64_t* __restrict__ nnz64, double* __restrict__ ave,
                                   double* __restrict__ sd) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= (int64_t)B * B) return;
  const ull R = (ull)rs.size(i / B), N = nnz[i];
  nnz64[i] = (int64_t)N;
  ave[i] = R ? (double)N / (double)R : 0.0;
  sd[i] = R ? sqrt(sq_dev(R, s2[i], N) / (double)R) : 0.0;
}

// per block: entries (from the row pointer), mean and deviation of its row
// lengths
template <typename I>
__global__ void block_finish_kernel(const I* __restrict__ rp, Split rs, int B, const ull* __restrict__ s2,
                                    int64_t* __restrict__ nnz, double* __restrict__ ave, double* __restrict__ sd) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  const int64_t r0 = rs.start(b), R = rs.size(b);
  const ull N = R ? (ull)((int64_t)rp[r0 + R] - (int64_t)rp[r0]) : 0;
  nnz[b] = (int64_t)N;
  ave[b] = R ? (double)N / (double)R : 0.0;
  sd[b] = R ? sqrt(sq_dev((ull)R, s2[b], N) / (double)R) : 0.0;
}

__global__ void to_i64_kernel(const ull* __restrict__ a, int64_t m, int64_t* __restrict__ b) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < m) b[i] = (int64_t)a[i];
}

size_t pass_smem(int B) { return (size_t)B * 8 * 3 + kWarps * 8 + 16 + (size_t)B * 4 + (size_t)kWarps * B * 4; }

template <typename I>
spops_status_t run_pass(Context* ctx, const Matrix* M, const Split& rs, const Split& cs, int B, int64_t s_major,
                        int64_t s_minor, const PassOut& o, int64_t* grid_out) {
  const int64_t longest = rs.m ? rs.q + 1 : rs.q;
  const int64_t cpb = (longest + kRowsPerCta - 1) / kRowsPerCta;
  *grid_out = (int64_t)B * cpb;
  if (cpb == 0) return SPOPS_OK;
  const size_t sm = pass_smem(B);
  static int set_for[64] = {0};  // per device: the largest dynamic size allowed so far
  const int dev = ctx->device & 63;
  if ((int)sm > set_for[dev]) {
    SPOPS_CUDA(cudaFuncSetAttribute(tile_pass_kernel<I>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    set_for[dev] = (int)sm;
  }
  tile_pass_kernel<I><<<(unsigned)(B * cpb), kWarps * 32, sm, ctx->stream>>>(
      M->row.as<I>(), M->col.as<I>(), rs, cs, B, cpb, s_major, s_minor, o);
  SPOPS_LAUNCH_CHECK();
  return SPOPS_OK;
}

template <typename T>
spops_status_t download(Context* ctx, T* host, const void* dev, int64_t count) {
  if (host && count > 0)
    SPOPS_CUDA(cudaMemcpyAsync(host, dev, (size_t)count * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream));
  return SPOPS_OK;
}

// the reference's CalculateTilesFeatures on one count vector: the non-empty
// ratio and the variance start from -1, min from 100000000
void summarise(const CountSummary& c, int64_t len, double ave, int64_t* mn, int64_t* mx, double* nzr,
               double* ave_out, double* var, double* sd, double* p, double* gini) {
  *mn = std::min<int64_t>(c.mn, 100000000);
  *mx = std::max<int64_t>(c.mx, 0);
  *nzr = ((double)c.nz - 1.0) / (double)len;
  *ave_out = ave;
  *var = (c.sq - 1.0) / (double)len;
  *sd = std::sqrt(std::max(*var, 0.0));
  *p = c.p;
  *gini = c.gini;
}

template <typename I>
spops_status_t tile_features_t(Context* ctx, Matrix* A, int B, spops_tile_features_t* f,
                               const spops_tile_maps_t* maps) {
  cudaStream_t st = ctx->stream;
  const int64_t n = A->rows, nc = A->cols, nnz = A->nnz, T = (int64_t)B * B;
  std::memset(f, 0, sizeof(*f));
  const Split rs = make_split(n, B), cs = make_split(nc, B);
  f->num_blocks = B;
  f->rows_per_block = rs.q;
  f->rows_mod = rs.m;
  f->cols_per_block = cs.q;
  f->cols_mod = cs.m;
  Matrix* AT = nullptr;
  SPOPS_TRY(csr_transpose_view(ctx, A, &AT));
  // device arrays: tiles (nnz, s2, max, rows, cols as ull; nnz64; ave, sd),
  // blocks (max, s2 for RB and CB; nnz64, ave, sd for RB and CB)
  PoolBuf tiles(ctx), blocks(ctx), dist(ctx), red(ctx), tmp(ctx);
  SPOPS_TRY(tiles.alloc((size_t)T * 8 * 8));
  SPOPS_TRY(blocks.alloc((size_t)B * 8 * 10));
  ull* t_nnz = tiles.as<ull>();
  ull* t_s2 = t_nnz + T;
  ull* t_max = t_s2 + T;
  ull* t_rows = t_max + T;
  ull* t_cols = t_rows + T;
  int64_t* t_nnz64 = reinterpret_cast<int64_t*>(t_cols + T);
  double* t_ave = reinterpret_cast<double*>(t_nnz64 + T);
  double* t_sd = t_ave + T;
  ull* rb_max = blocks.as<ull>();
  ull* rb_s2 = rb_max + B;
  ull* cb_max = rb_s2 + B;
  ull* cb_s2 = cb_max + B;
  int64_t* rb_nnz = reinterpret_cast<int64_t*>(cb_s2 + B);
  int64_t* cb_nnz = rb_nnz + B;
  double* rb_ave = reinterpret_cast<double*>(cb_nnz + B);
  double* rb_sd = rb_ave + B;
  double* cb_ave = rb_sd + B;
  double* cb_sd = cb_ave + B;
  SPOPS_CUDA(cudaMemsetAsync(tiles.p, 0, (size_t)T * 8 * 5, st));
  SPOPS_CUDA(cudaMemsetAsync(blocks.p, 0, (size_t)B * 8 * 4, st));
  const int64_t cpb_r = ((rs.m ? rs.q + 1 : rs.q) + kRowsPerCta - 1) / kRowsPerCta;
  const int64_t grid_r = (int64_t)B * cpb_r;
  SPOPS_TRY(dist.alloc((size_t)std::max<int64_t>(grid_r, 1) * 8));
  int64_t g = 0;
  SPOPS_TRY(run_pass<I>(ctx, A, rs, cs, B, B, 1, PassOut{t_nnz, t_s2, t_max, t_rows, rb_max, rb_s2, dist.as<double>()},
                        &g));
  SPOPS_TRY(run_pass<I>(ctx, AT, cs, rs, B, 1, B, PassOut{nullptr, nullptr, nullptr, t_cols, cb_max, cb_s2, nullptr},
                        &g));
  tile_finish_kernel<<<grid_of(T), 256, 0, st>>>(t_nnz, t_s2, rs, B, t_nnz64, t_ave, t_sd);
  block_finish_kernel<I><<<grid_of(B), 256, 0, st>>>(A->row.as<I>(), rs, B, rb_s2, rb_nnz, rb_ave, rb_sd);
  block_finish_kernel<I><<<grid_of(B), 256, 0, st>>>(AT->row.as<I>(), cs, B, cb_s2, cb_nnz, cb_ave, cb_sd);
  SPOPS_LAUNCH_CHECK();
  // sums: rows per tile, columns per tile, row distances
  SPOPS_TRY(red.alloc(64));
  ull* r_sum = red.as<ull>();
  double* d_sum = reinterpret_cast<double*>(r_sum + 2);
  size_t b1 = 0, b2 = 0;
  SPOPS_CUDA(cub::DeviceReduce::Sum(nullptr, b1, t_rows, r_sum, T, st));
  if (grid_r > 0) SPOPS_CUDA(cub::DeviceReduce::Sum(nullptr, b2, dist.as<double>(), d_sum, grid_r, st));
  SPOPS_TRY(tmp.alloc(std::max(b1, b2) + 256));
  SPOPS_CUDA(cub::DeviceReduce::Sum(tmp.p, b1, t_rows, r_sum, T, st));
  SPOPS_CUDA(cub::DeviceReduce::Sum(tmp.p, b1, t_cols, r_sum + 1, T, st));
  SPOPS_CUDA(cudaMemsetAsync(d_sum, 0, 8, st));
  if (grid_r > 0) SPOPS_CUDA(cub::DeviceReduce::Sum(tmp.p, b2, dist.as<double>(), d_sum, grid_r, st));
  CountSummary ts, rbs, cbs;
  SPOPS_TRY(count_summary(ctx, t_nnz64, T, nnz, &ts));
  SPOPS_TRY(count_summary(ctx, rb_nnz, B, nnz, &rbs));
  SPOPS_TRY(count_summary(ctx, cb_nnz, B, nnz, &cbs));
  ull h_sums[2] = {0, 0};
  double h_dist = 0.0;
  SPOPS_CUDA(cudaMemcpyAsync(h_sums, r_sum, 16, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaMemcpyAsync(&h_dist, d_sum, 8, cudaMemcpyDeviceToHost, st));
  if (maps) {
    if (maps->tile_nnz) SPOPS_TRY(download(ctx, maps->tile_nnz, t_nnz64, T));
    if (maps->tile_rows) SPOPS_TRY(download(ctx, maps->tile_rows, t_rows, T));
    if (maps->tile_cols) SPOPS_TRY(download(ctx, maps->tile_cols, t_cols, T));
    if (maps->tile_max_row_nnz) SPOPS_TRY(download(ctx, maps->tile_max_row_nnz, t_max, T));
    if (maps->tile_ave_row_nnz) SPOPS_TRY(download(ctx, maps->tile_ave_row_nnz, t_ave, T));
    if (maps->tile_std_row_nnz) SPOPS_TRY(download(ctx, maps->tile_std_row_nnz, t_sd, T));
    if (maps->rb_nnz) SPOPS_TRY(download(ctx, maps->rb_nnz, rb_nnz, B));
    if (maps->rb_max_row_nnz) SPOPS_TRY(download(ctx, maps->rb_max_row_nnz, rb_max, B));
    if (maps->rb_ave_row_nnz) SPOPS_TRY(download(ctx, maps->rb_ave_row_nnz, rb_ave, B));
    if (maps->rb_std_row_nnz) SPOPS_TRY(download(ctx, maps->rb_std_row_nnz, rb_sd, B));
    if (maps->cb_nnz) SPOPS_TRY(download(ctx, maps->cb_nnz, cb_nnz, B));
    if (maps->cb_max_col_nnz) SPOPS_TRY(download(ctx, maps->cb_max_col_nnz, cb_max, B));
    if (maps->cb_ave_col_nnz) SPOPS_TRY(download(ctx, maps->cb_ave_col_nnz, cb_ave, B));
    if (maps->cb_std_col_nnz) SPOPS_TRY(download(ctx, maps->cb_std_col_nnz, cb_sd, B));
  }
  SPOPS_CUDA(cudaStreamSynchronize(st));
  const double ave_t = (double)nnz / ((double)B * (double)B), ave_b = (double)nnz / (double)B;
  summarise(ts, T, ave_t, &f->min_nnz_tile, &f->max_nnz_tile, &f->nz_ratio_tiles, &f->ave_nnz_tile,
            &f->var_nnz_tile, &f->std_nnz_tile, &f->p_ratio_tiles, &f->gini_tiles);
  summarise(rbs, B, ave_b, &f->min_nnz_rb, &f->max_nnz_rb, &f->nz_ratio_rb, &f->ave_nnz_rb, &f->var_nnz_rb,
            &f->std_nnz_rb, &f->p_ratio_rb, &f->gini_rb);
  summarise(cbs, B, ave_b, &f->min_nnz_cb, &f->max_nnz_cb, &f->nz_ratio_cb, &f->ave_nnz_cb, &f->var_nnz_cb,
            &f->std_nnz_cb, &f->p_ratio_cb, &f->gini_cb);
  f->uniq_r = (double)h_sums[0] / (double)nnz;
  f->uniq_c = (double)h_sums[1] / (double)nnz;
  f->pot_reuse_r = (double)h_sums[0] / (double)n;
  f->pot_reuse_c = (double)h_sums[1] / (double)nc;
  f->distance_per_row = h_dist / (double)n;
  return SPOPS_OK;
}

}  // namespace
}  // namespace spops

using namespace spops;

extern "C" {

spops_status_t spops_matrix_tile_features(spops_context_t ctx, spops_matrix_t csr, int64_t num_blocks,
                                          spops_tile_features_t* features, const spops_tile_maps_t* maps) {
  if (!ctx || !csr || !features) return fail(SPOPS_ERR_INVALID, "spops_matrix_tile_features: null argument");
  if (csr->format != SPOPS_FMT_CSR) return fail(SPOPS_ERR_INVALID, "spops_matrix_tile_features: needs a CSR matrix");
  if (num_blocks <= 0) num_blocks = 256;
  if (num_blocks > kMaxBlocks)
    return fail(SPOPS_ERR_TOO_LARGE, "spops_matrix_tile_features: num_blocks %lld > %d", (long long)num_blocks,
                kMaxBlocks);
  DeviceGuard g(ctx->device);
  if (!csr->plan.ready) SPOPS_TRY(csr_analyse(ctx, csr));  // validates the pattern
  if (csr->itype == SPOPS_INDEX_I32) return tile_features_t<int32_t>(ctx, csr, (int)num_blocks, features, maps);
  return tile_features_t<int64_t>(ctx, csr, (int)num_blocks, features, maps);
}

}  // extern "C"
