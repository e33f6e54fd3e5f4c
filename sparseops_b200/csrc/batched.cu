// Batched SpMV / SpMM: many matrices of uneven sizes in ONE persistent launch.
//
// No reference counterpart (the reference runs one SpOps_<fmt> call per
// matrix and has no multi-RHS product); its per-matrix loop is the baseline.
//
// A batch lists work items (matrix, kind, index) over all its matrices, in
// matrix order so each matrix's x stays in L2 while its items run:
//   kind 0  CSR segment of the matrix's CSR plan (csr_segment_spmv / _spmm)
//   kind 1  32 stored rows of the matrix's padded (SELL) form (padded_rows32)
//   kind 2  one piece of a long padded row (padded_piece)
//   kind 3  four tiles of the matrix's CSR tile plan (separate tile-item
//           launch and a batch-wide calibration; k = 1, 8, 16, 32)
// A persistent grid (SMs x resident blocks) of warps walks the item list.
// Per-matrix pointers live in a device table; the launch itself (on the
// batch's own stream, ordered against the caller's stream with events) can
// be captured once into a CUDA graph and replayed.
//
// Autotuner (spops_batch_tune): per matrix, times the candidate forms with
// CUDA events on the device -- CSR (segments of kCsrCap entries), and
// SELL-C-sigma with C = 32 and sigma in {256, 4096}, row-major and
// column-major chunks -- and keeps the fastest for the batched launch, then
// times the whole batch with those choices and with every matrix in CSR and
// keeps the faster of the two.  With one right-hand side a CSR matrix runs
// as SpMV tile items (the single-matrix tile kernel's body) when its arrays
// allow the vector loads, otherwise as segments.  For k > 1 the CSR form is
// used and the tuner picks the RHS tile (8 or 32 lanes).
#include <algorithm>
#include <cstring>
#include <vector>

#include "device_util.cuh"
#include "csr_tile.cuh"
#include "spops_internal.h"
#include "warp_work.cuh"

namespace spops {

struct BatchItem {
  int32_t mat;
  int32_t kind;
  int64_t idx;
};

struct BatchMat {
  // CSR form
  const void* rp;
  const void* ci;
  const void* val;
  const CsrSeg* seg;
  void* partial;  // CSR long-row chunk sums (k per chunk for SpMM)
  int* counter;
  // padded form
  const void* pcol;
  const void* pval;
  const void* chunk_len;
  const int64_t* chunk_off;
  const int* row_len;
  const void* reorder;
  const PadPiece* pieces;
  void* ppartial;
  int* pcounter;
  int64_t C;
  int32_t colmajor;
  int32_t band;  // x window half-width of the CSR segments (0: none)
  int64_t rows, cols;
  // vectors
  const void* x;
  void* y;
  int64_t ldx, ldy;
  // k = 8 register tiles on the matrix's SpMV tile plan (csr_tile.cuh)
  const int64_t* tile_row;
  const uint8_t* tflags;
  int64_t tiles, nnz;
  void* tcin;      // V [tiles * 8]: heads before each tile's first row start
  void* tosum;     // V [tiles * 8]: the row open at each tile's end
  int64_t* topen;  // [tiles]: that row, or -1
  const int64_t* tempty;
  int64_t tnempty;
};

namespace {

constexpr int kBatchBlock = 256;

// Items are taken from a queue (next_item, zeroed before the launch) kGrab at
// a time, the next grab requested while the current one runs: the items in
// flight stay a contiguous window of the list, so the matrices whose vectors
// must be in L2 at once are the one or two that window covers.  (A fixed
// stride per warp lets warps drift apart across many matrices.)
constexpr int kGrab = 2;

template <typename I, typename V, int KT, bool kBand = false>
__global__ void __launch_bounds__(kBatchBlock, KT == 1 ? 4 : 3) batch_kernel(const BatchItem* __restrict__ items, int64_t nitems,
                                                               const BatchMat* __restrict__ mats, int64_t k, V alpha,
                                                               V beta, bool bz,
                                                               unsigned long long* __restrict__ next_item) {
  __shared__ V prod_all[KT == 1 ? kBatchBlock / 32 : 1][KT == 1 ? 2 * kCsrCap : 1];
  // staged x windows (kBand: the context option "batch_band")
  __shared__ V xs_all[KT == 1 && kBand ? kBatchBlock / 32 : 1][KT == 1 && kBand ? kBandWin : 1];
  extern __shared__ __align__(16) unsigned char batch_dyn_smem[];  // SpMM: one SpmmStage per warp
  const int lane = threadIdx.x & 31;
  V* prod = prod_all[KT == 1 ? threadIdx.x >> 5 : 0];
  SpmmStage<I, V>& stage = reinterpret_cast<SpmmStage<I, V>*>(batch_dyn_smem)[KT == 1 ? 0 : threadIdx.x >> 5];
  unsigned long long grab = 0, ahead = 0;
  if (lane == 0) {
    grab = atomicAdd(next_item, (unsigned long long)kGrab);
    ahead = atomicAdd(next_item, (unsigned long long)kGrab);
  }
  grab = __shfl_sync(0xffffffffu, grab, 0);
  for (;;) {
    if ((int64_t)grab >= nitems) break;
    const int64_t jend = (int64_t)grab + kGrab < nitems ? (int64_t)grab + kGrab : nitems;
    for (int64_t j = (int64_t)grab; j < jend; ++j) {
    const BatchItem it = items[j];
    const BatchMat& M = mats[it.mat];
    if (KT == 1) {
      if (it.kind == 0) {
        csr_segment_spmv<I, V, 8>(M.seg[it.idx], it.idx, static_cast<const I*>(M.ci), static_cast<const V*>(M.val),
                                  static_cast<const I*>(M.rp), static_cast<const V*>(M.x), static_cast<V*>(M.y),
                                  alpha, beta, bz, prod, static_cast<V*>(M.partial), M.counter, lane,
                                  kBand ? M.band : 0, M.cols, xs_all[KT == 1 && kBand ? threadIdx.x >> 5 : 0]);
      } else if (it.kind == 1) {
        if (M.colmajor)
          padded_rows32<I, V, true>(it.idx * 32, static_cast<const I*>(M.pcol), static_cast<const V*>(M.pval),
                                    static_cast<const I*>(M.chunk_len), M.chunk_off, M.row_len,
                                    static_cast<const I*>(M.reorder), M.rows, M.C, static_cast<const V*>(M.x),
                                    static_cast<V*>(M.y), alpha, beta, bz, lane);
        else
          padded_rows32<I, V, false>(it.idx * 32, static_cast<const I*>(M.pcol), static_cast<const V*>(M.pval),
                                     static_cast<const I*>(M.chunk_len), M.chunk_off, M.row_len,
                                     static_cast<const I*>(M.reorder), M.rows, M.C, static_cast<const V*>(M.x),
                                     static_cast<V*>(M.y), alpha, beta, bz, lane);
      } else {
        if (M.colmajor)
          padded_piece<I, V, true>(it.idx, M.pieces[it.idx], static_cast<const I*>(M.pcol),
                                   static_cast<const V*>(M.pval), static_cast<const I*>(M.chunk_len), M.chunk_off,
                                   M.row_len, static_cast<const I*>(M.reorder), M.C, static_cast<const V*>(M.x),
                                   static_cast<V*>(M.y), alpha, beta, bz, static_cast<V*>(M.ppartial), M.pcounter,
                                   lane);
        else
          padded_piece<I, V, false>(it.idx, M.pieces[it.idx], static_cast<const I*>(M.pcol),
                                    static_cast<const V*>(M.pval), static_cast<const I*>(M.chunk_len), M.chunk_off,
                                    M.row_len, static_cast<const I*>(M.reorder), M.C, static_cast<const V*>(M.x),
                                    static_cast<V*>(M.y), alpha, beta, bz, static_cast<V*>(M.ppartial), M.pcounter,
                                    lane);
      }
    } else {
      csr_segment_spmm<I, V, KT>(M.seg[it.idx], it.idx, static_cast<const I*>(M.ci), static_cast<const V*>(M.val),
                                 static_cast<const I*>(M.rp), static_cast<const V*>(M.x), M.ldx,
                                 static_cast<V*>(M.y), M.ldy, k, alpha, beta, bz, static_cast<V*>(M.partial),
                                 M.counter, stage, lane);
    }
    }
    grab = __shfl_sync(0xffffffffu, ahead, 0);
    if (lane == 0 && (int64_t)grab < nitems) ahead = atomicAdd(next_item, (unsigned long long)kGrab);
  }
}

// Tile items (k = 8, 16, 32): item idx covers tiles [idx, idx + kTilesPerItem) of its
// matrix, taken from the queue as in batch_kernel.
constexpr int64_t kTilesPerItem = 4;

template <typename I, typename V, int G>
__global__ void __launch_bounds__(kBatchBlock, 2) batch_tile_kernel(const BatchItem* __restrict__ items,
                                                                   int64_t nitems, const BatchMat* __restrict__ mats,
                                                                   V alpha, V beta, bool bz,
                                                                   unsigned long long* __restrict__ next_item) {
  const int lane = threadIdx.x & 31;
  unsigned long long grab = 0, ahead = 0;
  if (lane == 0) {
    grab = atomicAdd(next_item, (unsigned long long)kGrab);
    ahead = atomicAdd(next_item, (unsigned long long)kGrab);
  }
  grab = __shfl_sync(0xffffffffu, grab, 0);
  for (;;) {
    if ((int64_t)grab >= nitems) break;
    const int64_t jend = (int64_t)grab + kGrab < nitems ? (int64_t)grab + kGrab : nitems;
    for (int64_t j = (int64_t)grab; j < jend; ++j) {
      const BatchItem it = items[j];
      const BatchMat& M = mats[it.mat];
      const int64_t t1 = it.idx + kTilesPerItem < M.tiles ? it.idx + kTilesPerItem : M.tiles;
      for (int64_t t = it.idx; t < t1; ++t)
        spmm_tile_groups<I, V, G>(static_cast<const I*>(M.rp), M.rows, M.nnz, static_cast<const I*>(M.ci),
                                  static_cast<const V*>(M.val), M.tile_row, M.tflags, t, static_cast<const V*>(M.x),
                                  M.ldx, static_cast<V*>(M.y), M.ldy, alpha, beta, bz, static_cast<V*>(M.tcin),
                                  static_cast<V*>(M.tosum), M.topen, lane);
    }
    grab = __shfl_sync(0xffffffffu, ahead, 0);
    if (lane == 0 && (int64_t)grab < nitems) ahead = atomicAdd(next_item, (unsigned long long)kGrab);
  }
}

// Tile items with one right-hand side: the SpMV tile body (csr_tile.cuh; the
// default single-matrix CSR kernel) over tiles [idx, idx + kTilesPerItem) of
// the item's matrix, the next tile's entries loaded before this one's
// gathers are used.
template <typename I, typename V>
__global__ void __launch_bounds__(kBatchBlock, 2) batch_tile1_kernel(const BatchItem* __restrict__ items,
                                                                    int64_t nitems, const BatchMat* __restrict__ mats,
                                                                    V alpha, V beta, bool bz,
                                                                    unsigned long long* __restrict__ next_item) {
  constexpr int K = 8;
  const int lane = threadIdx.x & 31;
  unsigned long long grab = 0, ahead = 0;
  if (lane == 0) {
    grab = atomicAdd(next_item, (unsigned long long)kGrab);
    ahead = atomicAdd(next_item, (unsigned long long)kGrab);
  }
  grab = __shfl_sync(0xffffffffu, grab, 0);
  for (;;) {
    if ((int64_t)grab >= nitems) break;
    const int64_t jend = (int64_t)grab + kGrab < nitems ? (int64_t)grab + kGrab : nitems;
    for (int64_t j = (int64_t)grab; j < jend; ++j) {
      const BatchItem it = items[j];
      const BatchMat& M = mats[it.mat];
      const I* ci = static_cast<const I*>(M.ci);
      const V* val = static_cast<const V*>(M.val);
      const V* x = static_cast<const V*>(M.x);
      const int64_t t1 = it.idx + kTilesPerItem < M.tiles ? it.idx + kTilesPerItem : M.tiles;
      I c[K];
      V a[K];
      int64_t t = it.idx;
      tile_load<I, V, K>(ci, val, M.nnz, t, lane, c, a);
      uint32_t flags = M.tflags[t * 32 + lane];
      int64_t tr = M.tile_row[t];
      for (; t < t1; ++t) {
        V pr[K];
#pragma unroll
        for (int b = 0; b < K; ++b) pr[b] = a[b] * ld_gather(x + c[b]);
        const uint32_t f = flags;
        const int64_t r0 = tr;
        if (t + 1 < t1) {
          tile_load<I, V, K>(ci, val, M.nnz, t + 1, lane, c, a);
          flags = M.tflags[(t + 1) * 32 + lane];
          tr = M.tile_row[t + 1];
        }
        tile_finish<I, V, K>(static_cast<const I*>(M.rp), M.rows, M.nnz, t, lane, f, r0, pr, static_cast<V*>(M.y),
                             alpha, beta, bz, static_cast<V*>(M.tcin), static_cast<V*>(M.tosum), M.topen);
      }
    }
    grab = __shfl_sync(0xffffffffu, ahead, 0);
    if (lane == 0 && (int64_t)grab < nitems) ahead = atomicAdd(next_item, (unsigned long long)kGrab);
  }
}

// Calibration of every tile matrix of a single-vector batch (as below).
template <typename V>
__global__ void batch_calibrate1_kernel(const int64_t* __restrict__ cal_off, const int32_t* __restrict__ cal_mat,
                                        int ncal, int64_t total, const BatchMat* __restrict__ mats, V alpha, V beta,
                                        bool bz) {
  const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (g >= total) return;
  int lo = 0, hi = ncal;  // last i with cal_off[i] <= g
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (cal_off[mid] <= g) lo = mid; else hi = mid;
  }
  const BatchMat& M = mats[cal_mat[lo]];
  spmv_calibrate1<V>(g - cal_off[lo], M.tiles, static_cast<const V*>(M.tcin), static_cast<const V*>(M.tosum),
                     M.topen, M.tempty, M.tnempty, static_cast<V*>(M.y), alpha, beta, bz);
}

// Calibration of every tile matrix: thread g takes entry g - cal_off[i] of
// tile matrix i (its tiles, then its empty rows).
template <typename V, int KC>
__global__ void batch_calibrate_kernel(const int64_t* __restrict__ cal_off, const int32_t* __restrict__ cal_mat,
                                       int ncal, int64_t total, const BatchMat* __restrict__ mats, V alpha, V beta,
                                       bool bz) {
  const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (g >= total) return;
  int lo = 0, hi = ncal;  // last i with cal_off[i] <= g
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (cal_off[mid] <= g) lo = mid; else hi = mid;
  }
  const BatchMat& M = mats[cal_mat[lo]];
  spmm_calibrate<V, KC>(g - cal_off[lo], M.tiles, static_cast<const V*>(M.tcin), static_cast<const V*>(M.tosum),
                        M.topen, M.tempty, M.tnempty, static_cast<V*>(M.y), M.ldy, alpha, beta, bz);
}

// Single-matrix SpMM over the CSR plan (the per-matrix path of spops_spmm).
template <typename I, typename V, int KT>
__global__ void __launch_bounds__(256, 3) spmm_kernel(const CsrSeg* __restrict__ segs, int64_t nseg,
                                                      const I* __restrict__ ci, const V* __restrict__ val,
                                                      const I* __restrict__ rp, const V* __restrict__ X, int64_t ldx,
                                                      V* __restrict__ Y, int64_t ldy, int64_t k, V alpha, V beta,
                                                      bool bz, V* __restrict__ partial, int* __restrict__ counter) {
  extern __shared__ __align__(16) unsigned char spmm_dyn_smem[];  // one SpmmStage per warp
  SpmmStage<I, V>& stage = reinterpret_cast<SpmmStage<I, V>*>(spmm_dyn_smem)[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t j = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; j < nseg; j += nwarps)
    csr_segment_spmm<I, V, KT>(segs[j], j, ci, val, rp, X, ldx, Y, ldy, k, alpha, beta, bz, partial, counter, stage,
                               lane);
}

// dynamic shared memory of the SpMM kernels: one stage per warp
template <typename I, typename V>
constexpr size_t spmm_smem(int threads) {
  return (size_t)(threads / 32) * sizeof(SpmmStage<I, V>);
}

template <typename K>
int occupancy(K kernel, int threads, size_t smem = 0) {
  int bps = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kernel, threads, smem) != cudaSuccess || bps < 1) return 1;
  return bps;
}

// Resident blocks per SM of a kernel with `smem` bytes of dynamic shared
// memory, the attribute set once per instantiation and device; 0 when it
// cannot be set.
constexpr int kMaxDevices = 64;

template <typename K>
int blocks_per_sm(K kern, int threads, size_t smem, int* cache) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) dev = 0;
  if (cache[dev] == 0) {
    if (smem && cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return 0;
    cache[dev] = occupancy(kern, threads, smem);
  }
  return cache[dev];
}

template <typename I, typename V, int KT>
int spmm_blocks_per_sm() {
  static int cache[kMaxDevices];
  return blocks_per_sm(spmm_kernel<I, V, KT>, 256, spmm_smem<I, V>(256), cache);
}

template <typename I, typename V, int KT, bool kBand = false>
int batch_blocks_per_sm() {
  static int cache[kMaxDevices];
  return blocks_per_sm(batch_kernel<I, V, KT, kBand>, kBatchBlock, KT == 1 ? 0 : spmm_smem<I, V>(kBatchBlock), cache);
}

}  // namespace

// ------------------------------------------------------------- SpMM (single)
template <typename I, typename V>
static spops_status_t spmm_t(Context* ctx, Matrix* A, double alpha, const void* X, int64_t ldx, int64_t k,
                             double beta, void* Y, int64_t ldy) {
  CsrPlan& P = A->plan;
  if (P.nblocks == 0 || k == 0) return SPOPS_OK;
  if (P.nlong > 0 && A->spmm_partial.bytes < (size_t)P.nblocks * k * sizeof(V))
    SPOPS_TRY(A->spmm_partial.alloc((size_t)P.nblocks * k * sizeof(V)));
  const int kt = k >= 32 ? 32 : (k >= 8 ? 8 : 8);
  const bool bz = beta == 0.0;
  auto launch = [&](auto kern, int bps) -> spops_status_t {
    const size_t smem = spmm_smem<I, V>(256);
    if (bps < 1) return fail(SPOPS_ERR_CUDA, "spmm: kernel attributes could not be set");
    int64_t grid = (int64_t)ctx->num_sms * bps;
    const int64_t need = (P.nblocks + 7) / 8;
    if (grid > need) grid = need;
    kern<<<(unsigned)grid, 256, smem, ctx->stream>>>(P.seg.as<CsrSeg>(), P.nblocks, A->col.as<I>(), A->val.as<V>(),
                                                  A->row.as<I>(), static_cast<const V*>(X), ldx, static_cast<V*>(Y),
                                                  ldy, k, (V)alpha, (V)beta, bz, A->spmm_partial.as<V>(),
                                                  P.counter.as<int>());
    SPOPS_LAUNCH_CHECK();
    return SPOPS_OK;
  };
  if (kt == 32) return launch(spmm_kernel<I, V, 32>, spmm_blocks_per_sm<I, V, 32>());
  return launch(spmm_kernel<I, V, 8>, spmm_blocks_per_sm<I, V, 8>());
}

spops_status_t csr_spmm(Context* ctx, Matrix* A, double alpha, const void* X, int64_t ldx, int64_t k, double beta,
                        void* Y, int64_t ldy) {
  if (A->format != SPOPS_FMT_CSR) return fail(SPOPS_ERR_UNSUPPORTED, "SpMM needs a CSR matrix");
  if (!A->plan.ready) SPOPS_TRY(csr_analyse(ctx, A));
  // k = 8, 16, 32 with X rows at most 2k wide: register tiles on the SpMV's
  // plan.  (Passes of 8 columns over wider rows measured slower than the
  // segment kernel: four passes at k = 32 took 20.5 ms against 6.5 ms on the
  // power-law matrix.)
  if (ctx->csr_variant == 0) {
    bool used = false;
    SPOPS_TRY(csr_tile_spmm(ctx, A, alpha, X, ldx, k, beta, Y, ldy, &used));
    if (used) return SPOPS_OK;
  }
  const bool i32 = A->itype == SPOPS_INDEX_I32, f64 = A->vtype == SPOPS_VALUE_F64;
  if (i32 && f64) return spmm_t<int32_t, double>(ctx, A, alpha, X, ldx, k, beta, Y, ldy);
  if (i32) return spmm_t<int32_t, float>(ctx, A, alpha, X, ldx, k, beta, Y, ldy);
  if (f64) return spmm_t<int64_t, double>(ctx, A, alpha, X, ldx, k, beta, Y, ldy);
  return spmm_t<int64_t, float>(ctx, A, alpha, X, ldx, k, beta, Y, ldy);
}

// ------------------------------------------------------------------ batch
struct Batch {
  Context* ctx = nullptr;
  int64_t count = 0, k = 1;
  spops_index_t itype = SPOPS_INDEX_I32;
  spops_value_t vtype = SPOPS_VALUE_F64;
  std::vector<Matrix*> src;
  std::vector<Matrix*> form;  // padded form chosen by the tuner (owned), or null for CSR
  std::vector<int> choice;    // 0 CSR, 1.. padded candidate index
  std::vector<BatchMat> host;
  std::vector<DevBuf> spmm_partial;
  // k = 8: matrices on register tiles, their carry buffers, items and the
  // calibration index (offsets into all tile matrices' tiles + empty rows)
  std::vector<char> tile_ok;
  std::vector<DevBuf> t_cin, t_osum;
  DevBuf titems, tqueue, cal_off, cal_mat;
  int64_t ntitems = 0, ncal_total = 0;
  int ncal = 0;
  DevBuf items, table;
  DevBuf queue;  // next item of the running launch
  int64_t nitems = 0;
  int kt = 8;  // RHS tile for k > 1
  bool dirty = true;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  double cap_alpha = 0, cap_beta = 0;
  ~Batch() {
    for (Matrix* m : form)
      if (m) {
        m->release_all();
        delete static_cast<spops_matrix_s*>(m);
      }
    for (auto& b : spmm_partial) b.release();
    for (auto& b : t_cin) b.release();
    for (auto& b : t_osum) b.release();
    titems.release();
    tqueue.release();
    cal_off.release();
    cal_mat.release();
    items.release();
    table.release();
    queue.release();
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (ev_in) cudaEventDestroy(ev_in);
    if (ev_out) cudaEventDestroy(ev_out);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

// the padded candidates the tuner tries: (sigma, layout)
const int64_t kCandSigma[4] = {256, 4096, 256, 4096};
const spops_layout_t kCandLayout[4] = {SPOPS_ROW_MAJOR, SPOPS_ROW_MAJOR, SPOPS_COL_MAJOR, SPOPS_COL_MAJOR};

spops_status_t build_items(Batch* B) {
  std::vector<BatchItem> it, tit;
  std::vector<int64_t> off;
  std::vector<int32_t> mat;
  int64_t total = 0;
  for (int64_t m = 0; m < B->count; ++m) {
    Matrix* A = B->src[m];
    Matrix* F = B->form[m];
    if (B->tile_ok[m]) {
      const CsrTiles& D = A->plan.tiles;
      for (int64_t t = 0; t < D.tiles; t += kTilesPerItem) tit.push_back(BatchItem{(int32_t)m, 3, t});
      off.push_back(total);
      mat.push_back((int32_t)m);
      total += D.tiles + D.nempty;
    } else if (!F || B->k > 1) {
      for (int64_t s = 0; s < A->plan.nblocks; ++s) it.push_back(BatchItem{(int32_t)m, 0, s});
    } else {
      const int64_t groups = (F->rows + 31) / 32;
      for (int64_t g = 0; g < groups; ++g) it.push_back(BatchItem{(int32_t)m, 1, g});
      for (int64_t q = 0; q < F->pad.npieces; ++q) it.push_back(BatchItem{(int32_t)m, 2, q});
    }
  }
  B->nitems = (int64_t)it.size();
  if (!B->queue.p) SPOPS_TRY(B->queue.alloc(8));
  SPOPS_TRY(B->items.alloc(std::max<size_t>(it.size(), 1) * sizeof(BatchItem)));
  if (!it.empty())
    SPOPS_CUDA(cudaMemcpy(B->items.p, it.data(), it.size() * sizeof(BatchItem), cudaMemcpyHostToDevice));
  B->ntitems = (int64_t)tit.size();
  B->ncal = (int)off.size();
  B->ncal_total = total;
  if (!tit.empty()) {
    if (!B->tqueue.p) SPOPS_TRY(B->tqueue.alloc(8));
    SPOPS_TRY(B->titems.alloc(tit.size() * sizeof(BatchItem)));
    SPOPS_TRY(B->cal_off.alloc(off.size() * 8));
    SPOPS_TRY(B->cal_mat.alloc(mat.size() * 4));
    SPOPS_CUDA(cudaMemcpy(B->titems.p, tit.data(), tit.size() * sizeof(BatchItem), cudaMemcpyHostToDevice));
    SPOPS_CUDA(cudaMemcpy(B->cal_off.p, off.data(), off.size() * 8, cudaMemcpyHostToDevice));
    SPOPS_CUDA(cudaMemcpy(B->cal_mat.p, mat.data(), mat.size() * 4, cudaMemcpyHostToDevice));
  }
  return SPOPS_OK;
}

spops_status_t build_table(Batch* B) {
  for (int64_t m = 0; m < B->count; ++m) {
    Matrix* A = B->src[m];
    Matrix* F = B->form[m];
    BatchMat& t = B->host[m];
    t.rp = A->row.p;
    t.ci = A->col.p;
    t.val = A->val.p;
    t.seg = A->plan.seg.as<CsrSeg>();
    t.partial = B->k > 1 ? B->spmm_partial[m].p : A->plan.partial.p;
    t.counter = A->plan.counter.as<int>();
    t.rows = A->rows;
    t.cols = A->cols;
    t.band = B->k == 1 && B->ctx->batch_band && A->plan.band > 0 ? A->plan.band : 0;
    if (B->tile_ok[m]) {
      const CsrTiles& D = A->plan.tiles;
      t.tile_row = D.tile_row.as<int64_t>();
      t.tflags = D.flags.as<uint8_t>();
      t.tiles = D.tiles;
      t.nnz = A->nnz;
      t.tcin = B->t_cin[m].p;
      t.tosum = B->t_osum[m].p;
      t.topen = D.open_row.as<int64_t>();
      t.tempty = D.empty.as<int64_t>();
      t.tnempty = D.nempty;
    }
    if (F) {
      t.pcol = F->col.p;
      t.pval = F->val.p;
      t.chunk_len = F->pad.chunk_len.p;
      t.chunk_off = F->pad.chunk_off.as<int64_t>();
      t.row_len = F->pad.row_len.as<int>();
      t.reorder = F->pad.sorted ? F->pad.reorder.p : nullptr;
      t.pieces = F->pad.piece.as<PadPiece>();
      t.ppartial = F->pad.partial.p;
      t.pcounter = F->pad.counter.as<int>();
      t.C = F->pad.C;
      t.colmajor = F->layout == SPOPS_COL_MAJOR;
    }
  }
  SPOPS_TRY(B->table.alloc(std::max<size_t>(B->host.size(), 1) * sizeof(BatchMat)));
  SPOPS_CUDA(cudaMemcpy(B->table.p, B->host.data(), B->host.size() * sizeof(BatchMat), cudaMemcpyHostToDevice));
  return SPOPS_OK;
}

template <typename I, typename V>
int tile1_blocks_per_sm() {
  static int cache[kMaxDevices];
  return blocks_per_sm(batch_tile1_kernel<I, V>, kBatchBlock, 0, cache);
}

template <typename I, typename V>
spops_status_t launch_tiles1(Batch* B, double alpha, double beta, cudaStream_t st) {
  const bool bz = beta == 0.0;
  const int bps = tile1_blocks_per_sm<I, V>();
  if (bps < 1) return fail(SPOPS_ERR_CUDA, "batch: kernel attributes could not be set");
  int64_t grid = (int64_t)B->ctx->num_sms * bps;
  const int64_t need = (B->ntitems + 7) / 8;
  if (grid > need) grid = need;
  SPOPS_CUDA(cudaMemsetAsync(B->tqueue.p, 0, 8, st));
  batch_tile1_kernel<I, V><<<(unsigned)grid, kBatchBlock, 0, st>>>(B->titems.as<BatchItem>(), B->ntitems,
                                                                  B->table.as<BatchMat>(), (V)alpha, (V)beta, bz,
                                                                  B->tqueue.as<unsigned long long>());
  SPOPS_LAUNCH_CHECK();
  if (B->ncal_total > 0) {
    batch_calibrate1_kernel<V><<<(unsigned)((B->ncal_total + 255) / 256), 256, 0, st>>>(
        B->cal_off.as<int64_t>(), B->cal_mat.as<int32_t>(), B->ncal, B->ncal_total, B->table.as<BatchMat>(),
        (V)alpha, (V)beta, bz);
    SPOPS_LAUNCH_CHECK();
  }
  return SPOPS_OK;
}

template <typename I, typename V, int G>
int tile_blocks_per_sm() {
  static int cache[kMaxDevices];
  return blocks_per_sm(batch_tile_kernel<I, V, G>, kBatchBlock, 0, cache);
}

template <typename I, typename V, int G>
spops_status_t launch_tiles(Batch* B, double alpha, double beta, cudaStream_t st) {
  const bool bz = beta == 0.0;
  const int bps = tile_blocks_per_sm<I, V, G>();
  if (bps < 1) return fail(SPOPS_ERR_CUDA, "batch: kernel attributes could not be set");
  int64_t grid = (int64_t)B->ctx->num_sms * bps;
  const int64_t need = (B->ntitems + 7) / 8;
  if (grid > need) grid = need;
  SPOPS_CUDA(cudaMemsetAsync(B->tqueue.p, 0, 8, st));
  batch_tile_kernel<I, V, G><<<(unsigned)grid, kBatchBlock, 0, st>>>(B->titems.as<BatchItem>(), B->ntitems,
                                                                    B->table.as<BatchMat>(), (V)alpha, (V)beta, bz,
                                                                    B->tqueue.as<unsigned long long>());
  SPOPS_LAUNCH_CHECK();
  if (B->ncal_total > 0) {
    batch_calibrate_kernel<V, 4 * G><<<(unsigned)((B->ncal_total + 255) / 256), 256, 0, st>>>(
        B->cal_off.as<int64_t>(), B->cal_mat.as<int32_t>(), B->ncal, B->ncal_total, B->table.as<BatchMat>(),
        (V)alpha, (V)beta, bz);
    SPOPS_LAUNCH_CHECK();
  }
  return SPOPS_OK;
}

template <typename I, typename V>
spops_status_t launch_batch(Batch* B, double alpha, double beta, cudaStream_t st) {
  const bool bz = beta == 0.0;
  if (B->ntitems > 0) {  // tile items, then their calibration
    if (B->k == 1) SPOPS_TRY((launch_tiles1<I, V>(B, alpha, beta, st)));
    else if (B->k == 8) SPOPS_TRY((launch_tiles<I, V, 2>(B, alpha, beta, st)));
    else if (B->k == 16) SPOPS_TRY((launch_tiles<I, V, 4>(B, alpha, beta, st)));
    else SPOPS_TRY((launch_tiles<I, V, 8>(B, alpha, beta, st)));
  }
  if (B->nitems == 0) return SPOPS_OK;
  auto go = [&](auto kern, size_t smem, int bps) -> spops_status_t {
    if (bps < 1) return fail(SPOPS_ERR_CUDA, "batch: kernel attributes could not be set");
    int64_t grid = (int64_t)B->ctx->num_sms * bps;
    const int64_t need = (B->nitems + 7) / 8;
    if (grid > need) grid = need;
    SPOPS_CUDA(cudaMemsetAsync(B->queue.p, 0, 8, st));
    kern<<<(unsigned)grid, kBatchBlock, smem, st>>>(B->items.as<BatchItem>(), B->nitems, B->table.as<BatchMat>(), B->k,
                                                 (V)alpha, (V)beta, bz, B->queue.as<unsigned long long>());
    SPOPS_LAUNCH_CHECK();
    return SPOPS_OK;
  };
  if (B->k == 1 && B->ctx->batch_band)
    return go(batch_kernel<I, V, 1, true>, 0, batch_blocks_per_sm<I, V, 1, true>());
  if (B->k == 1) return go(batch_kernel<I, V, 1>, 0, batch_blocks_per_sm<I, V, 1>());
  if (B->kt == 32)
    return go(batch_kernel<I, V, 32>, spmm_smem<I, V>(kBatchBlock), batch_blocks_per_sm<I, V, 32>());
  return go(batch_kernel<I, V, 8>, spmm_smem<I, V>(kBatchBlock), batch_blocks_per_sm<I, V, 8>());
}

spops_status_t launch_any(Batch* B, double alpha, double beta, cudaStream_t st) {
  const bool i32 = B->itype == SPOPS_INDEX_I32, f64 = B->vtype == SPOPS_VALUE_F64;
  if (i32 && f64) return launch_batch<int32_t, double>(B, alpha, beta, st);
  if (i32) return launch_batch<int32_t, float>(B, alpha, beta, st);
  if (f64) return launch_batch<int64_t, double>(B, alpha, beta, st);
  return launch_batch<int64_t, float>(B, alpha, beta, st);
}

// Entries within 16, 32 and 64 (kBandMax) of the diagonal (warp per row).
template <typename I>
__global__ void band_count_kernel(const I* __restrict__ rp, const I* __restrict__ ci, int64_t n,
                                  unsigned long long* __restrict__ cnt) {
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  unsigned long long c[3] = {0, 0, 0};
  if (r < n)
    for (int64_t k = (int64_t)rp[r] + lane; k < (int64_t)rp[r + 1]; k += 32) {
      const int64_t d = (int64_t)ci[k] - r;
      const int64_t a = d < 0 ? -d : d;
#pragma unroll
      for (int b = 0; b < 3; ++b) c[b] += a <= (16 << b) ? 1 : 0;
    }
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    for (int o = 16; o; o >>= 1) c[b] += __shfl_xor_sync(0xffffffffu, c[b], o);
    if (lane == 0 && c[b]) atomicAdd(cnt + b, c[b]);
  }
}

// Half-width of the x window the batch's CSR segments stage: the smallest of
// 16 .. kBandMax that holds 90 % of the entries the widest one holds, when
// that is at least a tenth of all entries; otherwise 0 (no staging).
spops_status_t csr_band(Context* ctx, Matrix* A) {
  if (A->plan.band >= 0) return SPOPS_OK;
  A->plan.band = 0;
  if (A->nnz == 0 || A->rows == 0) return SPOPS_OK;
  cudaStream_t st = ctx->stream;
  PoolBuf cnt(ctx);
  SPOPS_TRY(cnt.alloc(32));
  SPOPS_CUDA(cudaMemsetAsync(cnt.p, 0, 32, st));
  const unsigned grid = (unsigned)((A->rows * 32 + 255) / 256);
  if (A->itype == SPOPS_INDEX_I32)
    band_count_kernel<int32_t><<<grid, 256, 0, st>>>(A->row.as<int32_t>(), A->col.as<int32_t>(), A->rows,
                                                     cnt.as<unsigned long long>());
  else
    band_count_kernel<int64_t><<<grid, 256, 0, st>>>(A->row.as<int64_t>(), A->col.as<int64_t>(), A->rows,
                                                     cnt.as<unsigned long long>());
  SPOPS_LAUNCH_CHECK();
  unsigned long long h[3];
  SPOPS_CUDA(cudaMemcpyAsync(h, cnt.p, 24, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  if ((double)h[2] < 0.1 * (double)A->nnz) return SPOPS_OK;
  for (int b = 0; b < 3; ++b)
    if ((double)h[b] >= 0.9 * (double)h[2]) {
      A->plan.band = 16 << b;
      break;
    }
  return SPOPS_OK;
}

spops_status_t prepare(Batch* B) {
  if (!B->dirty) return SPOPS_OK;
  B->tile_ok.assign((size_t)B->count, 0);
  B->t_cin.resize((size_t)B->count);
  B->t_osum.resize((size_t)B->count);
  for (int64_t m = 0; m < B->count; ++m) {
    Matrix* A = B->src[m];
    if (!A->plan.ready) SPOPS_TRY(csr_analyse(B->ctx, A));
    if (B->k == 1 && B->ctx->batch_band) SPOPS_TRY(csr_band(B->ctx, A));
    // k = 8, 16, 32 over X rows at most 2k wide, vector loads aligned: register tiles
    const BatchMat& h = B->host[m];
    const size_t vs = A->vsize();
    if (B->k == 1 && !B->form[m] && csr_tile_usable(A, 0)) {  // CSR with one vector: SpMV tile items
      if (!A->plan.tiles.ready || A->plan.tiles.k != 8) SPOPS_TRY(csr_tile_analyse(B->ctx, A, 8));
      const size_t bytes = (size_t)A->plan.tiles.tiles * vs;
      if (B->t_cin[m].bytes < bytes) SPOPS_TRY(B->t_cin[m].alloc(bytes));
      if (B->t_osum[m].bytes < bytes) SPOPS_TRY(B->t_osum[m].alloc(bytes));
      B->tile_ok[m] = 1;
    } else if (csr_tile_spmm_usable(A, h.x, h.ldx, B->k) && h.ldy >= B->k) {
      if (!A->plan.tiles.ready || A->plan.tiles.k != 8) SPOPS_TRY(csr_tile_analyse(B->ctx, A, 8));
      const size_t bytes = (size_t)A->plan.tiles.tiles * (size_t)B->k * vs;
      if (B->t_cin[m].bytes < bytes) SPOPS_TRY(B->t_cin[m].alloc(bytes));
      if (B->t_osum[m].bytes < bytes) SPOPS_TRY(B->t_osum[m].alloc(bytes));
      B->tile_ok[m] = 1;
    }
    if (B->k > 1 && A->plan.nlong > 0) {
      const size_t bytes = (size_t)A->plan.nblocks * B->k * A->vsize();
      if (B->spmm_partial[m].bytes < bytes) SPOPS_TRY(B->spmm_partial[m].alloc(bytes));
    }
  }
  SPOPS_TRY(build_items(B));
  SPOPS_TRY(build_table(B));
  if (B->exec) {
    cudaGraphExecDestroy(B->exec);
    B->exec = nullptr;
  }
  if (B->graph) {
    cudaGraphDestroy(B->graph);
    B->graph = nullptr;
  }
  B->dirty = false;
  return SPOPS_OK;
}

// time fn() on stream st: min over reps of CUDA-event durations (ms)
template <typename F>
spops_status_t time_ms(cudaStream_t st, F fn, int reps, float* out) {
  cudaEvent_t a, b;
  SPOPS_CUDA(cudaEventCreate(&a));
  SPOPS_CUDA(cudaEventCreate(&b));
  float best = 1e30f;
  spops_status_t s = fn();  // warm-up
  for (int r = 0; r < reps && s == SPOPS_OK; ++r) {
    cudaEventRecord(a, st);
    s = fn();
    cudaEventRecord(b, st);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    best = std::min(best, ms);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *out = best;
  return s;
}

}  // namespace

spops_status_t batch_tune(Batch* B, int flags) {
  Context* ctx = B->ctx;
  cudaStream_t st = ctx->stream;
  const bool try_padded = !(flags & 1);
  for (int64_t m = 0; m < B->count; ++m) {
    Matrix* A = B->src[m];
    if (!A->plan.ready) SPOPS_TRY(csr_analyse(ctx, A));
    if (B->form[m]) {
      B->form[m]->release_all();
      delete static_cast<spops_matrix_s*>(B->form[m]);
      B->form[m] = nullptr;
    }
    B->choice[m] = 0;
    if (B->k > 1 || !try_padded) continue;
    const BatchMat& t = B->host[m];
    if (!t.x || !t.y) return fail(SPOPS_ERR_INVALID, "spops_batch_tune: vectors not set");
    float best = 0;
    SPOPS_TRY(time_ms(st, [&] { return csr_spmv(ctx, A, 1.0, t.x, 0.0, t.y); }, 3, &best));
    for (int c = 0; c < 4; ++c) {
      spops_format_params_t p;
      std::memset(&p, 0, sizeof(p));
      p.sigma = kCandSigma[c];
      p.chunk = 32;
      p.alignment = 1;
      p.layout = kCandLayout[c];
      Matrix* F = nullptr;
      spops_status_t s = convert_from_csr(ctx, A, SPOPS_FMT_SELL_C_SIGMA, p, &F);
      if (s == SPOPS_ERR_TOO_LARGE) continue;
      SPOPS_TRY(s);
      float ms = 0;
      s = time_ms(st, [&] { return padded_spmv(ctx, F, 1.0, t.x, 0.0, t.y); }, 3, &ms);
      if (s != SPOPS_OK || ms >= 0.97f * best) {  // keep CSR unless clearly faster
        F->release_all();
        delete static_cast<spops_matrix_s*>(F);
        SPOPS_TRY(s);
        continue;
      }
      if (B->form[m]) {
        B->form[m]->release_all();
        delete static_cast<spops_matrix_s*>(B->form[m]);
      }
      B->form[m] = F;
      B->choice[m] = 1 + c;
      best = ms;
    }
  }
  if (B->k == 1 && try_padded) {
    // Each matrix timed alone says little about how the forms run together
    // in one launch (a small matrix's time is mostly launch latency): keep
    // the per-matrix choices only if the whole batch runs faster with them
    // than with every matrix in CSR.
    float t_mixed = 0, t_csr = 0;
    B->dirty = true;
    SPOPS_TRY(prepare(B));
    SPOPS_TRY(time_ms(st, [&] { return launch_any(B, 1.0, 0.0, st); }, 3, &t_mixed));
    std::vector<Matrix*> kept = B->form;
    const std::vector<int> kept_choice = B->choice;
    for (int64_t m = 0; m < B->count; ++m) {
      B->form[m] = nullptr;
      B->choice[m] = 0;
    }
    B->dirty = true;
    spops_status_t s = prepare(B);
    if (s == SPOPS_OK) s = time_ms(st, [&] { return launch_any(B, 1.0, 0.0, st); }, 3, &t_csr);
    if (s != SPOPS_OK || t_csr > t_mixed) {  // the per-matrix forms win (or CSR could not be timed)
      B->form = kept;
      B->choice = kept_choice;
    } else {
      for (Matrix* F : kept)
        if (F) {
          F->release_all();
          delete static_cast<spops_matrix_s*>(F);
        }
    }
    SPOPS_TRY(s);
  }
  if (B->k > 1) {  // RHS tile: time both on the whole batch
    float t8 = 0, t32 = 0;
    B->kt = 8;
    B->dirty = true;
    SPOPS_TRY(prepare(B));
    SPOPS_TRY(time_ms(st, [&] { return launch_any(B, 1.0, 0.0, st); }, 3, &t8));
    if (B->k >= 32) {
      B->kt = 32;
      SPOPS_TRY(time_ms(st, [&] { return launch_any(B, 1.0, 0.0, st); }, 3, &t32));
      B->kt = t32 < t8 ? 32 : 8;
    }
  }
  B->dirty = true;
  return prepare(B);
}

spops_status_t batch_run(Batch* B, double alpha, double beta) {
  Context* ctx = B->ctx;
  SPOPS_TRY(prepare(B));
  // order the batch's stream after the caller's, and the caller's after it
  SPOPS_CUDA(cudaEventRecord(B->ev_in, ctx->stream));
  SPOPS_CUDA(cudaStreamWaitEvent(B->stream, B->ev_in, 0));
  if (B->exec && alpha == B->cap_alpha && beta == B->cap_beta) {
    SPOPS_CUDA(cudaGraphLaunch(B->exec, B->stream));
  } else {
    SPOPS_TRY(launch_any(B, alpha, beta, B->stream));
  }
  SPOPS_CUDA(cudaEventRecord(B->ev_out, B->stream));
  SPOPS_CUDA(cudaStreamWaitEvent(ctx->stream, B->ev_out, 0));
  return SPOPS_OK;
}

spops_status_t batch_capture(Batch* B, double alpha, double beta) {
  SPOPS_TRY(prepare(B));
  if (B->exec) {
    cudaGraphExecDestroy(B->exec);
    B->exec = nullptr;
  }
  if (B->graph) {
    cudaGraphDestroy(B->graph);
    B->graph = nullptr;
  }
  // warm the occupancy queries outside the capture
  SPOPS_TRY(launch_any(B, alpha, beta, B->stream));
  SPOPS_CUDA(cudaStreamSynchronize(B->stream));
  SPOPS_CUDA(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
  spops_status_t s = launch_any(B, alpha, beta, B->stream);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(B->stream, &g);
  if (s != SPOPS_OK) {
    if (g) cudaGraphDestroy(g);
    return s;
  }
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture", __FILE__, __LINE__);
  B->graph = g;
  SPOPS_CUDA(cudaGraphInstantiate(&B->exec, B->graph, 0));
  B->cap_alpha = alpha;
  B->cap_beta = beta;
  return SPOPS_OK;
}

}  // namespace spops

using namespace spops;

struct spops_batch_s : spops::Batch {};

extern "C" {

spops_status_t spops_spmm(spops_context_t ctx, double alpha, spops_matrix_t A, const void* X, int64_t ldx, int64_t k,
                          double beta, void* Y, int64_t ldy) {
  if (!ctx || !A) return fail(SPOPS_ERR_INVALID, "spops_spmm: null context/matrix");
  if (k < 0 || ldx < k || ldy < k) return fail(SPOPS_ERR_INVALID, "spops_spmm: k / leading dimensions");
  DeviceGuard g(ctx->device);
  return csr_spmm(ctx, A, alpha, X, ldx, k, beta, Y, ldy);
}

spops_status_t spops_batch_create(spops_context_t ctx, spops_batch_t* out, int64_t count, const spops_matrix_t* mats,
                                  int64_t k) {
  if (!ctx || !out || (count > 0 && !mats)) return fail(SPOPS_ERR_INVALID, "spops_batch_create: null argument");
  if (count < 0 || count > INT32_MAX || k < 1) return fail(SPOPS_ERR_INVALID, "spops_batch_create: count/k");
  for (int64_t m = 0; m < count; ++m) {
    if (!mats[m] || mats[m]->format != SPOPS_FMT_CSR)
      return fail(SPOPS_ERR_INVALID, "spops_batch_create: matrix %lld is not a CSR handle", (long long)m);
    if (mats[m]->itype != mats[0]->itype || mats[m]->vtype != mats[0]->vtype)
      return fail(SPOPS_ERR_INVALID, "spops_batch_create: mixed index/value types");
  }
  DeviceGuard g(ctx->device);
  spops_batch_s* B = new spops_batch_s();
  B->ctx = ctx;
  B->count = count;
  B->k = k;
  if (count > 0) {
    B->itype = mats[0]->itype;
    B->vtype = mats[0]->vtype;
  }
  B->src.assign(mats, mats + count);
  B->form.assign((size_t)count, nullptr);
  B->choice.assign((size_t)count, 0);
  B->host.assign((size_t)count, BatchMat{});
  B->spmm_partial.resize((size_t)count);
  cudaError_t e = cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&B->ev_in, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&B->ev_out, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    delete B;
    return cuda_fail(e, "batch stream/events", __FILE__, __LINE__);
  }
  *out = B;
  return SPOPS_OK;
}

spops_status_t spops_batch_destroy(spops_batch_t B) {
  if (!B) return SPOPS_OK;
  DeviceGuard g(B->ctx->device);
  cudaStreamSynchronize(B->stream);
  delete B;
  return SPOPS_OK;
}

spops_status_t spops_batch_set_vectors(spops_batch_t B, const void* const* X, const int64_t* ldx, void* const* Y,
                                       const int64_t* ldy) {
  if (!B || (B->count > 0 && (!X || !Y))) return fail(SPOPS_ERR_INVALID, "spops_batch_set_vectors: null argument");
  for (int64_t m = 0; m < B->count; ++m) {
    const int64_t lx = ldx ? ldx[m] : B->k, ly = ldy ? ldy[m] : B->k;
    if (lx < B->k || ly < B->k) return fail(SPOPS_ERR_INVALID, "spops_batch_set_vectors: leading dimension < k");
    B->host[m].x = X[m];
    B->host[m].y = Y[m];
    B->host[m].ldx = lx;
    B->host[m].ldy = ly;
  }
  B->dirty = true;
  return SPOPS_OK;
}

spops_status_t spops_batch_tune(spops_context_t ctx, spops_batch_t B, int32_t flags) {
  if (!ctx || !B) return fail(SPOPS_ERR_INVALID, "spops_batch_tune: null argument");
  DeviceGuard g(ctx->device);
  B->ctx = ctx;
  return batch_tune(B, flags);
}

spops_status_t spops_batch_run(spops_context_t ctx, spops_batch_t B, double alpha, double beta) {
  if (!ctx || !B) return fail(SPOPS_ERR_INVALID, "spops_batch_run: null argument");
  DeviceGuard g(ctx->device);
  B->ctx = ctx;
  return batch_run(B, alpha, beta);
}

spops_status_t spops_batch_capture(spops_context_t ctx, spops_batch_t B, double alpha, double beta) {
  if (!ctx || !B) return fail(SPOPS_ERR_INVALID, "spops_batch_capture: null argument");
  DeviceGuard g(ctx->device);
  B->ctx = ctx;
  return batch_capture(B, alpha, beta);
}

spops_status_t spops_batch_info(spops_batch_t B, int64_t* items, int32_t* choice, int32_t* rhs_tile) {
  if (!B) return fail(SPOPS_ERR_INVALID, "spops_batch_info: null batch");
  if (items) *items = B->nitems + B->ntitems;
  if (choice)
    for (int64_t m = 0; m < B->count; ++m) choice[m] = B->choice[m];
  if (rhs_tile) *rhs_tile = B->k > 1 ? B->kt : 1;
  return SPOPS_OK;
}

}  // extern "C"
