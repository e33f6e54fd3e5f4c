// Internal C++ view of the library state behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <chrono>
#include <cstdlib>

#include <cstdint>
#include <cstdio>
#include <string>
#include <functional>
#include <utility>
#include <vector>

#include "../../include/sparseops_b200.h"

namespace spops {

// ----------------------------------------------------------------- errors
void set_error(const char* fmt, ...);
spops_status_t fail(spops_status_t s, const char* fmt, ...);
spops_status_t cuda_fail(cudaError_t e, const char* what, const char* file, int line);

#define SPOPS_CUDA(call)                                                     \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess) return ::spops::cuda_fail(e_, #call, __FILE__, __LINE__); \
  } while (0)

#define SPOPS_TRY(call)                        \
  do {                                         \
    spops_status_t s_ = (call);                \
    if (s_ != SPOPS_OK) return s_;             \
  } while (0)

// Kernel launch check: launch-configuration errors only (no synchronisation).
#define SPOPS_LAUNCH_CHECK() SPOPS_CUDA(cudaGetLastError())

// ---------------------------------------------------------------- buffers
// Device allocation owned by a handle (or borrowed when own == false).
struct Context;
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  bool own = false;
  Context* home = nullptr;  // set by alloc_cached: released into home's block cache
  spops_status_t alloc(size_t n);
  // n bytes, reusing a block of about that size that an earlier result of
  // this context released (large results only; see Context::block_cache)
  spops_status_t alloc_cached(Context* ctx, size_t n);
  void release();
  void borrow(const void* q, size_t n) { release(); p = const_cast<void*>(q); bytes = n; own = false; }
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

// ---------------------------------------------------------------- context
struct Context {
  int device = 0;
  cudaStream_t stream = nullptr;
  int num_sms = 148;
  // grow-only scratch for temporary device storage (CUB temp, staging)
  DevBuf scratch;
  spops_status_t scratch_reserve(size_t bytes);
  // device error word: bounded waits that ran out set bits here
  DevBuf errword;
  spops_status_t ensure_errword();
  // CSR SpMV kernel variant (spmv_csr.cu)
  int csr_variant = 0;
  // batched k = 1: stage each CSR segment's banded x window in shared memory
  // (measured slower on the 256-matrix batch than plain gathers, so off unless set)
  int batch_band = 0;
  // A^T x through the transpose's permutation: source-row bands (0: as many
  // as put each band's values within 64 MB, when A's values exceed 96 MB;
  // 1: one pass; 2..8: that many bands)
  int adjoint_bands = 0;
  // SELL (C = 32, column-major): a chunk's slots beyond its fourth-longest
  // row are read from row-contiguous tails (1) or in place (0, the default:
  // measured faster on the power-law matrix); read when the matrix is
  // converted or uploaded
  int sell_tails = 0;
  // SELL (C = 32, column-major): the chunks' windows are listed longest chunk
  // first, so that warps running together hold rows of like length (1), or
  // in chunk order (0); read when the matrix is converted or uploaded
  int sell_order = 1;
  // pinned staging for host x / y in spops_spmv_host
  void* pinned = nullptr;
  size_t pinned_bytes = 0;
  DevBuf xbuf, ybuf;
  // second stream and per-range events of the pipelined spops_spmv_host
  cudaStream_t copy_stream = nullptr;
  std::vector<cudaEvent_t> part_events;
  // spops_spmv_host_async: two slots of device x / y used in turn, the
  // upload stream, and per slot the events that order its upload (in), the
  // SpMV's last read of x / y (read) and the download of y (out)
  DevBuf axbuf[2], aybuf[2];
  cudaStream_t in_stream = nullptr;
  cudaEvent_t a_in[2] = {nullptr, nullptr}, a_read[2] = {nullptr, nullptr}, a_out[2] = {nullptr, nullptr};
  int a_next = 0;
  bool a_pending = false;
  // pinned staging of the Matrix Market reader (file chunks on their way to
  // the device) and the event that frees each buffer for its next chunk
  std::vector<void*> file_stage;
  std::vector<cudaEvent_t> file_events;
  // stream-ordered pool for per-call temporaries (PoolBuf): memory freed by
  // one call is handed to the next without returning it to the driver
  cudaMemPool_t pool = nullptr;
  spops_status_t pool_alloc(void** p, size_t bytes);
  void pool_free(void* p);
  // arena for the temporaries of one call inside an ArenaScope: one buffer
  // kept by the context and handed out by a bump pointer, so a call whose
  // temporaries are the same sizes as the last one's maps no memory.  (The
  // stream-ordered pool remaps its free pages into a new range when no free
  // range fits, at several microseconds per 2 MB page.)  An allocation that
  // does not fit goes to the pool; the arena is then regrown, between calls,
  // to the largest total the scopes asked for.
  DevBuf arena;
  // large blocks released by results allocated with DevBuf::alloc_cached (a
  // SpGEMM's C, for instance), kept for the next result of about the same
  // size: cudaMalloc / cudaFree of a GB-sized array cost milliseconds, and
  // their time varies.  Each block carries an event recorded on the context
  // stream when it was released; a reuse waits for it.
  struct CachedBlock {
    void* p;
    size_t bytes;
    cudaEvent_t done;
  };
  std::vector<CachedBlock> block_cache;
  size_t block_cache_bytes = 0;
  void cache_block(void* p, size_t bytes);
  bool take_block(size_t n, void** p, size_t* bytes);
  void drop_block_cache();
  size_t arena_top = 0;       // bytes handed out
  size_t arena_over = 0;      // bytes of live pool allocations made in a scope
  size_t arena_need = 0;      // largest arena_top + arena_over seen
  int arena_depth = 0;        // open ArenaScopes
  cudaEvent_t arena_done = nullptr;    // recorded when the outermost scope ends
  cudaStream_t arena_stream = nullptr;  // the stream that event was recorded on
};

// Temporary device buffer of one API call, from the context's pool and
// ordered on its stream (alloc and free both enqueue on ctx->stream, so the
// memory is reused only by work queued after this call's last use of it).
// SPOPS_TRACE=1 in the environment: wall time of each step of a host-side
// driver on stderr, prefixed by its name (the stream is synchronised at every
// mark, so tracing changes the timing it reports only by those waits).
struct Trace {
  bool on = false;
  const char* name;
  std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
  explicit Trace(const char* who) : name(who) {
    const char* e = std::getenv("SPOPS_TRACE");
    on = e && (e[0] == '1' || e[0] == '2');
  }
  void mark(cudaStream_t st, const char* what) {
    if (!on) return;
    cudaStreamSynchronize(st);
    const auto n = std::chrono::steady_clock::now();
    std::fprintf(stderr, "[%s] %-30s %9.3f ms\n", name, what,
                 std::chrono::duration<double, std::milli>(n - t).count());
    t = n;
  }
};

// Temporary device buffer of one API call.  Inside an ArenaScope it comes
// from the context's arena (released with the scope; the newest buffer is
// handed back at once when released first), otherwise, and when the arena is
// full, from the stream-ordered pool.
struct PoolBuf {
  Context* ctx;
  void* p = nullptr;
  size_t bytes = 0;
  size_t span = 0;     // arena bytes taken (0: pool memory)
  bool over = false;   // pool memory counted in ctx->arena_over
  explicit PoolBuf(Context* c) : ctx(c) {}
  PoolBuf(const PoolBuf&) = delete;
  PoolBuf& operator=(const PoolBuf&) = delete;
  ~PoolBuf() { release(); }
  spops_status_t alloc(size_t n) {
    release();
    if (n == 0) n = 16;
    if (ctx->arena_depth > 0) {
      const size_t a = (n + 255) & ~size_t(255);
      if (ctx->arena_top + a <= ctx->arena.bytes) {
        p = static_cast<char*>(ctx->arena.p) + ctx->arena_top;
        ctx->arena_top += a;
        span = a;
        bytes = n;
        note_need();
        return SPOPS_OK;
      }
      over = true;
      ctx->arena_over += a;
      note_need();
    }
    spops_status_t s = ctx->pool_alloc(&p, n);
    if (s != SPOPS_OK) {
      p = nullptr;
      if (over) ctx->arena_over -= (n + 255) & ~size_t(255);
      over = false;
      return s;
    }
    bytes = n;
    return SPOPS_OK;
  }
  void release() {
    if (p && span) {
      if (static_cast<char*>(p) + span == static_cast<char*>(ctx->arena.p) + ctx->arena_top) ctx->arena_top -= span;
    } else if (p) {
      ctx->pool_free(p);
      if (over) ctx->arena_over -= (bytes + 255) & ~size_t(255);
    }
    p = nullptr;
    bytes = span = 0;
    over = false;
  }
  void swap(PoolBuf& o) {
    std::swap(p, o.p);
    std::swap(bytes, o.bytes);
    std::swap(span, o.span);
    std::swap(over, o.over);
  }
  template <typename T> T* as() const { return static_cast<T*>(p); }

 private:
  void note_need() {
    const size_t t = ctx->arena_top + ctx->arena_over;
    if (t > ctx->arena_need) ctx->arena_need = t;
  }
};

// The temporaries of the calls made while an ArenaScope is open come from
// the context's arena (PoolBuf).  Declare it before the call's PoolBufs.
// Opening the outermost scope regrows the arena to what earlier scopes
// needed (after the stream's queued work, which may still read it) and
// orders this stream after the last scope's work on another stream.
struct ArenaScope {
  Context* ctx;
  size_t mark = 0;
  explicit ArenaScope(Context* c);
  ~ArenaScope();
  ArenaScope(const ArenaScope&) = delete;
  ArenaScope& operator=(const ArenaScope&) = delete;
};

// RAII guard: make ctx->device current for the duration of an API call.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// --------------------------------------------------- CSR stream analysis
// One unit of CSR SpMV work: entries [p0, p1) of rows r0 .. r0+nr-1
// (chunk < 0), or chunk `chunk` of the long row r0 which has nr chunks.
struct CsrSeg {
  int64_t p0, p1, r0;
  int32_t nr;
  int32_t chunk;
};

// Tile analysis of a CSR matrix for the register-sum kernel
// (spmv_csr_tile.cu): tiles of 32*k consecutive entries, one warp each.
struct CsrTiles {
  bool ready = false;
  int k = 0;               // entries per lane
  int64_t tiles = 0;
  int64_t nempty = 0;
  DevBuf tile_row;         // int64 [tiles]: row of the tile's first entry (~row: tile spans an empty row)
  DevBuf flags;            // uint8 [tiles*32]: row starts within each lane's run
  DevBuf carry_in;         // V [tiles]: sum of the tile's entries before its first row start
  DevBuf open_sum;         // V [tiles]: partial sum of the row open at the tile's end
  DevBuf open_row;         // int64 [tiles]: that row, or -1 (no row starts in the tile)
  DevBuf empty;            // int64 [rows]: empty rows
  std::vector<int64_t> part_tb, part_rb;  // tile / row bounds of the pipelined host SpMV's ranges
  void release();
};

// Column-sorted row windows of a CSR matrix (spmv_csr_win.cu).
struct CsrWin {
  bool ready = false;
  int per_sm = 0;          // windows resident per SM (variant 7 / 8 / 9: 1 / 2 / 4)
  int64_t nwin = 0, ntiles = 0, nesc = 0;
  int64_t max_rows = 0;    // rows of the largest window (shared memory per CTA)
  DevBuf win_row0;         // int64 [nwin + 1]
  DevBuf win_tile0;        // int64 [nwin + 1]
  DevBuf tbase;            // int32 [ntiles]: first column, or -1 - escape index
  DevBuf tidx;             // uint32 [ntiles * 32]: (local row << 16) | column offset
  DevBuf tval;             // V [ntiles * 32]: copy of the values
  DevBuf tperm;            // int32 [ntiles * 32]: CSR entry of each slot (-1: padding)
  bool values_fresh = false;
  DevBuf tesc;             // int32 [nesc * 32]: full columns of wide tiles
  void release();
};

// Row-block partition of a CSR matrix for the streaming SpMV kernel
// (spmv_csr.cu).  Block b covers rows [blk_row[b], next block's row) when
// blk_chunk[b] < 0 (a segment of short rows whose entries fit in shared
// memory), or chunk blk_chunk[b] of the single long row blk_row[b].
struct CsrPlan {
  bool ready = false;
  int64_t nblocks = 0;
  int64_t nlong = 0;       // long rows (more than one chunk)
  int cap = 0;             // entries per chunk
  DevBuf blk_row;          // int64 [nblocks + 1]
  DevBuf blk_chunk;        // int32 [nblocks]
  DevBuf partial;          // V [nblocks] long-row chunk sums
  DevBuf counter;          // int32 [nblocks] arrival counters (zero between calls)
  DevBuf seg;              // CsrSeg [nblocks]
  CsrTiles tiles;          // built on first use by the tile kernel
  CsrWin win;              // built on first use by the window kernel
  int band = -1;           // half-width of the x window a segment stages (0 none, -1 not measured)
  void release() {
    blk_row.release(); blk_chunk.release(); partial.release(); counter.release(); seg.release();
    tiles.release();
    win.release();
    ready = false;
    band = -1;
  }
};

// --------------------------------------------------- padded-row formats
// SELL-C-sigma, SELL-C-R, S-ELL and ELL share one device representation:
// stored rows i = 0..rows-1 (sorted order for SELL-C-sigma / SELL-C-R),
// chunk c = i / C holding C stored rows of chunk_len[c] slots each, starting
// at chunk_off[c]; slot k of stored row i is at
//   row-major: chunk_off[c] + (i - c*C) * chunk_len[c] + k   (reference layout)
//   col-major: chunk_off[c] + (i - c*C) + k * C              (device-native)
// Padding slots hold column -1 and value 0.  row_len[i] is the number of
// slots of stored row i up to its last real entry; y[reorder[i]] (or y[i]
// when unsorted) receives its sum.  Rows longer than kPadLong slots are
// summed by whole thread blocks over pieces of kPadPiece slots.
struct PadPiece {
  int64_t row;      // stored row
  int32_t piece;    // piece index within the row
  int32_t npieces;  // pieces of this row
};

// Window of a 32-row column-major chunk: a head window sums slots
// [widx * kPadWindow, +kPadWindow) of the chunk's head (see padded_window32);
// a tail window sums one row's tail entries, which sit contiguously in the
// tail arrays.  The chunk's windows combine their per-row sums in window order.
struct PadWin {
  int64_t chunk;   // chunk index
  int64_t first;   // index of the chunk's first window
  int32_t widx;    // this window's index among the chunk's windows
  int32_t nw;      // windows of the chunk (head windows first, then tail windows)
  int64_t tail;    // tail window: first entry in the tail arrays; head window: -1
  int32_t tlen;    // tail window: entries
  int32_t tlane;   // tail window: the row's position in the chunk
};

// A stored row's tail: its slots [from, from + len) of a column-major chunk,
// copied to tail entries [start, start + len) (contiguous, row order).
struct PadTail {
  int64_t row;
  int64_t start;
  int32_t from;
  int32_t len;
};

struct PaddedData {
  int64_t C = 0, sigma = 0, align = 1, nchunks = 0, stored = 0;
  bool sorted = false;
  int64_t max_row = 0, min_row = 0;
  DevBuf reorder;    // I [rows]
  DevBuf chunk_len;  // I [nchunks]
  DevBuf chunk_off;  // int64 [nchunks + 1]
  DevBuf row_len;    // int32 [rows]
  int64_t npieces = 0;
  DevBuf piece;      // PadPiece [npieces]
  DevBuf partial;    // double [npieces]
  DevBuf counter;    // int32 [npieces]
  // windows of 32-row column-major chunks (C == 32 only).  A chunk's head
  // holds its slots up to the fourth-longest row's length; the slots beyond,
  // held by at most three rows, are copied row by row into the tail arrays so
  // that a row running alone is read contiguously.
  int64_t nwin = 0;
  DevBuf win;        // PadWin [nwin]
  DevBuf win_partial;  // double [nwin * 32]
  DevBuf win_counter;  // int32 [nchunks]
  DevBuf head;       // int32 [nchunks]: head width in slots
  int64_t ntails = 0, ntail_entries = 0;
  DevBuf tails;      // PadTail [ntails]
  DevBuf tcol, tval; // I / V [ntail_entries]
  bool tails_fresh = true;  // tail values copied from the current values
  void release() {
    reorder.release(); chunk_len.release(); chunk_off.release(); row_len.release();
    piece.release(); partial.release(); counter.release();
    win.release(); win_partial.release(); win_counter.release();
    head.release(); tails.release(); tcol.release(); tval.release();
    nwin = 0;
    ntails = ntail_entries = 0;
  }
};

// DIA: diag_offsets (int64, ndiag) in first-appearance order; diag_data
// [ndiag x stride] indexed by row (include/sparse_format.h:172-184).
struct DiaData {
  int64_t ndiag = 0, stride = 0;
  DevBuf offsets;  // int64 [ndiag]
  DevBuf data;     // V [ndiag * stride]
  // smallest / largest offset, read back once by the first SpMV: a block of
  // rows stages the x window its diagonals reach in shared memory when it fits
  bool span_known = false;
  int64_t lo = 0, hi = 0;
  void release() { offsets.release(); data.release(); }
};

// BSR: block rows of br x bc blocks stored row-major (include/sparse_format.h:110-127).
struct BsrData {
  int64_t br = 0, bc = 0, mb = 0, nb = 0, nnzb = 0;
  DevBuf row_ptr;  // I [mb + 1]
  DevBuf bcol;     // I [nnzb]
  DevBuf data;     // V [nnzb * br * bc]
  void release() { row_ptr.release(); bcol.release(); data.release(); }
};

// CSR5 tiles of 32 lanes x 16 entries (csr5.cu).
struct Csr5Data {
  int64_t tiles = 0, nempty = 0;
  DevBuf tcol, tval;   // I, V [tiles * 512], transposed within tiles
  DevBuf desc;         // uint32 [tiles * 32] row-start flags per lane
  DevBuf lane_row;     // int64 [tiles * 32] row of each lane's first entry
  DevBuf tile_ptr;     // uint32 [tiles + 1]
  DevBuf carry_in, open_sum, open_row;  // calibrator: V, V, int64 [tiles]
  DevBuf empty;        // int64 [nempty] empty rows
  void release();
};

// Transpose of a CSR pattern (A^T as CSR), built once per pattern; values
// refreshed through perm after A's values change (adjoint.cu).
struct Matrix;
struct TransposeData {
  bool ready = false, values_fresh = false;
  DevBuf rp;    // I [cols + 1]
  DevBuf ri;    // I [nnz]
  DevBuf perm;  // int64 [nnz]: entry of A at each position of A^T
  DevBuf val;   // V [nnz]
  Matrix* view = nullptr;  // CSR handle of A^T over the arrays above
  // Source-row bands for A^T x read through perm: band b holds, row by row,
  // the entries of A^T whose source rows lie in the b-th of nbands row ranges
  // of about equal entry counts, so that one band's slice of A's values stays
  // in L2 while its gathers run (adjoint.cu).  nbands = 0: not built.
  static constexpr int kMaxBands = 8;
  int nbands = 0;
  DevBuf brp[kMaxBands], bri[kMaxBands], bperm[kMaxBands];  // I [cols + 1], I, int64 [band entries]
  Matrix* bview[kMaxBands] = {};                             // CSR handles over them
  void release();
};

// ---------------------------------------------------------------- matrix
struct Matrix {
  Context* ctx = nullptr;
  spops_format_t format = SPOPS_FMT_CSR;
  spops_index_t itype = SPOPS_INDEX_I32;
  spops_value_t vtype = SPOPS_VALUE_F64;
  spops_layout_t layout = SPOPS_ROW_MAJOR;
  int64_t rows = 0, cols = 0, nnz = 0;
  // CSR / COO arrays (COO: row = row index array)
  DevBuf row, col, val;
  CsrPlan plan;
  PaddedData pad;
  DiaData dia;
  BsrData bsr;
  TransposeData tr;
  Csr5Data csr5;
  DevBuf spmm_partial;  // SpMM long-row chunk sums (k per chunk)
  // SPOPS_FMT_VLCLUSTER (row = rowptr [clusters + 1], col = colids [nnz],
  // val = values [cl_nnzv]; rows = CSR rows): rows per cluster, value
  // offsets per cluster, and the first row of every cluster (int64)
  DevBuf cl_sz, cl_rpv, cl_off;
  int64_t clusters = 0, cl_nnzv = 0, cl_max_sz = 0;
  // COO: the same entries as a CSR matrix sorted by row (owned)
  Matrix* csr_view = nullptr;
  // host copy of the pattern (int64), made once for the host clustering
  std::vector<int64_t> host_rp, host_ci;
  size_t isize() const { return itype == SPOPS_INDEX_I32 ? 4 : 8; }
  size_t vsize() const { return vtype == SPOPS_VALUE_F32 ? 4 : 8; }
  void release_all();
};

// LSH candidate pairs (device arrays, sorted by (i, j), unique)
struct PairSet {
  int64_t count = 0;
  DevBuf pi, pj, score;  // int64, int64, double
  void release() { pi.release(); pj.release(); score.release(); count = 0; }
};

struct SpgemmStats {
  int64_t flops = 0, clusters = 0, dense_clusters = 0, pairs = 0, cluster_columns = 0, c_cluster_columns = 0;
  double minhash_ms = 0, lsh_ms = 0, hc_ms = 0, cluster_ms = 0, symbolic_ms = 0, numeric_ms = 0, to_csr_ms = 0;
};

// ------------------------------------------------------------ kernels API
spops_status_t csr_analyse(Context* ctx, Matrix* A);
spops_status_t csr_spmv(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y);
// tile kernel (spmv_csr_tile.cu); usable when the column and value arrays are
// aligned for the lane's vector loads
bool csr_tile_usable(const Matrix* A, int variant);
// Y = alpha*A*X + beta*Y with k = 8, 16 or 32 right-hand sides on the SpMV's
// tile plan (k / 4 lanes per entry); *used = false (nothing done) unless the
// matrix and X allow its vector loads and X's row stride is at most 2k.
bool csr_tile_spmm_usable(const Matrix* A, const void* X, int64_t ldx, int64_t k);
spops_status_t csr_tile_spmm(Context* ctx, Matrix* A, double alpha, const void* X, int64_t ldx, int64_t k,
                             double beta, void* Y, int64_t ldy, bool* used);
spops_status_t csr_tile_analyse(Context* ctx, Matrix* A, int k);
// the tile SpMV with value e read as vsrc[perm[e]] (A's column and value
// arrays as csr_tile_usable(A, 0) wants; perm 64-byte aligned)
spops_status_t csr_tile_spmv_indirect(Context* ctx, Matrix* A, const int64_t* perm, const void* vsrc, double alpha,
                                      const void* x, double beta, void* y);
spops_status_t csr_tile_spmv(Context* ctx, Matrix* A, int variant, double alpha, const void* x, double beta, void* y);
// The default tile SpMV in `parts` row ranges; done(r0, r1) is called after
// each range is enqueued, when rows [r0, r1) of y are final on the stream.
spops_status_t csr_tile_spmv_parts(Context* ctx, Matrix* A, int parts, double alpha, const void* x, double beta,
                                   void* y, const std::function<spops_status_t(int64_t, int64_t)>& done);

// spmv_csr_win.cu
bool csr_win_usable(const Matrix* A);
spops_status_t csr_win_spmv(Context* ctx, Matrix* A, int variant, double alpha, const void* x, double beta, void* y);

// formats.cu
spops_status_t convert_from_csr(Context* ctx, Matrix* A, spops_format_t fmt, const spops_format_params_t& p,
                                Matrix** out);
spops_status_t padded_finish(Context* ctx, Matrix* M);  // row lengths, long pieces (after arrays are set)
spops_status_t padded_spmv(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y);
spops_status_t dia_spmv(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y);
spops_status_t bsr_spmv(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y);
spops_status_t coo_analyse(Context* ctx, Matrix* A);
// csr5.cu
spops_status_t csr5_build(Context* ctx, Matrix* A, Matrix* M);
spops_status_t csr5_spmv(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y);
// adjoint.cu
spops_status_t csr_spmv_transpose(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y);
spops_status_t csr_sddmm(Context* ctx, Matrix* A, double alpha, const void* g, const void* x, void* out);
// lsh.cu, hc.cpp, spgemm.cu
spops_status_t minhash_signatures(Context* ctx, Matrix* A, int k, uint64_t seed, uint64_t* sig);
spops_status_t lsh_pairs(Context* ctx, const uint64_t* sig, int64_t n, int k, int bands, bool constrain,
                         PairSet* out);
// Learned format choice (csrc/selector.cpp): the fitted decision tree over
// derived features; fills spops_convert parameters.
void tree_select(const spops_features_t& f, spops_format_t* format, spops_format_params_t* params);

spops_status_t hierarchical_clustering(const int64_t* rp, const int64_t* ci, int64_t n, const int64_t* pi,
                                       const int64_t* pj, const double* ps, int64_t np, int64_t cluster_size,
                                       std::vector<int64_t>& perm, std::vector<int64_t>& offsets);
// The same clustering on the device from device pairs (falls back to the
// host loop for pair lists that are not sorted i < j pairs); permutation and
// offsets written to device memory (offsets sized rows + 1).
spops_status_t hierarchical_clustering_device(Context* ctx, Matrix* A, const int64_t* pi, const int64_t* pj,
                                              const double* ps, int64_t np, int64_t cluster_size, int64_t* perm_d,
                                              int64_t* offs_d, int64_t* ncl_out, int64_t* rounds_out);
// cluster_out: C in the clustered form of A's clusters (SPOPS_FMT_VLCLUSTER,
// rows in cluster order) instead of CSR in A's row order
spops_status_t cluster_spgemm(Context* ctx, Matrix* A, Matrix* B, const int64_t* perm, const int64_t* offsets,
                              int64_t nclusters, bool sort_output, double l2_budget, Matrix** C, SpgemmStats* st,
                              bool rowwise = false, bool cluster_out = false, bool device_arrays = false);
// clustered (VLength) form of a CSR matrix and back (spgemm.cu)
spops_status_t vlcluster_from_csr(Context* ctx, Matrix* A, const int64_t* offsets, int64_t nclusters, Matrix** out);
spops_status_t vlcluster_to_csr(Context* ctx, Matrix* M, Matrix** out);
spops_status_t vlcluster_finish(Context* ctx, Matrix* M, const int64_t* off_h);  // cluster_sz, cl_off, max size
// spgemm_topk.cu
spops_status_t rowwise_spgemm(Context* ctx, Matrix* A, Matrix* B, bool sort_output, Matrix** C, SpgemmStats* st);
spops_status_t topk_spgemm(Context* ctx, Matrix* A, int64_t top_k, Matrix** C);
// adjoint.cu: A^T as a CSR handle owned by A (built once, values refreshed)
spops_status_t csr_transpose_view(Context* ctx, Matrix* A, Matrix** view);
// features.cu: statistics of a device count vector of length len whose
// entries sum to nnz -- non-zero count, min, max, mean, the sum of squared
// deviations from the mean, the P-ratio and the Gini coefficient
struct CountSummary {
  int64_t nz = 0, mn = 0, mx = 0;
  double ave = 0, sq = 0, p = 0, gini = 0;
};
spops_status_t count_summary(Context* ctx, const int64_t* cnt, int64_t len, int64_t nnz, CountSummary* out);
// batched.cu
spops_status_t csr_spmm(Context* ctx, Matrix* A, double alpha, const void* X, int64_t ldx, int64_t k, double beta,
                        void* Y, int64_t ldy);
spops_status_t validate_columns(Context* ctx, const void* col, int64_t count, spops_index_t it, int64_t ncols,
                                bool allow_pad);

}  // namespace spops

struct spops_context_s : spops::Context {};
struct spops_matrix_s : spops::Matrix {};
