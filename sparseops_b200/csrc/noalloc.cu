// CSR SpMV that allocates nothing: spops_csr_spmv_noalloc.
//
// Some callers cannot allocate device memory at the point where they need a
// product: code running under a memory pool that forbids cudaMalloc (a
// serving process that reserves all device memory up front), code inside a
// callback or plug-in that may not touch the allocator, or a real-time loop
// where an allocation's implicit synchronisation is not acceptable.  The
// handle-based path (spops_csr_create + spops_spmv) allocates its analysis
// (segment list, long-row chunk sums) once per matrix; this entry point
// instead keeps its scratch in one fixed array in device memory that the
// library declares at file scope, so a call needs no allocation at all.
//
// The work is cut into fixed windows of kWin entries (no per-matrix
// analysis).  One warp per window sums the rows that start in the window
// (products staged in shared memory, one lane per row), and
// records two partial sums in the scratch array: the part of the row that was
// already open when the window began (carry_in) and the part of the last row
// that is still open when it ends (open_sum, open_row).  A second kernel adds,
// in window order, the following windows' carry_in to every open row.
// The row pointer is checked on the device before any window is summed: a
// first kernel tests row_offset[0] == 0, row_offset[rows] == nnz and
// row_offset[r] <= row_offset[r + 1] for every row, and sets bit 2 of the
// error word if any fails; the window kernels read that word first and do
// nothing when it is set, so a malformed row pointer never steers an access.
// Column indices are range-checked in the window kernel: an index outside
// [0, cols) contributes nothing and sets bit 1 of the error word.  Either bit
// makes the call return SPOPS_ERR_INVALID.
//
// Limits and sharing:
//   * the scratch array holds kNoAllocScratchBytes (4 MiB) per device: 32
//     bytes per window, so nnz <= kMaxWindows * kWin = 134,217,728 entries;
//     larger matrices are rejected with SPOPS_ERR_TOO_LARGE before any work;
//   * every GPU that loads the library holds the array until the process
//     exits; the first call on a device (with that device current) looks up
//     its address once per CUDA context;
//   * all calls on a device share the array: two calls whose work overlaps
//     on the GPU (different streams, no ordering) race on it.  The error word
//     is cleared at the start of every call; the window slots need no
//     clearing (each call writes every slot it reads);
//   * the call synchronises `stream` at the end (to report range errors).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "device_util.cuh"
#include "spops_internal.h"

namespace spops {
namespace {

constexpr int64_t kNoAllocScratchBytes = 4ll << 20;
constexpr int kWin = 1024;  // entries per window
struct WinSlot {
  double carry_in;   // sum of the row open at the window's start, within the window
  double open_sum;   // sum of the row still open at the window's end, within the window
  int64_t open_row;  // that row, or -1
  int64_t pad;
};
constexpr int64_t kErrBytes = 256;  // error word, then the window slots
constexpr int64_t kMaxWindows = (kNoAllocScratchBytes - kErrBytes) / (int64_t)sizeof(WinSlot);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kErrColumn = 1;  // a column index outside [0, cols)
constexpr int kErrRowPtr = 2;  // row_offset not non-decreasing from 0 to nnz

// Per-device address of g_noalloc_scratch (host code must not use the symbol
// itself as a device address).  It is looked up once per device and kept with
// the unique ID of the CUDA context it was found in: after cudaDeviceReset the
// device gets a new primary context and the module is loaded again, so the
// address is looked up again instead of reusing a stale one.  The driver's
// context calls are reached through cudaGetDriverEntryPoint (no link against
// the driver library).
using CtxGetCurrentFn = int (*)(void**);
using CtxGetIdFn = int (*)(void*, unsigned long long*);
std::mutex g_mu;
void* g_addr[64] = {nullptr};
unsigned long long g_ctx_id[64] = {0};
CtxGetCurrentFn g_ctx_get = nullptr;
CtxGetIdFn g_ctx_id_of = nullptr;

spops_status_t driver_fn(const char* name, void** out) {
  cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
  SPOPS_CUDA(cudaGetDriverEntryPoint(name, out, cudaEnableDefault, &q));
  if (q != cudaDriverEntryPointSuccess || !*out)
    return fail(SPOPS_ERR_CUDA, "spops_csr_spmv_noalloc: driver entry point %s not available", name);
  return SPOPS_OK;
}

// ID of the current context, 0 if none is current yet.
unsigned long long current_ctx_id() {
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (g_ctx_get(&ctx) != 0 || !ctx) return 0;
  if (g_ctx_id_of(ctx, &id) != 0) return 0;
  return id;
}

spops_status_t scratch_address(void** out) {
  int dev = 0;
  SPOPS_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(SPOPS_ERR_UNSUPPORTED, "device ordinal %d", dev);
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_ctx_get) {
    void* f0 = nullptr;
    void* f1 = nullptr;
    SPOPS_TRY(driver_fn("cuCtxGetCurrent", &f0));
    SPOPS_TRY(driver_fn("cuCtxGetId", &f1));
    g_ctx_get = reinterpret_cast<CtxGetCurrentFn>(f0);
    g_ctx_id_of = reinterpret_cast<CtxGetIdFn>(f1);
  }
  const unsigned long long id = current_ctx_id();
  if (!g_addr[dev] || id == 0 || id != g_ctx_id[dev]) {
    void* p = nullptr;
    SPOPS_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));  // makes the primary context current
    const unsigned long long now = current_ctx_id();
    if (now == 0) return fail(SPOPS_ERR_CUDA, "spops_csr_spmv_noalloc: no current CUDA context");
    g_addr[dev] = p;
    g_ctx_id[dev] = now;
  }
  *out = g_addr[dev];
  return SPOPS_OK;
}

// row_offset[0] == 0, row_offset[n] == nnz, non-decreasing in between.
template <typename I>
__global__ void rowptr_check_kernel(const I* __restrict__ rp, int64_t n, int64_t nnz, int* __restrict__ err) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  bool bad = false;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += stride)
    bad |= (int64_t)rp[r] > (int64_t)rp[r + 1];
  if (blockIdx.x == 0 && threadIdx.x == 0) bad |= (int64_t)rp[0] != 0 || (int64_t)rp[n] != nnz;
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(err, kErrRowPtr);
}

template <typename I>
__device__ __forceinline__ int64_t lower_bound_rp(const I* rp, int64_t n, int64_t e) {
  int64_t lo = 0, hi = n + 1;  // first r in [0, n] with rp[r] >= e
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if ((int64_t)rp[mid] < e) lo = mid + 1; else hi = mid;
  }
  return lo;
}

template <typename I, typename V>
__global__ void __launch_bounds__(128) window_kernel(const I* __restrict__ rp, const I* __restrict__ ci,
                                                     const V* __restrict__ val, int64_t n, int64_t ncols, int64_t nnz,
                                                     int64_t nwin, const V* __restrict__ x, V* __restrict__ y,
                                                     V alpha, V beta, bool bz, WinSlot* __restrict__ slots,
                                                     int* __restrict__ err) {
  __shared__ V prod_all[4][kWin];
  const int lane = threadIdx.x & 31;
  const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (w >= nwin) return;
  if (*(volatile int*)err & kErrRowPtr) return;  // malformed row pointer: touch nothing
  V* prod = prod_all[(threadIdx.x >> 5) & 3];
  const int64_t e0 = w * kWin;
  const int64_t e1 = (e0 + kWin < nnz) ? e0 + kWin : nnz;
  // products of the window's entries (range-checked gathers)
  for (int64_t e = e0 + lane; e < e1; e += 32) {
    const int64_t c = (int64_t)ci[e];
    V p = V(0);
    if (c >= 0 && c < ncols) p = ld_stream(val + e) * ld_gather(x + c);
    else atomicOr(err, kErrColumn);
    prod[e - e0] = p;
  }
  __syncwarp();
  // rows starting in the window; the last window also owns rows starting at nnz
  // (the row pointer was checked: 0 <= ra <= rb <= n)
  const int64_t ra = lower_bound_rp(rp, n, e0);
  const int64_t rb = (w == nwin - 1) ? n : lower_bound_rp(rp, n, e1);
  // the row open at the window's start (it began before e0) owns the
  // entries up to the first row that starts inside the window
  V cin = V(0);
  {
    const int64_t first_start = (int64_t)rp[ra];  // ra <= n, rp[n] = nnz
    const int64_t lim = (first_start < e1 ? first_start : e1);
    V s = V(0);
    for (int64_t e = e0 + lane; e < lim; e += 32) s += prod[e - e0];
    cin = warp_sum(s);
  }
  int64_t open_row = -1;
  V open_sum = V(0);
  const int64_t nr = (rb < n ? rb : n) - ra;
  for (int64_t base = 0; base < nr; base += 32) {
    const int64_t rr = base + lane;
    V s = V(0);
    bool open = false;
    int64_t r = -1;
    if (rr < nr) {
      r = ra + rr;
      const int64_t s0 = rp[r], s1 = rp[r + 1];
      const int64_t lim = s1 < e1 ? s1 : e1;
      for (int64_t e = s0; e < lim; ++e) s += prod[e - e0];
      open = s1 > e1;
      if (!open) axpby_store(y + r, s, alpha, beta, bz);
    }
    const unsigned om = __ballot_sync(0xffffffffu, open);
    if (om) {  // only the last row starting in the window can run past its end
      const int src = 31 - __clz(om);
      open_row = __shfl_sync(0xffffffffu, r, src);
      open_sum = __shfl_sync(0xffffffffu, s, src);
    }
  }
  if (lane == 0) {
    slots[w].carry_in = (double)cin;
    slots[w].open_sum = (double)open_sum;
    slots[w].open_row = open_row;
  }
}

template <typename I, typename V>
__global__ void window_carry_kernel(const I* __restrict__ rp, int64_t nwin, const WinSlot* __restrict__ slots,
                                    V* __restrict__ y, V alpha, V beta, bool bz, const int* __restrict__ err) {
  const int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (w >= nwin) return;
  if (*(volatile const int*)err & kErrRowPtr) return;
  const int64_t r = slots[w].open_row;
  if (r < 0) return;
  const int64_t end = rp[r + 1];
  double tot = slots[w].open_sum;
  for (int64_t u = w + 1; u < nwin && u * kWin < end; ++u) tot += slots[u].carry_in;
  axpby_store(y + r, (V)tot, alpha, beta, bz);
}

template <typename I, typename V>
spops_status_t run_t(int64_t n, int64_t ncols, int64_t nnz, const void* rp, const void* ci, const void* val,
                     double alpha, const void* x, double beta, void* y, cudaStream_t st, unsigned char* scratch) {
  int* err = reinterpret_cast<int*>(scratch);
  WinSlot* slots = reinterpret_cast<WinSlot*>(scratch + kErrBytes);
  const int64_t nwin = nnz > 0 ? (nnz + kWin - 1) / kWin : 1;
  SPOPS_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
  const int64_t cblocks = std::min<int64_t>((n + 255) / 256 + 1, 148 * 8);
  rowptr_check_kernel<I><<<(unsigned)cblocks, 256, 0, st>>>(static_cast<const I*>(rp), n, nnz, err);
  SPOPS_LAUNCH_CHECK();
  const int64_t blocks = (nwin + 3) / 4;
  window_kernel<I, V><<<(unsigned)blocks, 128, 0, st>>>(
      static_cast<const I*>(rp), static_cast<const I*>(ci), static_cast<const V*>(val), n, ncols, nnz, nwin,
      static_cast<const V*>(x), static_cast<V*>(y), (V)alpha, (V)beta, beta == 0.0, slots, err);
  SPOPS_LAUNCH_CHECK();
  window_carry_kernel<I, V><<<(unsigned)((nwin + 255) / 256), 256, 0, st>>>(
      static_cast<const I*>(rp), nwin, slots, static_cast<V*>(y), (V)alpha, (V)beta, beta == 0.0, err);
  SPOPS_LAUNCH_CHECK();
  int herr = 0;
  SPOPS_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  if (herr & kErrRowPtr)
    return fail(SPOPS_ERR_INVALID,
                "spops_csr_spmv_noalloc: row_offset must rise from 0 to nnz without decreasing (y untouched)");
  if (herr & kErrColumn)
    return fail(SPOPS_ERR_INVALID, "spops_csr_spmv_noalloc: column index outside [0, cols) (skipped)");
  return SPOPS_OK;
}

}  // namespace
}  // namespace spops

using namespace spops;

extern "C" spops_status_t spops_csr_spmv_noalloc(int64_t rows, int64_t cols, int64_t nnz, const void* row_offset,
                                                 const void* col_index, const void* values, spops_index_t itype,
                                                 spops_value_t vtype, double alpha, const void* x, double beta,
                                                 void* y, void* stream) {
  if (rows < 0 || cols < 0 || nnz < 0) return fail(SPOPS_ERR_INVALID, "spops_csr_spmv_noalloc: negative size");
  if (itype != SPOPS_INDEX_I32 && itype != SPOPS_INDEX_I64) return fail(SPOPS_ERR_INVALID, "bad index type");
  if (vtype != SPOPS_VALUE_F32 && vtype != SPOPS_VALUE_F64) return fail(SPOPS_ERR_INVALID, "bad value type");
  const int64_t nwin = nnz > 0 ? (nnz + kWin - 1) / kWin : 1;
  if (nwin > kMaxWindows)
    return fail(SPOPS_ERR_TOO_LARGE, "spops_csr_spmv_noalloc: %lld entries exceed the fixed scratch (at most %lld)",
                (long long)nnz, (long long)(kMaxWindows * kWin));
  if (rows == 0) return SPOPS_OK;
  if (!row_offset || !y || (nnz > 0 && (!col_index || !values || !x)))
    return fail(SPOPS_ERR_INVALID, "spops_csr_spmv_noalloc: null array");
  void* scratch = nullptr;
  SPOPS_TRY(scratch_address(&scratch));
  unsigned char* s = static_cast<unsigned char*>(scratch);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const bool i32 = itype == SPOPS_INDEX_I32, f64 = vtype == SPOPS_VALUE_F64;
  if (i32 && f64) return run_t<int32_t, double>(rows, cols, nnz, row_offset, col_index, values, alpha, x, beta, y, st, s);
  if (i32) return run_t<int32_t, float>(rows, cols, nnz, row_offset, col_index, values, alpha, x, beta, y, st, s);
  if (f64) return run_t<int64_t, double>(rows, cols, nnz, row_offset, col_index, values, alpha, x, beta, y, st, s);
  return run_t<int64_t, float>(rows, cols, nnz, row_offset, col_index, values, alpha, x, beta, y, st, s);
}
