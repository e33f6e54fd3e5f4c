// CSR5 on the device: conversion and SpMV.
//
// Replaces csr_to_csr5 (reference include/sparse_conversion.h:946-1387) and
// SpOps_csr5 (src/spmv_csr5.cpp:113-457), the tile-segmented format of
// Liu & Vinter (ICS'15).  The reference sizes tiles for CPU SIMD (omega = SIMD
// lanes, sigma = 16) and writes its kernel with Intel-only intrinsics; here a
// tile is one warp: omega = 32 lanes x sigma = 16 entries = 512 entries.
//
// Layout (built on the device from CSR):
//   col / val      entries of tile t transposed so that step s of lane l,
//                  entry t*512 + l*16 + s, sits at t*512 + s*32 + l: every
//                  step is one coalesced 32-wide load.  The last partial tile is
//                  padded with zero values.
//   desc[t*32+l]   bit s set when entry l*16+s of the tile starts a non-empty
//                  row (the reference's bit_flag, include/sparse_format.h:140-165).
//   lane_row       the row holding each lane's first entry (replaces the
//                  reference's y_offset / tile_desc_offset search).
//   tile_ptr[t]    row of the tile's first entry, bit 31 set when the tile
//                  spans an empty row (as in the reference).
//   empty rows     listed separately (they hold no entry; y = beta*y).
// SpMV: one warp per tile.  Each lane sums its 16 products segment by segment
// (segments split at its flag bits): complete segments go straight to y; the
// part before the lane's first flag (head) and after its last flag (tail)
// combine across lanes with one warp prefix sum -- a row started in lane f
// and continued through lanes f+1..m receives tail(f) + sum(head(f+1..m)).
// The row still open at the end of a tile, and the head of every tile, are
// written to the calibrator arrays; a second small kernel adds, in tile order,
// the heads of the following tiles to each open row (the reference's
// calibrator pass, src/spmv_csr5.cpp:368-384).  Deterministic.
#include <cub/cub.cuh>

#include <algorithm>

#include "device_util.cuh"
#include "spops_internal.h"

namespace spops {
namespace {

constexpr int kOmega = 32, kSigma = 16, kTile = kOmega * kSigma;

inline unsigned grid_for(int64_t work, int threads = 256) {
  int64_t g = (work + threads - 1) / threads;
  return (unsigned)(g < 1 ? 1 : g);
}

// row holding entry e: last r with rp[r] <= e (rows 0..n-1)
template <typename I>
__device__ __forceinline__ int64_t row_of_entry(const I* rp, int64_t n, int64_t e) {
  int64_t lo = 0, hi = n;  // answer in [0, n-1]
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) >> 1;
    if ((int64_t)rp[mid] <= e) lo = mid; else hi = mid;
  }
  return lo;
}

template <typename I, typename V>
__global__ void csr5_build_kernel(const I* __restrict__ rp, const I* __restrict__ ci, const V* __restrict__ v,
                                  int64_t n, int64_t nnz, int64_t tiles, I* __restrict__ tcol, V* __restrict__ tval,
                                  uint32_t* __restrict__ desc, int64_t* __restrict__ lane_row) {
  const int64_t gl = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;  // global lane = t*32 + l
  if (gl >= tiles * kOmega) return;
  const int64_t t = gl / kOmega, l = gl % kOmega;
  const int64_t e0 = t * kTile + l * kSigma;
  uint32_t flags = 0;
  int64_t r = e0 < nnz ? row_of_entry(rp, n, e0) : n;
  lane_row[gl] = r < n ? r : n - 1;
  for (int s = 0; s < kSigma; ++s) {
    const int64_t e = e0 + s;
    const int64_t dst = t * kTile + (int64_t)s * kOmega + l;
    if (e < nnz) {
      while (r + 1 < n && (int64_t)rp[r + 1] <= e) ++r;  // row holding e
      if ((int64_t)rp[r] == e) flags |= 1u << s;         // e starts row r (non-empty)
      tcol[dst] = ci[e];
      tval[dst] = v[e];
    } else {
      tcol[dst] = 0;
      tval[dst] = V(0);
    }
  }
  desc[gl] = flags;
}

template <typename I>
__global__ void csr5_tile_ptr_kernel(const I* __restrict__ rp, int64_t n, int64_t tiles, const int64_t* __restrict__ lane_row,
                                     uint32_t* __restrict__ tile_ptr) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t > tiles) return;
  if (t == tiles) {
    tile_ptr[t] = (uint32_t)n;
    return;
  }
  const int64_t r0 = lane_row[t * kOmega], r1 = lane_row[t * kOmega + kOmega - 1];
  bool empty = false;
  for (int64_t r = r0; r <= r1 && !empty; ++r) empty = rp[r] == rp[r + 1];
  tile_ptr[t] = (uint32_t)r0 | (empty ? 0x80000000u : 0u);
}

template <typename I>
__global__ void csr5_empty_kernel(const I* __restrict__ rp, int64_t n, int64_t* __restrict__ list,
                                  unsigned long long* __restrict__ count) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r < n && rp[r] == rp[r + 1]) list[atomicAdd(count, 1ULL)] = r;
}

template <typename I, typename V>
__global__ void __launch_bounds__(256) csr5_kernel(const I* __restrict__ rp, int64_t n, const I* __restrict__ tcol,
                                                   const V* __restrict__ tval, const uint32_t* __restrict__ desc,
                                                   const int64_t* __restrict__ lane_row, int64_t tiles,
                                                   const V* __restrict__ x, V* __restrict__ y, V alpha, V beta,
                                                   bool bz, V* __restrict__ carry_in, V* __restrict__ open_sum,
                                                   int64_t* __restrict__ open_row, const int64_t* __restrict__ empty,
                                                   int64_t nempty) {
  const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= tiles) {  // empty rows: y = beta*y
    for (int64_t q = (w - tiles) * 32 + lane; q < nempty; q += (int64_t)gridDim.x * 8 * 32) {
      const int64_t r = empty[q];
      axpby_store(y + r, V(0), alpha, beta, bz);
    }
    return;
  }
  const int64_t t = w;
  const int64_t gl = t * kOmega + lane;
  const uint32_t flags = desc[gl];
  int64_t row = lane_row[gl];
  V head = V(0), acc = V(0);
  bool in_head = (flags & 1u) == 0;
  const I* tc = tcol + t * kTile + lane;
  const V* tv = tval + t * kTile + lane;
  V prod[kSigma];
#pragma unroll
  for (int s = 0; s < kSigma; ++s) prod[s] = ld_stream(tv + s * kOmega) * ld_gather(x + ld_stream(tc + s * kOmega));
#pragma unroll
  for (int s = 0; s < kSigma; ++s) {
    if (s > 0 && (flags >> s) & 1u) {  // a new row starts at step s
      if (in_head) {
        head = acc;
        in_head = false;
      } else {
        axpby_store(y + row, acc, alpha, beta, bz);  // complete segment inside the lane
      }
      acc = V(0);
      ++row;
      while (row + 1 < n && rp[row] == rp[row + 1]) ++row;  // skip empty rows
    }
    acc += prod[s];
  }
  const bool has_flag = flags != 0;
  V tail = V(0);
  if (in_head) head = acc; else tail = acc;
  // Heads of lanes f+1 .. m (m = next flagged lane, or 31) belong to the row
  // of flagged lane f; heads of lanes 0 .. m0 (first flagged lane) to the row
  // open at the tile's start.  Segmented inclusive scan of the heads with a
  // segment starting after every flagged lane (no prefix differences, so no
  // cancellation): S(m) = sum of its group.
  const unsigned fmask = __ballot_sync(0xffffffffu, has_flag);
  V S = head;
  bool seg = lane == 0 || ((fmask >> (lane - 1)) & 1u);
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const V su = __shfl_up_sync(0xffffffffu, S, o);
    const bool gu = __shfl_up_sync(0xffffffffu, seg, o);
    if (lane >= o) {
      if (!seg) S += su;
      seg = seg || gu;
    }
  }
  const unsigned later = fmask & ~((2u << lane) - 1u);  // flagged lanes after this one (lane 31: none)
  const int m = later ? __ffs(later) - 1 : 31;
  const V Sm = __shfl_sync(0xffffffffu, S, m);
  const int m0 = fmask ? __ffs(fmask) - 1 : 31;
  const V cin = __shfl_sync(0xffffffffu, S, m0);  // heads of lanes 0 .. m0
  if (has_flag) {
    if (later) {
      axpby_store(y + row, tail + Sm, alpha, beta, bz);
    } else {  // the tile's last row: may continue into the next tile
      open_sum[t] = tail + (lane < 31 ? Sm : V(0));
      open_row[t] = row;
    }
  }
  if (lane == 0) {
    carry_in[t] = cin;
    if (!fmask) open_row[t] = -1;
  }
}

// Add, in tile order, the heads of the following tiles to every open row.
template <typename V>
__global__ void csr5_calibrate_kernel(const uint32_t* __restrict__ desc, int64_t tiles, const V* __restrict__ carry_in,
                                      const V* __restrict__ open_sum, const int64_t* __restrict__ open_row,
                                      V* __restrict__ y, V alpha, V beta, bool bz) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= tiles) return;
  const int64_t r = open_row[t];
  if (r < 0) return;
  V tot = open_sum[t];
  for (int64_t u = t + 1; u < tiles; ++u) {
    tot += carry_in[u];
    bool flagged = false;
    for (int l = 0; l < kOmega && !flagged; ++l) flagged = desc[u * kOmega + l] != 0;
    if (flagged) break;
  }
  axpby_store(y + r, tot, alpha, beta, bz);
}

template <typename I, typename V>
spops_status_t build_t(Context* ctx, Matrix* A, Matrix* M) {
  cudaStream_t st = ctx->stream;
  Csr5Data& D = M->csr5;
  const int64_t n = A->rows, nnz = A->nnz;
  D.tiles = (nnz + kTile - 1) / kTile;
  const size_t slots = (size_t)std::max<int64_t>(D.tiles * kTile, 1);
  SPOPS_TRY(D.tcol.alloc(slots * sizeof(I)));
  SPOPS_TRY(D.tval.alloc(slots * sizeof(V)));
  SPOPS_TRY(D.desc.alloc((size_t)std::max<int64_t>(D.tiles * kOmega, 1) * 4));
  SPOPS_TRY(D.lane_row.alloc((size_t)std::max<int64_t>(D.tiles * kOmega, 1) * 8));
  SPOPS_TRY(D.tile_ptr.alloc((size_t)(D.tiles + 1) * 4));
  SPOPS_TRY(D.carry_in.alloc((size_t)std::max<int64_t>(D.tiles, 1) * sizeof(V)));
  SPOPS_TRY(D.open_sum.alloc((size_t)std::max<int64_t>(D.tiles, 1) * sizeof(V)));
  SPOPS_TRY(D.open_row.alloc((size_t)std::max<int64_t>(D.tiles, 1) * 8));
  SPOPS_TRY(D.empty.alloc((size_t)std::max<int64_t>(n, 1) * 8));
  if (D.tiles > 0 && n > 0) {
    csr5_build_kernel<I, V><<<grid_for(D.tiles * kOmega), 256, 0, st>>>(
        A->row.as<I>(), A->col.as<I>(), A->val.as<V>(), n, nnz, D.tiles, D.tcol.as<I>(), D.tval.as<V>(),
        D.desc.as<uint32_t>(), D.lane_row.as<int64_t>());
    csr5_tile_ptr_kernel<I><<<grid_for(D.tiles + 1), 256, 0, st>>>(A->row.as<I>(), n, D.tiles,
                                                                    D.lane_row.as<int64_t>(), D.tile_ptr.as<uint32_t>());
    SPOPS_LAUNCH_CHECK();
  }
  SPOPS_TRY(ctx->scratch_reserve(256));
  unsigned long long* cnt = ctx->scratch.as<unsigned long long>();
  SPOPS_CUDA(cudaMemsetAsync(cnt, 0, 8, st));
  if (n > 0) {
    csr5_empty_kernel<I><<<grid_for(n), 256, 0, st>>>(A->row.as<I>(), n, D.empty.as<int64_t>(), cnt);
    SPOPS_LAUNCH_CHECK();
  }
  unsigned long long h = 0;
  SPOPS_CUDA(cudaMemcpyAsync(&h, cnt, 8, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  D.nempty = (int64_t)h;
  // own copy of the row offsets (the kernel skips empty rows with them)
  SPOPS_TRY(M->row.alloc((size_t)(n + 1) * sizeof(I)));
  SPOPS_CUDA(cudaMemcpyAsync(M->row.p, A->row.p, (size_t)(n + 1) * sizeof(I), cudaMemcpyDeviceToDevice, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  return SPOPS_OK;
}

template <typename I, typename V>
spops_status_t spmv_t(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y) {
  const Csr5Data& D = A->csr5;
  if (A->rows == 0) return SPOPS_OK;
  const bool bz = beta == 0.0;
  const int64_t warps = D.tiles + (D.nempty + 31) / 32;
  if (warps > 0) {
    const int64_t grid = (warps + 7) / 8;
    csr5_kernel<I, V><<<(unsigned)grid, 256, 0, ctx->stream>>>(
        A->row.as<I>(), A->rows, D.tcol.as<I>(), D.tval.as<V>(), D.desc.as<uint32_t>(), D.lane_row.as<int64_t>(),
        D.tiles, static_cast<const V*>(x), static_cast<V*>(y), (V)alpha, (V)beta, bz, D.carry_in.as<V>(),
        D.open_sum.as<V>(), D.open_row.as<int64_t>(), D.empty.as<int64_t>(), D.nempty);
    SPOPS_LAUNCH_CHECK();
  }
  if (D.tiles > 0) {
    csr5_calibrate_kernel<V><<<grid_for(D.tiles), 256, 0, ctx->stream>>>(
        D.desc.as<uint32_t>(), D.tiles, D.carry_in.as<V>(), D.open_sum.as<V>(), D.open_row.as<int64_t>(),
        static_cast<V*>(y), (V)alpha, (V)beta, bz);
    SPOPS_LAUNCH_CHECK();
  }
  return SPOPS_OK;
}

}  // namespace

void Csr5Data::release() {
  tcol.release(); tval.release(); desc.release(); lane_row.release(); tile_ptr.release();
  carry_in.release(); open_sum.release(); open_row.release(); empty.release();
  tiles = 0;
  nempty = 0;
}

spops_status_t csr5_build(Context* ctx, Matrix* A, Matrix* M) {
  const bool i32 = A->itype == SPOPS_INDEX_I32, f64 = A->vtype == SPOPS_VALUE_F64;
  if (A->rows > (int64_t)0x7fffffff) return fail(SPOPS_ERR_UNSUPPORTED, "CSR5: more than 2^31 rows");
  if (i32 && f64) return build_t<int32_t, double>(ctx, A, M);
  if (i32) return build_t<int32_t, float>(ctx, A, M);
  if (f64) return build_t<int64_t, double>(ctx, A, M);
  return build_t<int64_t, float>(ctx, A, M);
}

spops_status_t csr5_spmv(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y) {
  const bool i32 = A->itype == SPOPS_INDEX_I32, f64 = A->vtype == SPOPS_VALUE_F64;
  if (i32 && f64) return spmv_t<int32_t, double>(ctx, A, alpha, x, beta, y);
  if (i32) return spmv_t<int32_t, float>(ctx, A, alpha, x, beta, y);
  if (f64) return spmv_t<int64_t, double>(ctx, A, alpha, x, beta, y);
  return spmv_t<int64_t, float>(ctx, A, alpha, x, beta, y);
}

}  // namespace spops
