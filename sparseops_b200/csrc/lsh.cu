// MinHash signatures and LSH candidate pairs on the device.
//
// Replaces minhash_signatures_flat (reference include/spgemm_MinHashLSH.h:119-180)
// and lsh_candidate_pairs_from_flat_vector (427-605), which
// lsh_candidate_pairs_vector (777-791) chains.  Outputs are bit-identical:
//   signatures  sig[r][d] = min over the row's columns c of a_d*c + b_d
//               (mod 2^64), a_d, b_d from the reference's LCG (40-43,
//               134-141); empty rows keep UINT64_MAX.  One warp per row, the
//               row's columns broadcast, each lane owning k/32 hash functions.
//   records     bucket = band hash of the band's r = k/bands values
//               (h = h*0x9e3779b97f4a7c15 + v, 277-283); the bands go in
//               batches (as many as 2^24 records hold), each batch one stable
//               radix sort of ((band, bucket) -> row) over records given in
//               (band, row) order, i.e. the reference's (band, bucket, row)
//               order, with one host synchronisation per batch.
//   pairs       each run of equal buckets (size >= 2) pairs every row with
//               every later row, or -- when constrained and the run is longer
//               than 256 -- with its next 16 rows (481-516); pairs (i < j)
//               from all bands are sorted and deduplicated (544-545).
//   scores      matches / k over the two signatures (183-204), one warp per
//               pair.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "spops_internal.h"

namespace spops {
namespace {

inline unsigned grid_for(int64_t work, int threads = 256) {
  int64_t g = (work + threads - 1) / threads;
  return (unsigned)(g < 1 ? 1 : g);
}

template <typename I>
__global__ void minhash_kernel(const I* __restrict__ rp, const I* __restrict__ ci, int64_t n, int k,
                               const uint64_t* __restrict__ a, const uint64_t* __restrict__ b,
                               uint64_t* __restrict__ sig) {
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  const int64_t s = rp[r], e = rp[r + 1];
  for (int d0 = 0; d0 < k; d0 += 64) {  // two hash functions per lane per pass
    const int d1 = d0 + lane, d2 = d0 + 32 + lane;
    const uint64_t a1 = d1 < k ? a[d1] : 0, b1 = d1 < k ? b[d1] : 0;
    const uint64_t a2 = d2 < k ? a[d2] : 0, b2 = d2 < k ? b[d2] : 0;
    uint64_t m1 = ~0ULL, m2 = ~0ULL;
    for (int64_t t = s; t < e; ++t) {
      const uint64_t x = (uint64_t)(int64_t)ci[t];
      const uint64_t h1 = a1 * x + b1, h2 = a2 * x + b2;
      m1 = h1 < m1 ? h1 : m1;
      m2 = h2 < m2 ? h2 : m2;
    }
    if (d1 < k) sig[r * k + d1] = m1;
    if (d2 < k) sig[r * k + d2] = m2;
  }
}

// Bands [band0, band0 + nb): record q = b * n + i holds row i's hash in band
// band0 + b.
__global__ void band_hash_kernel(const uint64_t* __restrict__ sig, int64_t n, int k, int band0, int nb, int r,
                                 uint64_t* __restrict__ bucket, int32_t* __restrict__ rows) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= n * nb) return;
  const int64_t b = q / n, i = q - b * n;
  const uint64_t* s = sig + i * k + (band0 + b) * r;
  uint64_t h = 0;
  for (int t = 0; t < r; ++t) h = h * 0x9e3779b97f4a7c15ULL + s[t];
  bucket[q] = h;
  rows[q] = (int32_t)i;
}

// Bucket value -> a small id: its slot in its band's open-addressing table of
// at least 2n slots (equal values get equal slots, different values different
// ones), so that the rows are grouped by a sort on the band's index and
// log2(slots) + 1 bits instead of 64.  The value ~0 (the table's empty mark)
// gets id mask + 1.  The key becomes band << id_bits | id.
__global__ void bucket_id_kernel(uint64_t* __restrict__ key, int64_t n, int nb, unsigned long long* __restrict__ tabs,
                                 uint64_t mask, int id_bits, int* __restrict__ err) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= n * nb) return;
  const int64_t b = q / n;
  unsigned long long* tab = tabs + b * (int64_t)(mask + 1);
  const uint64_t hi = (uint64_t)b << id_bits;
  const unsigned long long h = key[q];
  if (h == ~0ULL) {
    key[q] = hi | (mask + 1);
    return;
  }
  unsigned long long x = h ^ (h >> 29);
  x *= 0xbf58476d1ce4e5b9ULL;
  x ^= x >> 32;
  uint64_t slot = x & mask;
  for (uint64_t probe = 0; probe <= mask; ++probe) {
    const unsigned long long old = atomicCAS(tab + slot, ~0ULL, h);
    if (old == ~0ULL || old == h) {
      key[q] = hi | slot;
      return;
    }
    slot = (slot + 1) & mask;
  }
  atomicOr(err, 1);  // table full: cannot happen with 2n slots
}

__global__ void run_flag_kernel(const uint64_t* __restrict__ key, int64_t n, int64_t* __restrict__ flag) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) flag[i] = (i == 0 || key[i] != key[i - 1]) ? 1 : 0;
}

// Per sorted record: pairs it starts (with later rows of its run).
__global__ void pair_count_kernel(const int64_t* __restrict__ gid, const int64_t* __restrict__ run_off,
                                  const int64_t* __restrict__ run_len, int64_t n, bool constrain,
                                  int64_t* __restrict__ cnt) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t g = gid[i] - 1;
  const int64_t size = run_len[g];
  int64_t c = run_off[g] + size - 1 - i;  // later rows in the run
  if (constrain && size > 256 && c > 16) c = 16;
  cnt[i] = size >= 2 ? c : 0;
}

__global__ void pair_emit_kernel(const int32_t* __restrict__ rows, int64_t n, const int64_t* __restrict__ cnt,
                                 const int64_t* __restrict__ off, uint64_t* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t c = cnt[i], o = off[i];
  const uint64_t ri = (uint64_t)(uint32_t)rows[i];
  for (int64_t t = 0; t < c; ++t) out[o + t] = (ri << 32) | (uint64_t)(uint32_t)rows[i + 1 + t];
}

__global__ void score_kernel(const uint64_t* __restrict__ sig, int k, const uint64_t* __restrict__ pairs,
                             int64_t np, int64_t* __restrict__ pi, int64_t* __restrict__ pj,
                             double* __restrict__ score) {
  const int64_t p = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (p >= np) return;
  const uint64_t key = pairs[p];
  const int64_t i = (int64_t)(key >> 32), j = (int64_t)(key & 0xffffffffULL);
  int m = 0;
  for (int d = lane; d < k; d += 32) m += (sig[i * k + d] == sig[j * k + d]) ? 1 : 0;
  for (int o = 16; o > 0; o >>= 1) m += __shfl_down_sync(0xffffffffu, m, o);
  if (lane == 0) {
    pi[p] = i;
    pj[p] = j;
    score[p] = (double)m / (double)k;
  }
}

template <typename I>
spops_status_t minhash_t(Context* ctx, Matrix* A, int k, uint64_t seed, uint64_t* sig) {
  std::vector<uint64_t> ha((size_t)k), hb((size_t)k);
  uint64_t s = seed;
  for (int d = 0; d < k; ++d) {  // the reference's LCG (spgemm_MinHashLSH.h:40-43, 134-141)
    s = s * 6364136223846793005ULL + 1442695040888963407ULL;
    ha[d] = (s >> 1) * 2 + 1;
    s = s * 6364136223846793005ULL + 1442695040888963407ULL;
    hb[d] = s;
  }
  SPOPS_TRY(ctx->scratch_reserve(2 * (size_t)k * 8 + 512));
  uint64_t* da = ctx->scratch.as<uint64_t>();
  uint64_t* db = da + k;
  SPOPS_CUDA(cudaMemcpyAsync(da, ha.data(), (size_t)k * 8, cudaMemcpyHostToDevice, ctx->stream));
  SPOPS_CUDA(cudaMemcpyAsync(db, hb.data(), (size_t)k * 8, cudaMemcpyHostToDevice, ctx->stream));
  if (A->rows > 0)
    minhash_kernel<I><<<grid_for(A->rows * 32), 256, 0, ctx->stream>>>(A->row.as<I>(), A->col.as<I>(), A->rows, k, da,
                                                                       db, sig);
  SPOPS_LAUNCH_CHECK();
  SPOPS_CUDA(cudaStreamSynchronize(ctx->stream));  // da/db live in scratch
  return SPOPS_OK;
}

}  // namespace

spops_status_t minhash_signatures(Context* ctx, Matrix* A, int k, uint64_t seed, uint64_t* sig) {
  if (A->format != SPOPS_FMT_CSR) return fail(SPOPS_ERR_INVALID, "MinHash needs a CSR matrix");
  if (k <= 0) return fail(SPOPS_ERR_INVALID, "MinHash: k must be positive");
  if (!A->plan.ready) SPOPS_TRY(csr_analyse(ctx, A));  // validates the pattern
  return A->itype == SPOPS_INDEX_I32 ? minhash_t<int32_t>(ctx, A, k, seed, sig)
                                     : minhash_t<int64_t>(ctx, A, k, seed, sig);
}

spops_status_t lsh_pairs(Context* ctx, const uint64_t* sig, int64_t n, int k, int bands, bool constrain,
                         PairSet* out) {
  out->release();
  if (n <= 0 || bands <= 0 || k <= 0 || k % bands) return SPOPS_OK;  // the reference returns no pairs
  if (n > INT32_MAX) return fail(SPOPS_ERR_UNSUPPORTED, "LSH: more than 2^31 rows");
  const int r = k / bands;
  cudaStream_t st = ctx->stream;
  Trace tr("lsh");
  ArenaScope scope(ctx);  // this call's temporaries come from the arena
  // bands per batch: the records (band, row) of a batch stay below 2^24
  // (about 80 bytes each of temporaries) unless one band alone has more
  const int nb = (int)std::max<int64_t>(1, std::min<int64_t>(bands, ((int64_t)1 << 24) / n));
  const int64_t m = (int64_t)nb * n;  // records of a full batch
  const size_t mm = (size_t)m;
  uint64_t slots = 1;  // per band
  while (slots < 2 * (uint64_t)n) slots <<= 1;
  int id_bits = 1;  // ids are below slots + 1
  while (id_bits < 64 && (uint64_t(1) << id_bits) <= slots) ++id_bits;
  int band_bits = 0;
  while ((1 << band_bits) < nb) ++band_bits;
  const int key_bits = id_bits + band_bits;
  size_t cub_sort = 0, cub_scan = 0, cub_rle = 0;
  {
    uint64_t* kk = nullptr;
    int32_t* vv = nullptr;
    int64_t* cc = nullptr;
    SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, cub_sort, kk, kk, vv, vv, m, 0, key_bits, st));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, cub_scan, cc, cc, m, st));
    SPOPS_CUDA(cub::DeviceRunLengthEncode::Encode(nullptr, cub_rle, kk, kk, cc, cc, m, st));
    size_t inc = 0;
    SPOPS_CUDA(cub::DeviceScan::InclusiveSum(nullptr, inc, cc, cc, m, st));
    cub_scan = std::max(cub_scan, inc);
  }
  const size_t cub_max = std::max({cub_sort, cub_scan, cub_rle});
  PoolBuf key_in(ctx), key_out(ctx), row_in(ctx), row_out(ctx), flag(ctx), gid(ctx), ukeys(ctx), run_len(ctx),
      run_off(ctx), cnt(ctx), off(ctx), small(ctx), cub_tmp(ctx), tab(ctx);
  SPOPS_TRY(key_in.alloc(mm * 8));
  SPOPS_TRY(key_out.alloc(mm * 8));
  SPOPS_TRY(row_in.alloc(mm * 4));
  SPOPS_TRY(row_out.alloc(mm * 4));
  SPOPS_TRY(flag.alloc(mm * 8));
  SPOPS_TRY(gid.alloc(mm * 8));
  SPOPS_TRY(ukeys.alloc(mm * 8));
  SPOPS_TRY(run_len.alloc(mm * 8));
  SPOPS_TRY(run_off.alloc(mm * 8));
  SPOPS_TRY(cnt.alloc(mm * 8));
  SPOPS_TRY(off.alloc(mm * 8));
  SPOPS_TRY(small.alloc(64));  // the run count, the table error flag
  SPOPS_TRY(cub_tmp.alloc(cub_max + 256));
  SPOPS_TRY(tab.alloc((size_t)nb * slots * 8));
  int64_t* nruns = small.as<int64_t>();
  int* id_err = reinterpret_cast<int*>(small.as<char>() + 8);
  SPOPS_CUDA(cudaMemsetAsync(id_err, 0, 4, st));

  tr.mark(st, "setup");
  // pairs of every band, appended
  PoolBuf all(ctx);
  int64_t total = 0, cap = 0;
  for (int band0 = 0; band0 < bands; band0 += nb) {
    const int nbb = std::min(nb, bands - band0);
    const int64_t mb = (int64_t)nbb * n;
    band_hash_kernel<<<grid_for(mb), 256, 0, st>>>(sig, n, k, band0, nbb, r, key_in.as<uint64_t>(),
                                                   row_in.as<int32_t>());
    SPOPS_CUDA(cudaMemsetAsync(tab.p, 0xff, (size_t)nbb * slots * 8, st));
    bucket_id_kernel<<<grid_for(mb), 256, 0, st>>>(key_in.as<uint64_t>(), n, nbb, tab.as<unsigned long long>(),
                                                   slots - 1, id_bits, id_err);
    SPOPS_LAUNCH_CHECK();
    size_t sort_bytes = cub_max;
    SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(cub_tmp.p, sort_bytes, key_in.as<uint64_t>(), key_out.as<uint64_t>(),
                                               row_in.as<int32_t>(), row_out.as<int32_t>(), mb, 0, key_bits, st));
    run_flag_kernel<<<grid_for(mb), 256, 0, st>>>(key_out.as<uint64_t>(), mb, flag.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
    size_t b1 = cub_max, b2 = cub_max, b3 = cub_max;
    SPOPS_CUDA(cub::DeviceScan::InclusiveSum(cub_tmp.p, b1, flag.as<int64_t>(), gid.as<int64_t>(), mb, st));
    SPOPS_CUDA(cub::DeviceRunLengthEncode::Encode(cub_tmp.p, b2, key_out.as<uint64_t>(), ukeys.as<uint64_t>(),
                                                  run_len.as<int64_t>(), nruns, mb, st));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(cub_tmp.p, b3, run_len.as<int64_t>(), run_off.as<int64_t>(), mb, st));
    pair_count_kernel<<<grid_for(mb), 256, 0, st>>>(gid.as<int64_t>(), run_off.as<int64_t>(), run_len.as<int64_t>(),
                                                    mb, constrain, cnt.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
    size_t b4 = cub_max;
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(cub_tmp.p, b4, cnt.as<int64_t>(), off.as<int64_t>(), mb, st));
    int64_t h[2];
    int herr = 0;
    SPOPS_CUDA(cudaMemcpyAsync(&h[0], off.as<int64_t>() + mb - 1, 8, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaMemcpyAsync(&h[1], cnt.as<int64_t>() + mb - 1, 8, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaMemcpyAsync(&herr, id_err, 4, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
    if (herr) return fail(SPOPS_ERR_CUDA, "LSH: bucket table full");
    const int64_t np = h[0] + h[1];
    if (np == 0) continue;
    if (total + np > cap) {  // grow the pair buffer
      PoolBuf bigger(ctx);
      const int64_t ncap = std::max<int64_t>(2 * cap, total + np);
      SPOPS_TRY(bigger.alloc((size_t)ncap * 8));
      if (total) SPOPS_CUDA(cudaMemcpyAsync(bigger.p, all.p, (size_t)total * 8, cudaMemcpyDeviceToDevice, st));
      all.swap(bigger);
      cap = ncap;
    }
    pair_emit_kernel<<<grid_for(mb), 256, 0, st>>>(row_out.as<int32_t>(), mb, cnt.as<int64_t>(), off.as<int64_t>(),
                                                   all.as<uint64_t>() + total);
    SPOPS_LAUNCH_CHECK();
    total += np;
  }
  tr.mark(st, "bands");
  if (total == 0) return SPOPS_OK;
  // sort + unique all pairs (key i << 32 | j: only the bits of i in use above 32)
  int kend = 33;
  while (kend < 64 && (int64_t(1) << (kend - 32)) < n) ++kend;
  size_t cub2 = 0, cub3 = 0;
  int64_t* nsel = nullptr;
  {
    uint64_t* kk = nullptr;
    SPOPS_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, cub2, kk, kk, total, 0, kend, st));
    SPOPS_CUDA(cub::DeviceSelect::Unique(nullptr, cub3, kk, kk, nsel, total, st));
  }
  PoolBuf sorted(ctx), uniq(ctx), tmp(ctx);
  SPOPS_TRY(sorted.alloc((size_t)total * 8));
  SPOPS_TRY(uniq.alloc((size_t)total * 8));
  const size_t nsel_off = (std::max(cub2, cub3) + 255) & ~(size_t)255;  // 8-byte aligned count slot
  SPOPS_TRY(tmp.alloc(nsel_off + 256));
  nsel = reinterpret_cast<int64_t*>(tmp.as<char>() + nsel_off);
  SPOPS_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, cub2, all.as<uint64_t>(), sorted.as<uint64_t>(), total, 0, kend, st));
  SPOPS_CUDA(cub::DeviceSelect::Unique(tmp.p, cub3, sorted.as<uint64_t>(), uniq.as<uint64_t>(), nsel, total, st));
  int64_t nu = 0;
  SPOPS_CUDA(cudaMemcpyAsync(&nu, nsel, 8, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  tr.mark(st, "sort + unique");
  SPOPS_TRY(out->pi.alloc_cached(ctx, (size_t)nu * 8));
  SPOPS_TRY(out->pj.alloc_cached(ctx, (size_t)nu * 8));
  SPOPS_TRY(out->score.alloc_cached(ctx, (size_t)nu * 8));
  score_kernel<<<grid_for(nu * 32), 256, 0, st>>>(sig, k, uniq.as<uint64_t>(), nu, out->pi.as<int64_t>(),
                                                  out->pj.as<int64_t>(), out->score.as<double>());
  SPOPS_LAUNCH_CHECK();
  SPOPS_CUDA(cudaStreamSynchronize(st));
  tr.mark(st, "scores");
  out->count = nu;
  return SPOPS_OK;
}

}  // namespace spops
