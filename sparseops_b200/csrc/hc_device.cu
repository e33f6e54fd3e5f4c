// Hierarchical clustering of rows from LSH candidate pairs, on the device.
//
// Replaces hierarchical_clustering_v0_fast (reference include/spgemm_utility.h:
// 742-915) with the same output bit for bit: the permutation and offsets of
// csrc/hc.cpp, whose merge rules restate the reference's.  That loop takes
// candidates best first and each step reads and writes the union-find state
// of two clusters only.  Here every candidate is a task with a priority -- the
// order in which the sequential loop would take it: (score, i, j) descending,
// which is both the initial list's order (pairs sorted by (i, j), scores
// stable-sorted descending, equal scores in reverse input order) and the
// order of the heap of pairs found while merging -- and the tasks run in
// rounds of deterministic reservations:
//   1. every live task finds the roots of its two rows and reserves both
//      (an atomic max of priority per root);
//   2. a task that holds both reservations applies the sequential step to
//      them: merge two open roots (the smaller cluster joins the larger, ties
//      keep row i; a cluster reaching cluster_size closes), or, when its rows
//      are not both roots, queue the root pair with its exact Jaccard score if
//      it is new and not an initial pair -- a new task, live from the next
//      round;
//   3. (nothing to clear: a reservation carries its round's number, so the
//      next round sees every old one as free).
// A task that holds its roots is the highest-priority live task touching
// them, so every cluster sees its steps in the sequential order; steps on
// disjoint clusters commute.  A new task touches only its creator's roots,
// which its creator held.  A task whose roots are the same or one of them is
// closed can have no effect, now or later (closed clusters never merge or
// reopen), and retires at once.  Each round retires at least the best live
// task, so the rounds end; their count is the longest chain of tasks on
// shared clusters.
//
// Output: the root of every row, then one stable radix sort of (root, row)
// pairs: clusters by root row, rows ascending inside each -- the reference's
// order (spgemm_utility.h:890-915).
//
// Used when the pairs are i < j, in range, sorted by (i, j) and unique (what
// spops_lsh_pairs produces); anything else goes to the host loop.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <vector>

#include "spops_internal.h"

namespace spops {

namespace {

inline unsigned hc_grid(int64_t work, int threads = 256) {
  const int64_t g = (work + threads - 1) / threads;
  return (unsigned)(g < 1 ? 1 : (g > 1048576 ? 1048576 : g));
}

struct Tasks {
  double* s;
  int32_t* i;
  int32_t* j;
};

// priority of task a above task b: (score, i, j) larger
__device__ __forceinline__ bool hc_above(const Tasks& T, int32_t a, int32_t b) {
  const double sa = T.s[a], sb = T.s[b];
  if (sa != sb) return sa > sb;
  if (T.i[a] != T.i[b]) return T.i[a] > T.i[b];
  return T.j[a] > T.j[b];
}

// root of x: union by size keeps every tree under 32 levels, so 64 steps
// always reach it; a node that is not a root after them reports an error
__device__ __forceinline__ int32_t hc_find(const int32_t* __restrict__ parent, int32_t x, int* __restrict__ err) {
  for (int step = 0; step < 64; ++step) {
    const int32_t p = parent[x];
    if (p == x) return x;
    x = p;
  }
  atomicOr(err, 32);
  return x;
}

constexpr int kCasLimit = 1 << 22;  // CAS attempts on one root before the round reports an error

// A reservation is (round << 32 | task): one made in an earlier round is
// stale, so nothing needs clearing between rounds.
__device__ __forceinline__ unsigned long long hc_stamp(uint32_t round, int32_t c) {
  return ((unsigned long long)round << 32) | (uint32_t)c;
}

// keep the better of the current holder (of this round) and task c in res[r]
__device__ __forceinline__ void hc_reserve(unsigned long long* __restrict__ res, int32_t r, int32_t c, uint32_t round,
                                           const Tasks& T, int* __restrict__ err) {
  unsigned long long cur = res[r];
  const unsigned long long mine = hc_stamp(round, c);
  for (int it = 0; it < kCasLimit; ++it) {
    if ((uint32_t)(cur >> 32) == round && !hc_above(T, c, (int32_t)(uint32_t)cur)) return;
    const unsigned long long old = atomicCAS(res + r, cur, mine);
    if (old == cur) return;
    cur = old;
  }
  atomicOr(err, 4);
}

__global__ void hc_check_pairs_kernel(const int64_t* __restrict__ pi, const int64_t* __restrict__ pj, int64_t np,
                                      int64_t n, int* __restrict__ bad) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= np) return;
  const int64_t a = pi[t], b = pj[t];
  bool ok = a >= 0 && a < b && b < n;
  if (ok && t > 0) ok = pi[t - 1] < a || (pi[t - 1] == a && pj[t - 1] < b);
  if (!ok) atomicOr(bad, 1);
}

__global__ void hc_init_rows_kernel(int64_t n, int32_t* __restrict__ parent, int32_t* __restrict__ size,
                                    unsigned char* __restrict__ open, unsigned long long* __restrict__ res) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  parent[r] = (int32_t)r;
  size[r] = 1;
  open[r] = 1;
  res[r] = 0;  // round 0: no round runs as 0
}

__global__ void hc_init_tasks_kernel(const int64_t* __restrict__ pi, const int64_t* __restrict__ pj,
                                     const double* __restrict__ ps, int64_t np, Tasks T, int32_t* __restrict__ live) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= np) return;
  T.s[t] = ps[t];
  T.i[t] = (int32_t)pi[t];
  T.j[t] = (int32_t)pj[t];
  live[t] = (int32_t)t;
}

// 1. roots and reservations; tasks that can have no effect retire here.
// Also zeroes the count of the next round's live tasks (the commit kernel
// after it adds to that count).
__global__ void hc_reserve_kernel(const int32_t* __restrict__ live, const unsigned long long* __restrict__ nlive_d,
                                  unsigned long long* __restrict__ nnext, uint32_t round, Tasks T,
                                  const int32_t* __restrict__ parent, const unsigned char* __restrict__ open,
                                  unsigned long long* __restrict__ res, int32_t* __restrict__ ri_out,
                                  int32_t* __restrict__ rj_out, int* __restrict__ err) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q == 0) *nnext = 0;
  if (q >= (int64_t)*nlive_d) return;
  const int32_t c = live[q];
  const int32_t ri = hc_find(parent, T.i[c], err), rj = hc_find(parent, T.j[c], err);
  if (ri == rj || !open[ri] || !open[rj]) {  // no effect, now or later
    ri_out[q] = -1;
    rj_out[q] = -1;
    return;
  }
  ri_out[q] = ri;
  rj_out[q] = rj;
  hc_reserve(res, ri, c, round, T, err);
  hc_reserve(res, rj, c, round, T, err);
}

// |row a ∩ row b| / |row a ∪ row b| over entry counts, as the host loop
// computes it: the entries of row b whose column occurs in row a
template <typename I>
__device__ double hc_jaccard(const I* __restrict__ rp, const I* __restrict__ ci, int64_t a, int64_t b) {
  const int64_t a0 = rp[a], a1 = rp[a + 1], b0 = rp[b], b1 = rp[b + 1];
  bool sorted = true;
  for (int64_t x = a0 + 1; x < a1 && sorted; ++x) sorted = ci[x - 1] < ci[x];
  int64_t common = 0;
  for (int64_t y = b0; y < b1; ++y) {
    const I c = ci[y];
    bool hit = false;
    if (sorted) {
      int64_t lo = a0, hi = a1;
      while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (ci[mid] < c) lo = mid + 1; else hi = mid;
      }
      hit = lo < a1 && ci[lo] == c;
    } else {
      for (int64_t x = a0; x < a1 && !hit; ++x) hit = ci[x] == c;
    }
    common += hit ? 1 : 0;
  }
  const int64_t u = (a1 - a0) + (b1 - b0) - common;
  return u == 0 ? 0.0 : (1.0 * (double)common / (double)u);
}

// (a, b) among the initial pairs (sorted by (i, j))
__device__ __forceinline__ bool hc_given(const int64_t* __restrict__ pi, const int64_t* __restrict__ pj, int64_t np,
                                         int64_t a, int64_t b) {
  int64_t lo = 0, hi = np;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (pi[mid] < a || (pi[mid] == a && pj[mid] < b)) lo = mid + 1; else hi = mid;
  }
  return lo < np && pi[lo] == a && pj[lo] == b;
}

// insert key into the open-addressing set; true if it was not there
__device__ __forceinline__ bool hc_seen_insert(unsigned long long* __restrict__ tab, uint64_t mask,
                                               unsigned long long key, int* __restrict__ err) {
  unsigned long long h = key * 0x9e3779b97f4a7c15ULL;
  h ^= h >> 29;
  for (uint64_t probe = 0; probe <= mask; ++probe) {
    const uint64_t slot = (h + probe) & mask;
    const unsigned long long old = atomicCAS(tab + slot, ~0ULL, key);
    if (old == ~0ULL) return true;
    if (old == key) return false;
  }
  atomicOr(err, 8);  // table full (sized for every possible pair: unreachable)
  return false;
}

// 2. tasks holding both roots apply the sequential step
template <typename I>
__global__ void hc_commit_kernel(const int32_t* __restrict__ live, const unsigned long long* __restrict__ nlive_d,
                                 Tasks T,
                                 const int32_t* __restrict__ ri_in, const int32_t* __restrict__ rj_in,
                                 const unsigned long long* __restrict__ res, uint32_t round,
                                 int32_t* __restrict__ parent,
                                 int32_t* __restrict__ size, unsigned char* __restrict__ open, int64_t cluster_size,
                                 const I* __restrict__ rp, const I* __restrict__ ci, const int64_t* __restrict__ pi,
                                 const int64_t* __restrict__ pj, int64_t np, unsigned long long* __restrict__ seen,
                                 uint64_t seen_mask, int64_t cap, unsigned long long* __restrict__ ntasks,
                                 int32_t* __restrict__ next_live, unsigned long long* __restrict__ nnext,
                                 int* __restrict__ err) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= (int64_t)*nlive_d) return;
  const int32_t ri = ri_in[q], rj = rj_in[q];
  if (ri < 0) return;  // retired in the reserve pass
  const int32_t c = live[q];
  const unsigned long long mine = hc_stamp(round, c);
  if (res[ri] != mine || res[rj] != mine) {  // a better task holds a root: next round
    next_live[atomicAdd(nnext, 1ULL)] = c;
    return;
  }
  const int32_t i = T.i[c], j = T.j[c];
  if (ri == i && rj == j) {  // both rows are roots, both open: merge
    const int32_t keep = size[i] < size[j] ? j : i, join = keep == j ? i : j;
    parent[join] = keep;
    size[keep] += size[join];
    if (size[keep] >= cluster_size) open[keep] = 0;
    return;
  }
  const int32_t a = ri < rj ? ri : rj, b = ri < rj ? rj : ri;
  if (hc_given(pi, pj, np, a, b)) return;
  const unsigned long long key = ((unsigned long long)(uint32_t)a << 32) | (uint32_t)b;
  if (!hc_seen_insert(seen, seen_mask, key, err)) return;
  const unsigned long long t = atomicAdd(ntasks, 1ULL);
  if ((int64_t)t >= cap) {
    atomicOr(err, 16);
    return;
  }
  T.s[t] = hc_jaccard<I>(rp, ci, a, b);
  T.i[t] = a;
  T.j[t] = b;
  next_live[atomicAdd(nnext, 1ULL)] = (int32_t)t;
}

// the found pairs (tasks np .. ntask - 1) into a new, larger set
__global__ void hc_seen_rebuild_kernel(Tasks T, int64_t np, int64_t ntask, unsigned long long* __restrict__ tab,
                                       uint64_t mask, int* __restrict__ err) {
  const int64_t t = np + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= ntask) return;
  const unsigned long long key = ((unsigned long long)(uint32_t)T.i[t] << 32) | (uint32_t)T.j[t];
  hc_seen_insert(tab, mask, key, err);
}

__global__ void hc_roots_kernel(const int32_t* __restrict__ parent, int64_t n, uint32_t* __restrict__ key,
                                int64_t* __restrict__ row, int* __restrict__ err) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  key[r] = (uint32_t)hc_find(parent, (int32_t)r, err);
  row[r] = r;
}

__global__ void hc_run_start_kernel(const uint32_t* __restrict__ skey, int64_t n, int64_t* __restrict__ flag) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r < n) flag[r] = (r == 0 || skey[r] != skey[r - 1]) ? 1 : 0;
}

__global__ void hc_offsets_kernel(const int64_t* __restrict__ flag, const int64_t* __restrict__ cid, int64_t n,
                                  int64_t* __restrict__ offsets) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r < n && flag[r]) offsets[cid[r] - 1] = r;
  if (r == 0) offsets[cid[n - 1]] = n;
}

int bits_for(int64_t v) {  // smallest b with 2^b > v
  int b = 1;
  while (b < 32 && ((int64_t)1 << b) <= v) ++b;
  return b;
}

template <typename I>
spops_status_t hc_device_t(Context* ctx, Matrix* A, const int64_t* pi, const int64_t* pj, const double* ps,
                           int64_t np, int64_t cluster_size, int64_t* perm_d, int64_t* offs_d, int64_t* ncl_out,
                           int64_t* rounds_out) {
  cudaStream_t st = ctx->stream;
  const int64_t n = A->rows;
  Trace tr("hc");
  // rows
  ArenaScope scope(ctx);  // this call's temporaries come from the arena
  PoolBuf parent(ctx), size(ctx), open(ctx), res(ctx), flags(ctx);
  const size_t nn = (size_t)std::max<int64_t>(n, 1);
  SPOPS_TRY(parent.alloc(nn * 4));
  SPOPS_TRY(size.alloc(nn * 4));
  SPOPS_TRY(open.alloc(nn));
  SPOPS_TRY(res.alloc(nn * 8));
  SPOPS_TRY(flags.alloc(64));
  SPOPS_CUDA(cudaMemsetAsync(flags.p, 0, 64, st));
  int* err = flags.as<int>();
  unsigned long long* ntasks = reinterpret_cast<unsigned long long*>(flags.as<char>() + 8);
  // live counts: cnt[cur] of the round about to run, cnt[cur ^ 1] of the next
  unsigned long long* cnt = reinterpret_cast<unsigned long long*>(flags.as<char>() + 16);
  if (n > 0) {
    hc_init_rows_kernel<<<hc_grid(n), 256, 0, st>>>(n, parent.as<int32_t>(), size.as<int32_t>(),
                                                    open.as<unsigned char>(), res.as<unsigned long long>());
    SPOPS_LAUNCH_CHECK();
  }
  // tasks: the initial pairs, then the pairs found while merging.  A round
  // creates at most one task per live task and never raises the live count,
  // so the live lists hold np entries and the task arrays grow (between
  // rounds) to ntask + nlive when needed; the set of found pairs grows with them.
  int64_t cap = np + n + 1;
  const size_t nl = (size_t)std::max<int64_t>(np, 1);
  PoolBuf ts(ctx), ti(ctx), tj(ctx), liveA(ctx), liveB(ctx), ri(ctx), rj(ctx), seen(ctx);
  SPOPS_TRY(ts.alloc((size_t)cap * 8));
  SPOPS_TRY(ti.alloc((size_t)cap * 4));
  SPOPS_TRY(tj.alloc((size_t)cap * 4));
  SPOPS_TRY(liveA.alloc(nl * 4));
  SPOPS_TRY(liveB.alloc(nl * 4));
  SPOPS_TRY(ri.alloc(nl * 4));
  SPOPS_TRY(rj.alloc(nl * 4));
  uint64_t seen_slots = 1;
  while (seen_slots < (uint64_t)(2 * cap)) seen_slots <<= 1;
  SPOPS_TRY(seen.alloc((size_t)seen_slots * 8));
  SPOPS_CUDA(cudaMemsetAsync(seen.p, 0xff, (size_t)seen_slots * 8, st));
  Tasks T{ts.as<double>(), ti.as<int32_t>(), tj.as<int32_t>()};
  int64_t ntask = np;
  if (np > 0) {
    hc_init_tasks_kernel<<<hc_grid(np), 256, 0, st>>>(pi, pj, ps, np, T, liveA.as<int32_t>());
    SPOPS_LAUNCH_CHECK();
  }
  const unsigned long long np_u[2] = {(unsigned long long)np, (unsigned long long)np};
  SPOPS_CUDA(cudaMemcpyAsync(ntasks, np_u, 16, cudaMemcpyHostToDevice, st));  // tasks made, cnt[0]
  tr.mark(st, "setup");
  // rounds, several per host synchronisation once few tasks are live: the
  // kernels read the live count on the device (grids sized by the last count
  // the host read, which no later round exceeds), and a round with no live
  // task does nothing
  int32_t* live = liveA.as<int32_t>();
  int32_t* next = liveB.as<int32_t>();
  int64_t nlive = np, rounds = 0;
  int cur = 0;
  uint64_t round_stamp = 0;  // below 2^32: the round bound keeps it there
  while (nlive > 0) {
    const int K = nlive > 65536 ? 1 : (int)std::min<int64_t>(16, std::max<int64_t>(1, 65536 / nlive));
    // every round retires at least one task, so rounds <= tasks ever made
    rounds += K;
    if (rounds > cap + 2 + 16) return fail(SPOPS_ERR_CUDA, "clustering: rounds did not end");
    if (ntask + (int64_t)K * nlive > cap) {  // room for these rounds' new tasks (at most one per live task each)
      const int64_t ncap = std::max<int64_t>(2 * cap, ntask + (int64_t)K * nlive + 1);
      if (ncap > (int64_t)INT32_MAX) return fail(SPOPS_ERR_UNSUPPORTED, "clustering: more than 2^31 tasks");
      PoolBuf ts2(ctx), ti2(ctx), tj2(ctx), seen2(ctx);
      SPOPS_TRY(ts2.alloc((size_t)ncap * 8));
      SPOPS_TRY(ti2.alloc((size_t)ncap * 4));
      SPOPS_TRY(tj2.alloc((size_t)ncap * 4));
      SPOPS_CUDA(cudaMemcpyAsync(ts2.p, ts.p, (size_t)ntask * 8, cudaMemcpyDeviceToDevice, st));
      SPOPS_CUDA(cudaMemcpyAsync(ti2.p, ti.p, (size_t)ntask * 4, cudaMemcpyDeviceToDevice, st));
      SPOPS_CUDA(cudaMemcpyAsync(tj2.p, tj.p, (size_t)ntask * 4, cudaMemcpyDeviceToDevice, st));
      uint64_t slots2 = seen_slots;
      while (slots2 < (uint64_t)(2 * ncap)) slots2 <<= 1;
      SPOPS_TRY(seen2.alloc((size_t)slots2 * 8));
      SPOPS_CUDA(cudaMemsetAsync(seen2.p, 0xff, (size_t)slots2 * 8, st));
      ts.swap(ts2);
      ti.swap(ti2);
      tj.swap(tj2);
      seen.swap(seen2);
      seen_slots = slots2;
      cap = ncap;
      T = Tasks{ts.as<double>(), ti.as<int32_t>(), tj.as<int32_t>()};
      if (ntask > np) {
        hc_seen_rebuild_kernel<<<hc_grid(ntask - np), 256, 0, st>>>(T, np, ntask, seen.as<unsigned long long>(),
                                                                     seen_slots - 1, err);
        SPOPS_LAUNCH_CHECK();
      }
    }
    const unsigned g = hc_grid(nlive);
    for (int r = 0; r < K; ++r) {
      const unsigned long long* nl_d = cnt + cur;
      const uint32_t stamp = (uint32_t)(++round_stamp);  // reservations of earlier rounds are stale
      hc_reserve_kernel<<<g, 256, 0, st>>>(live, nl_d, cnt + (cur ^ 1), stamp, T, parent.as<int32_t>(),
                                           open.as<unsigned char>(), res.as<unsigned long long>(), ri.as<int32_t>(),
                                           rj.as<int32_t>(), err);
      hc_commit_kernel<I><<<g, 256, 0, st>>>(live, nl_d, T, ri.as<int32_t>(), rj.as<int32_t>(),
                                             res.as<unsigned long long>(), stamp, parent.as<int32_t>(),
                                             size.as<int32_t>(), open.as<unsigned char>(), cluster_size,
                                             A->row.as<I>(), A->col.as<I>(), pi, pj, np,
                                             seen.as<unsigned long long>(), seen_slots - 1, cap, ntasks, next,
                                             cnt + (cur ^ 1), err);
      SPOPS_LAUNCH_CHECK();
      std::swap(live, next);
      cur ^= 1;
    }
    int herr = 0;
    unsigned long long hn[3] = {0, 0, 0};  // tasks made, cnt[0], cnt[1]
    SPOPS_CUDA(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaMemcpyAsync(hn, flags.as<char>() + 8, 24, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
    if (herr) return fail(SPOPS_ERR_CUDA, "clustering: device task error %d", herr);
    ntask = (int64_t)hn[0];
    nlive = (int64_t)hn[1 + cur];
    if (tr.on) {
      char what[64];
      std::snprintf(what, sizeof(what), "rounds to %lld: %lld live", (long long)rounds, (long long)nlive);
      tr.mark(st, what);
    }
  }
  if (tr.on) {
    char what[48];
    std::snprintf(what, sizeof(what), "merge rounds (%lld)", (long long)rounds);
    tr.mark(st, what);
  }
  // clusters by root row, rows ascending inside each
  PoolBuf key(ctx), skey(ctx), row(ctx), flag(ctx), cid(ctx), tmp(ctx);
  SPOPS_TRY(key.alloc(nn * 4));
  SPOPS_TRY(skey.alloc(nn * 4));
  SPOPS_TRY(row.alloc(nn * 8));
  SPOPS_TRY(flag.alloc(nn * 8));
  SPOPS_TRY(cid.alloc(nn * 8));
  int64_t ncl = 0;
  if (n > 0) {
    hc_roots_kernel<<<hc_grid(n), 256, 0, st>>>(parent.as<int32_t>(), n, key.as<uint32_t>(), row.as<int64_t>(), err);
    SPOPS_LAUNCH_CHECK();
    const int kb = bits_for(n);
    size_t c1 = 0, c2 = 0;
    SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, c1, key.as<uint32_t>(), skey.as<uint32_t>(), row.as<int64_t>(),
                                               perm_d, n, 0, kb, st));
    SPOPS_CUDA(cub::DeviceScan::InclusiveSum(nullptr, c2, flag.as<int64_t>(), cid.as<int64_t>(), n, st));
    SPOPS_TRY(tmp.alloc(std::max(c1, c2) + 256));
    SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, c1, key.as<uint32_t>(), skey.as<uint32_t>(), row.as<int64_t>(),
                                               perm_d, n, 0, kb, st));
    hc_run_start_kernel<<<hc_grid(n), 256, 0, st>>>(skey.as<uint32_t>(), n, flag.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
    SPOPS_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, c2, flag.as<int64_t>(), cid.as<int64_t>(), n, st));
    hc_offsets_kernel<<<hc_grid(n), 256, 0, st>>>(flag.as<int64_t>(), cid.as<int64_t>(), n, offs_d);
    SPOPS_LAUNCH_CHECK();
    SPOPS_CUDA(cudaMemcpyAsync(&ncl, cid.as<int64_t>() + n - 1, 8, cudaMemcpyDeviceToHost, st));
  } else {
    SPOPS_CUDA(cudaMemsetAsync(offs_d, 0, 8, st));
  }
  int herr = 0;
  SPOPS_CUDA(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  if (herr) return fail(SPOPS_ERR_CUDA, "clustering: device error %d", herr);
  tr.mark(st, "roots + order");
  *ncl_out = ncl;
  if (rounds_out) *rounds_out = rounds;
  return SPOPS_OK;
}

}  // namespace

spops_status_t hierarchical_clustering_device(Context* ctx, Matrix* A, const int64_t* pi, const int64_t* pj,
                                              const double* ps, int64_t np, int64_t cluster_size, int64_t* perm_d,
                                              int64_t* offs_d, int64_t* ncl_out, int64_t* rounds_out) {
  const int64_t n = A->rows;
  if (n > (int64_t)INT32_MAX - 1) return fail(SPOPS_ERR_UNSUPPORTED, "clustering: more than 2^31 rows");
  if (np > (int64_t)INT32_MAX / 2) return fail(SPOPS_ERR_UNSUPPORTED, "clustering: more than 2^30 pairs");
  cudaStream_t st = ctx->stream;
  int bad = 0;
  if (np > 0) {
    PoolBuf flag(ctx);
    SPOPS_TRY(flag.alloc(8));
    SPOPS_CUDA(cudaMemsetAsync(flag.p, 0, 8, st));
    hc_check_pairs_kernel<<<hc_grid(np), 256, 0, st>>>(pi, pj, np, n, flag.as<int>());
    SPOPS_LAUNCH_CHECK();
    SPOPS_CUDA(cudaMemcpyAsync(&bad, flag.p, 4, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
  }
  if (bad) {  // the host loop takes any pair list
    std::vector<int64_t> hpi((size_t)np), hpj((size_t)np), rp((size_t)n + 1), ci((size_t)A->nnz), perm, offs;
    std::vector<double> hps((size_t)np);
    SPOPS_CUDA(cudaMemcpy(hpi.data(), pi, (size_t)np * 8, cudaMemcpyDeviceToHost));
    SPOPS_CUDA(cudaMemcpy(hpj.data(), pj, (size_t)np * 8, cudaMemcpyDeviceToHost));
    SPOPS_CUDA(cudaMemcpy(hps.data(), ps, (size_t)np * 8, cudaMemcpyDeviceToHost));
    if (A->itype == SPOPS_INDEX_I64) {
      SPOPS_CUDA(cudaMemcpy(rp.data(), A->row.p, rp.size() * 8, cudaMemcpyDeviceToHost));
      if (A->nnz) SPOPS_CUDA(cudaMemcpy(ci.data(), A->col.p, ci.size() * 8, cudaMemcpyDeviceToHost));
    } else {
      std::vector<int32_t> r32(rp.size()), c32(ci.size());
      SPOPS_CUDA(cudaMemcpy(r32.data(), A->row.p, r32.size() * 4, cudaMemcpyDeviceToHost));
      if (A->nnz) SPOPS_CUDA(cudaMemcpy(c32.data(), A->col.p, c32.size() * 4, cudaMemcpyDeviceToHost));
      std::copy(r32.begin(), r32.end(), rp.begin());
      std::copy(c32.begin(), c32.end(), ci.begin());
    }
    SPOPS_TRY(hierarchical_clustering(rp.data(), ci.data(), n, hpi.data(), hpj.data(), hps.data(), np, cluster_size,
                                      perm, offs));
    SPOPS_CUDA(cudaMemcpy(perm_d, perm.data(), perm.size() * 8, cudaMemcpyHostToDevice));
    SPOPS_CUDA(cudaMemcpy(offs_d, offs.data(), offs.size() * 8, cudaMemcpyHostToDevice));
    *ncl_out = (int64_t)offs.size() - 1;
    if (rounds_out) *rounds_out = 0;
    return SPOPS_OK;
  }
  if (A->itype == SPOPS_INDEX_I64)
    return hc_device_t<int64_t>(ctx, A, pi, pj, ps, np, cluster_size, perm_d, offs_d, ncl_out, rounds_out);
  return hc_device_t<int32_t>(ctx, A, pi, pj, ps, np, cluster_size, perm_d, offs_d, ncl_out, rounds_out);
}

}  // namespace spops
