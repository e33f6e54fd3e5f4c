// Context, error reporting and device buffers behind the C ABI.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "spops_internal.h"

namespace spops {

namespace {
thread_local char g_err[1024] = "";
}

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

spops_status_t fail(spops_status_t s, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return s;
}

spops_status_t cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
  const char* base = strrchr(file, '/');
  set_error("%s failed: %s (%s:%d)", what, cudaGetErrorString(e), base ? base + 1 : file, line);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();  // clear the sticky-free allocation error
    return SPOPS_ERR_ALLOC;
  }
  return SPOPS_ERR_CUDA;
}

spops_status_t DevBuf::alloc(size_t n) {
  release();
  if (n == 0) n = 16;
  cudaError_t e = cudaMalloc(&p, n);
  if (e != cudaSuccess) {
    p = nullptr;
    bytes = 0;
    return cuda_fail(e, "cudaMalloc", __FILE__, __LINE__);
  }
  bytes = n;
  own = true;
  return SPOPS_OK;
}

void DevBuf::release() {
  if (own && p) {
    if (home) home->cache_block(p, bytes);
    else cudaFree(p);
  }
  p = nullptr;
  bytes = 0;
  own = false;
  home = nullptr;
}

constexpr size_t kCacheMin = size_t(1) << 20;   // blocks below this go back to the driver
constexpr size_t kCacheMax = size_t(24) << 30;  // bytes the cache may hold

spops_status_t DevBuf::alloc_cached(Context* ctx, size_t n) {
  release();
  if (n == 0) n = 16;
  static const bool trace = [] {
    const char* e = std::getenv("SPOPS_TRACE");
    return e && (e[0] == '1' || e[0] == '2');
  }();
  if (n >= kCacheMin) {
    void* q = nullptr;
    size_t b = 0;
    if (ctx->take_block(n, &q, &b)) {
      if (trace) std::fprintf(stderr, "[cache] %zu bytes from a cached block of %zu\n", n, b);
      p = q;
      bytes = b;
      own = true;
      home = ctx;
      return SPOPS_OK;
    }
    if (trace)
      std::fprintf(stderr, "[cache] %zu bytes: no cached block (%zu blocks, %zu bytes held)\n", n,
                   ctx->block_cache.size(), ctx->block_cache_bytes);
  }
  SPOPS_TRY(alloc(n));
  if (n >= kCacheMin) home = ctx;
  return SPOPS_OK;
}

void Context::cache_block(void* q, size_t b) {
  if (b < kCacheMin || block_cache_bytes + b > kCacheMax) {
    cudaFree(q);
    return;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventRecord(e, stream) != cudaSuccess) {  // cannot order a reuse: give it back
    if (e) cudaEventDestroy(e);
    cudaGetLastError();
    cudaFree(q);
    return;
  }
  block_cache.push_back(CachedBlock{q, b, e});
  block_cache_bytes += b;
}

bool Context::take_block(size_t n, void** q, size_t* b) {
  // the smallest block of at least n bytes and at most n + n / 8 + 2 MB
  const size_t hi = n + n / 8 + (size_t(2) << 20);
  int best = -1;
  for (int i = 0; i < (int)block_cache.size(); ++i) {
    const size_t s = block_cache[i].bytes;
    if (s >= n && s <= hi && (best < 0 || s < block_cache[best].bytes)) best = i;
  }
  if (best < 0) return false;
  const CachedBlock c = block_cache[best];
  block_cache.erase(block_cache.begin() + best);
  block_cache_bytes -= c.bytes;
  cudaStreamWaitEvent(stream, c.done, 0);  // work queued before the release may still use it
  cudaEventDestroy(c.done);
  *q = c.p;
  *b = c.bytes;
  return true;
}

void Context::drop_block_cache() {
  for (const CachedBlock& c : block_cache) {
    cudaEventSynchronize(c.done);
    cudaEventDestroy(c.done);
    cudaFree(c.p);
  }
  block_cache.clear();
  block_cache_bytes = 0;
}

spops_status_t Context::pool_alloc(void** out, size_t bytes) {
  if (!pool) {
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    SPOPS_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = ~0ULL;  // never trim on synchronisation: the next call reuses the memory
    SPOPS_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  }
  static const int trace = [] {  // SPOPS_TRACE=2: time every pool allocation
    const char* e = std::getenv("SPOPS_TRACE");
    return e && e[0] == '2' ? 2 : 0;
  }();
  if (trace == 2) {
    cudaStreamSynchronize(stream);
    const auto t0 = std::chrono::steady_clock::now();
    SPOPS_CUDA(cudaMallocFromPoolAsync(out, bytes, pool, stream));
    const auto t1 = std::chrono::steady_clock::now();
    cudaStreamSynchronize(stream);
    const auto t2 = std::chrono::steady_clock::now();
    std::fprintf(stderr, "[pool] %12zu bytes: call %.3f ms, stream %.3f ms\n", bytes,
                 std::chrono::duration<double, std::milli>(t1 - t0).count(),
                 std::chrono::duration<double, std::milli>(t2 - t1).count());
    return SPOPS_OK;
  }
  SPOPS_CUDA(cudaMallocFromPoolAsync(out, bytes, pool, stream));
  return SPOPS_OK;
}

void Context::pool_free(void* q) {
  if (q) cudaFreeAsync(q, stream);
}

ArenaScope::ArenaScope(Context* c) : ctx(c) {
  if (ctx->arena_depth++ > 0) {
    mark = ctx->arena_top;
    return;
  }
  // the last scope's work on another stream may still read the arena
  if (ctx->arena_done && ctx->arena_stream != ctx->stream) cudaStreamWaitEvent(ctx->stream, ctx->arena_done, 0);
  if (ctx->arena_need > ctx->arena.bytes) {  // regrow to what the earlier scopes needed
    const size_t want = ((ctx->arena_need + ctx->arena_need / 8) + (size_t(2) << 20) - 1) & ~((size_t(2) << 20) - 1);
    cudaDeviceSynchronize();  // queued work may still read the old arena
    ctx->arena.release();
    if (ctx->arena.alloc(want) != SPOPS_OK) {  // no room: temporaries keep coming from the pool
      ctx->arena.release();
      cudaGetLastError();
    }
    ctx->arena_need = 0;
  }
  ctx->arena_top = 0;
  ctx->arena_over = 0;
  mark = 0;
}

ArenaScope::~ArenaScope() {
  ctx->arena_top = mark;
  if (--ctx->arena_depth > 0) return;
  if (!ctx->arena_done) cudaEventCreateWithFlags(&ctx->arena_done, cudaEventDisableTiming);
  if (ctx->arena_done) cudaEventRecord(ctx->arena_done, ctx->stream);
  ctx->arena_stream = ctx->stream;
}

spops_status_t Context::scratch_reserve(size_t n) {
  if (scratch.bytes >= n && scratch.p) return SPOPS_OK;
  // work queued on the stream may still read the old scratch
  SPOPS_CUDA(cudaStreamSynchronize(stream));
  size_t want = n + n / 4 + 4096;
  return scratch.alloc(want);
}

spops_status_t Context::ensure_errword() {
  if (errword.p) return SPOPS_OK;
  SPOPS_TRY(errword.alloc(16));
  SPOPS_CUDA(cudaMemsetAsync(errword.p, 0, 16, stream));
  return SPOPS_OK;
}

}  // namespace spops

using namespace spops;

extern "C" {

const char* spops_last_error(void) { return g_err; }

int spops_abi_version(void) { return SPOPS_ABI_VERSION; }

const char* spops_status_string(spops_status_t s) {
  switch (s) {
    case SPOPS_OK: return "SPOPS_OK";
    case SPOPS_ERR_INVALID: return "SPOPS_ERR_INVALID";
    case SPOPS_ERR_UNSUPPORTED: return "SPOPS_ERR_UNSUPPORTED";
    case SPOPS_ERR_ALLOC: return "SPOPS_ERR_ALLOC";
    case SPOPS_ERR_CUDA: return "SPOPS_ERR_CUDA";
    case SPOPS_ERR_TOO_LARGE: return "SPOPS_ERR_TOO_LARGE";
    case SPOPS_ERR_TIMEOUT: return "SPOPS_ERR_TIMEOUT";
  }
  return "SPOPS_ERR_UNKNOWN";
}

spops_status_t spops_create(spops_context_t* out, int device, void* stream) {
  if (!out) return fail(SPOPS_ERR_INVALID, "spops_create: null output");
  int ndev = 0;
  SPOPS_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(SPOPS_ERR_INVALID, "spops_create: device %d of %d", device, ndev);
  DeviceGuard g(device);
  spops_context_s* c = new spops_context_s();
  c->device = device;
  c->stream = static_cast<cudaStream_t>(stream);
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
  *out = c;
  return SPOPS_OK;
}

spops_status_t spops_destroy(spops_context_t c) {
  if (!c) return SPOPS_OK;
  DeviceGuard g(c->device);
  cudaStreamSynchronize(c->stream);
  if (c->in_stream) cudaStreamSynchronize(c->in_stream);
  if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
  c->scratch.release();
  c->errword.release();
  c->xbuf.release();
  c->ybuf.release();
  for (cudaEvent_t e : c->part_events) cudaEventDestroy(e);
  c->part_events.clear();
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  c->copy_stream = nullptr;
  if (c->pinned) cudaFreeHost(c->pinned);
  for (int i = 0; i < 2; ++i) {
    c->axbuf[i].release();
    c->aybuf[i].release();
    for (cudaEvent_t e : {c->a_in[i], c->a_read[i], c->a_out[i]})
      if (e) cudaEventDestroy(e);
  }
  if (c->in_stream) cudaStreamDestroy(c->in_stream);
  for (cudaEvent_t e : c->file_events) cudaEventDestroy(e);
  for (void* b : c->file_stage) cudaFreeHost(b);
  if (c->arena_done) {
    cudaEventSynchronize(c->arena_done);
    cudaEventDestroy(c->arena_done);
  }
  c->arena.release();
  c->drop_block_cache();
  if (c->pool) {
    cudaStreamSynchronize(c->stream);
    cudaMemPoolDestroy(c->pool);
  }
  delete c;
  return SPOPS_OK;
}

spops_status_t spops_set_stream(spops_context_t c, void* stream) {
  if (!c) return fail(SPOPS_ERR_INVALID, "spops_set_stream: null context");
  c->stream = static_cast<cudaStream_t>(stream);
  return SPOPS_OK;
}

spops_status_t spops_check_device(spops_context_t c, int32_t* flags) {
  if (!c) return fail(SPOPS_ERR_INVALID, "spops_check_device: null context");
  DeviceGuard g(c->device);
  int32_t f = 0;
  if (c->errword.p) {
    SPOPS_CUDA(cudaMemcpyAsync(&f, c->errword.p, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    SPOPS_CUDA(cudaStreamSynchronize(c->stream));
    if (f) SPOPS_CUDA(cudaMemsetAsync(c->errword.p, 0, sizeof(int32_t), c->stream));
  }
  if (flags) *flags = f;
  if (f) return fail(SPOPS_ERR_TIMEOUT, "a device-side wait gave up (flags 0x%x)", (unsigned)f);
  return SPOPS_OK;
}

spops_status_t spops_set_option(spops_context_t c, const char* key, int64_t value) {
  if (!c || !key) return fail(SPOPS_ERR_INVALID, "spops_set_option: null argument");
  if (!strcmp(key, "csr_variant")) {
    if (value < 0 || value > 10) return fail(SPOPS_ERR_INVALID, "csr_variant must be 0..10");
    c->csr_variant = (int)value;
    return SPOPS_OK;
  }
  if (!strcmp(key, "sell_order")) {
    if (value < 0 || value > 1) return fail(SPOPS_ERR_INVALID, "sell_order must be 0 or 1");
    c->sell_order = (int)value;
    return SPOPS_OK;
  }
  if (!strcmp(key, "sell_tails")) {
    if (value < 0 || value > 1) return fail(SPOPS_ERR_INVALID, "sell_tails must be 0 or 1");
    c->sell_tails = (int)value;
    return SPOPS_OK;
  }
  if (!strcmp(key, "adjoint_bands")) {
    if (value < 0 || value > TransposeData::kMaxBands)
      return fail(SPOPS_ERR_INVALID, "adjoint_bands must be 0 (automatic) or 1 .. %d", TransposeData::kMaxBands);
    c->adjoint_bands = (int)value;
    return SPOPS_OK;
  }
  if (!strcmp(key, "batch_band")) {
    if (value < 0 || value > 1) return fail(SPOPS_ERR_INVALID, "batch_band must be 0 or 1");
    c->batch_band = (int)value;
    return SPOPS_OK;
  }
  return fail(SPOPS_ERR_INVALID, "spops_set_option: unknown key '%s'", key);
}

spops_status_t spops_synchronize(spops_context_t c) {
  if (!c) return fail(SPOPS_ERR_INVALID, "spops_synchronize: null context");
  DeviceGuard g(c->device);
  SPOPS_CUDA(cudaStreamSynchronize(c->stream));
  return SPOPS_OK;
}

}  // extern "C"
