// C ABI: matrix handles and SpMV dispatch.
#include <cstring>

#include "spops_internal.h"

using namespace spops;

namespace {

spops_status_t check_types(spops_index_t it, spops_value_t vt) {
  if (it != SPOPS_INDEX_I32 && it != SPOPS_INDEX_I64) return fail(SPOPS_ERR_INVALID, "bad index type %d", (int)it);
  if (vt != SPOPS_VALUE_F32 && vt != SPOPS_VALUE_F64) return fail(SPOPS_ERR_INVALID, "bad value type %d", (int)vt);
  return SPOPS_OK;
}

// Place `bytes` of `src` in `dst`: borrow a device pointer or upload host data.
spops_status_t place(Context* ctx, DevBuf& dst, const void* src, size_t bytes, spops_mem_t mem) {
  if (bytes == 0) return dst.alloc(16);
  if (!src) return fail(SPOPS_ERR_INVALID, "null array of %zu bytes", bytes);
  if (mem == SPOPS_MEM_DEVICE) {
    dst.borrow(src, bytes);
    return SPOPS_OK;
  }
  SPOPS_TRY(dst.alloc(bytes));
  SPOPS_CUDA(cudaMemcpyAsync(dst.p, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
  return SPOPS_OK;
}

spops_status_t reserve_pinned(Context* c, size_t bytes) {
  if (c->pinned_bytes >= bytes) return SPOPS_OK;
  if (c->pinned) cudaFreeHost(c->pinned);
  c->pinned = nullptr;
  c->pinned_bytes = 0;
  SPOPS_CUDA(cudaMallocHost(&c->pinned, bytes));
  c->pinned_bytes = bytes;
  return SPOPS_OK;
}

}  // namespace

extern "C" {

spops_status_t spops_csr_create(spops_context_t ctx, spops_matrix_t* out, int64_t rows, int64_t cols, int64_t nnz,
                                const void* row_offset, const void* col_index, const void* values,
                                spops_index_t itype, spops_value_t vtype, spops_mem_t mem) {
  if (!ctx || !out) return fail(SPOPS_ERR_INVALID, "spops_csr_create: null context/output");
  if (rows < 0 || cols < 0 || nnz < 0) return fail(SPOPS_ERR_INVALID, "spops_csr_create: negative size");
  SPOPS_TRY(check_types(itype, vtype));
  if (itype == SPOPS_INDEX_I32 && (rows > INT32_MAX || cols > INT32_MAX || nnz > INT32_MAX))
    return fail(SPOPS_ERR_INVALID, "spops_csr_create: sizes exceed int32 indices");
  DeviceGuard g(ctx->device);
  spops_matrix_s* A = new spops_matrix_s();
  A->ctx = ctx;
  A->format = SPOPS_FMT_CSR;
  A->itype = itype;
  A->vtype = vtype;
  A->rows = rows;
  A->cols = cols;
  A->nnz = nnz;
  spops_status_t s = place(ctx, A->row, row_offset, (size_t)(rows + 1) * A->isize(), mem);
  if (s == SPOPS_OK) s = place(ctx, A->col, col_index, (size_t)nnz * A->isize(), mem);
  if (s == SPOPS_OK) s = place(ctx, A->val, values, (size_t)nnz * A->vsize(), mem);
  if (s != SPOPS_OK) {
    A->release_all();
    delete A;
    return s;
  }
  *out = A;
  return SPOPS_OK;
}

spops_status_t spops_matrix_destroy(spops_matrix_t A) {
  if (!A) return SPOPS_OK;
  DeviceGuard g(A->ctx->device);
  cudaStreamSynchronize(A->ctx->stream);
  A->release_all();
  delete A;
  return SPOPS_OK;
}

spops_status_t spops_matrix_info(spops_matrix_t A, spops_matrix_info_t* info) {
  if (!A || !info) return fail(SPOPS_ERR_INVALID, "spops_matrix_info: null argument");
  std::memset(info, 0, sizeof(*info));
  info->rows = A->rows;
  info->cols = A->cols;
  info->nnz = A->nnz;
  info->format = (int32_t)A->format;
  info->index_type = (int32_t)A->itype;
  info->value_type = (int32_t)A->vtype;
  info->layout = (int32_t)A->layout;
  return SPOPS_OK;
}

spops_status_t spops_matrix_touch(spops_matrix_t A) {
  if (!A) return fail(SPOPS_ERR_INVALID, "spops_matrix_touch: null matrix");
  return SPOPS_OK;  // the CSR plan depends on the pattern only
}

spops_status_t spops_matrix_analyse(spops_context_t ctx, spops_matrix_t A) {
  if (!ctx || !A) return fail(SPOPS_ERR_INVALID, "spops_matrix_analyse: null argument");
  DeviceGuard g(ctx->device);
  switch (A->format) {
    case SPOPS_FMT_CSR: return csr_analyse(ctx, A);
    default: return fail(SPOPS_ERR_UNSUPPORTED, "analysis for format %d", (int)A->format);
  }
}

spops_status_t spops_matrix_device_bytes(spops_matrix_t A, int64_t* bytes) {
  if (!A || !bytes) return fail(SPOPS_ERR_INVALID, "spops_matrix_device_bytes: null argument");
  auto own = [](const DevBuf& b) { return b.own ? (int64_t)b.bytes : 0; };
  const CsrPlan& P = A->plan;
  *bytes = own(A->row) + own(A->col) + own(A->val) + own(P.blk_row) + own(P.blk_chunk) + own(P.partial) +
           own(P.counter);
  return SPOPS_OK;
}

spops_status_t spops_spmv(spops_context_t ctx, double alpha, spops_matrix_t A, const void* x, double beta, void* y) {
  if (!ctx || !A) return fail(SPOPS_ERR_INVALID, "spops_spmv: null context/matrix");
  if ((!x && A->cols > 0) || (!y && A->rows > 0)) return fail(SPOPS_ERR_INVALID, "spops_spmv: null vector");
  DeviceGuard g(ctx->device);
  switch (A->format) {
    case SPOPS_FMT_CSR: return csr_spmv(ctx, A, alpha, x, beta, y);
    default: return fail(SPOPS_ERR_UNSUPPORTED, "SpMV for format %d", (int)A->format);
  }
}

spops_status_t spops_spmv_host(spops_context_t ctx, double alpha, spops_matrix_t A, const void* x_host,
                               double beta, void* y_host) {
  if (!ctx || !A) return fail(SPOPS_ERR_INVALID, "spops_spmv_host: null context/matrix");
  DeviceGuard g(ctx->device);
  const size_t xb = (size_t)A->cols * A->vsize(), yb = (size_t)A->rows * A->vsize();
  if (ctx->xbuf.bytes < xb) SPOPS_TRY(ctx->xbuf.alloc(xb));
  if (ctx->ybuf.bytes < yb) SPOPS_TRY(ctx->ybuf.alloc(yb));
  cudaStream_t st = ctx->stream;
  if (xb) SPOPS_CUDA(cudaMemcpyAsync(ctx->xbuf.p, x_host, xb, cudaMemcpyHostToDevice, st));
  if (beta != 0.0 && yb) SPOPS_CUDA(cudaMemcpyAsync(ctx->ybuf.p, y_host, yb, cudaMemcpyHostToDevice, st));
  SPOPS_TRY(spops_spmv(ctx, alpha, A, ctx->xbuf.p, beta, ctx->ybuf.p));
  if (yb) SPOPS_CUDA(cudaMemcpyAsync(y_host, ctx->ybuf.p, yb, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  (void)reserve_pinned;
  return SPOPS_OK;
}

}  // extern "C"
