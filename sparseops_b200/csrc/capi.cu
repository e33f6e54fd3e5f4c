// C ABI: matrix handles and SpMV dispatch.
#include <cstring>
#include <vector>

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

spops_status_t cuda_copy_to_host(Context* ctx, void* dst, const void* src, size_t bytes) {
  if (bytes == 0) return SPOPS_OK;
  SPOPS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  SPOPS_CUDA(cudaStreamSynchronize(ctx->stream));
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

spops_status_t spops_coo_create(spops_context_t ctx, spops_matrix_t* out, int64_t rows, int64_t cols, int64_t nnz,
                                const void* row_index, const void* col_index, const void* values,
                                spops_index_t itype, spops_value_t vtype, spops_mem_t mem) {
  if (!ctx || !out) return fail(SPOPS_ERR_INVALID, "spops_coo_create: null context/output");
  if (rows < 0 || cols < 0 || nnz < 0) return fail(SPOPS_ERR_INVALID, "spops_coo_create: negative size");
  SPOPS_TRY(check_types(itype, vtype));
  DeviceGuard g(ctx->device);
  spops_matrix_s* A = new spops_matrix_s();
  A->ctx = ctx;
  A->format = SPOPS_FMT_COO;
  A->itype = itype;
  A->vtype = vtype;
  A->rows = rows;
  A->cols = cols;
  A->nnz = nnz;
  spops_status_t s = place(ctx, A->row, row_index, (size_t)nnz * A->isize(), mem);
  if (s == SPOPS_OK) s = place(ctx, A->col, col_index, (size_t)nnz * A->isize(), mem);
  if (s == SPOPS_OK) s = place(ctx, A->val, values, (size_t)nnz * A->vsize(), mem);
  if (s == SPOPS_OK) s = coo_analyse(ctx, A);
  if (s != SPOPS_OK) {
    A->release_all();
    delete A;
    return s;
  }
  *out = A;
  return SPOPS_OK;
}

spops_status_t spops_convert(spops_context_t ctx, spops_matrix_t csr, spops_format_t format,
                             const spops_format_params_t* params, spops_matrix_t* out) {
  if (!ctx || !csr || !out) return fail(SPOPS_ERR_INVALID, "spops_convert: null argument");
  DeviceGuard g(ctx->device);
  spops_format_params_t p;
  std::memset(&p, 0, sizeof(p));
  if (params) p = *params;
  Matrix* M = nullptr;
  SPOPS_TRY(convert_from_csr(ctx, csr, format, p, &M));
  *out = static_cast<spops_matrix_s*>(M);
  return SPOPS_OK;
}

spops_status_t spops_padded_create(spops_context_t ctx, spops_matrix_t* out, spops_format_t format, int64_t rows,
                                   int64_t cols, int64_t nnz, int64_t chunk, int64_t sigma, int64_t alignment,
                                   spops_layout_t layout, const void* reorder, const void* chunk_len,
                                   int64_t nchunks, const void* col, const void* val, int64_t stored,
                                   spops_index_t itype, spops_value_t vtype, spops_mem_t mem) {
  if (!ctx || !out) return fail(SPOPS_ERR_INVALID, "spops_padded_create: null context/output");
  if (format != SPOPS_FMT_SELL_C_SIGMA && format != SPOPS_FMT_SELL_C_R && format != SPOPS_FMT_SELL &&
      format != SPOPS_FMT_ELL)
    return fail(SPOPS_ERR_INVALID, "spops_padded_create: format %d is not a padded-row format", (int)format);
  if (rows < 0 || cols < 0 || stored < 0 || chunk <= 0) return fail(SPOPS_ERR_INVALID, "spops_padded_create: sizes");
  if (nchunks != (rows + chunk - 1) / chunk) return fail(SPOPS_ERR_INVALID, "spops_padded_create: nchunks");
  const bool sorted = format == SPOPS_FMT_SELL_C_SIGMA || format == SPOPS_FMT_SELL_C_R;
  if (sorted && !reorder && rows > 0) return fail(SPOPS_ERR_INVALID, "spops_padded_create: reorder required");
  SPOPS_TRY(check_types(itype, vtype));
  DeviceGuard g(ctx->device);
  spops_matrix_s* A = new spops_matrix_s();
  A->ctx = ctx;
  A->format = format;
  A->itype = itype;
  A->vtype = vtype;
  A->layout = layout == SPOPS_COL_MAJOR ? SPOPS_COL_MAJOR : SPOPS_ROW_MAJOR;
  A->rows = rows;
  A->cols = cols;
  A->nnz = nnz;
  PaddedData& P = A->pad;
  P.C = chunk;
  P.sigma = sigma;
  P.align = alignment > 0 ? alignment : 1;
  P.nchunks = nchunks;
  P.stored = stored;
  P.sorted = sorted;
  spops_status_t s = SPOPS_OK;
  if (sorted) s = place(ctx, P.reorder, reorder, (size_t)rows * A->isize(), mem);
  if (s == SPOPS_OK) s = place(ctx, P.chunk_len, chunk_len, (size_t)nchunks * A->isize(), mem);
  if (s == SPOPS_OK) s = place(ctx, A->col, col, (size_t)stored * A->isize(), mem);
  if (s == SPOPS_OK) s = place(ctx, A->val, val, (size_t)stored * A->vsize(), mem);
  if (s == SPOPS_OK) s = validate_columns(ctx, A->col.p, stored, itype, cols, true);
  if (s == SPOPS_OK && sorted) s = validate_columns(ctx, P.reorder.p, rows, itype, rows, false);
  if (s == SPOPS_OK) {
    // chunk offsets from the chunk widths (host scan of nchunks values)
    std::vector<int64_t> len((size_t)nchunks), off((size_t)nchunks + 1, 0);
    if (nchunks > 0) {
      if (itype == SPOPS_INDEX_I32) {
        std::vector<int32_t> tmp((size_t)nchunks);
        s = cuda_copy_to_host(ctx, tmp.data(), P.chunk_len.p, tmp.size() * 4);
        for (int64_t c = 0; c < nchunks; ++c) len[c] = tmp[c];
      } else {
        s = cuda_copy_to_host(ctx, len.data(), P.chunk_len.p, len.size() * 8);
      }
    }
    for (int64_t c = 0; s == SPOPS_OK && c < nchunks; ++c) {
      if (len[c] < 0) s = fail(SPOPS_ERR_INVALID, "negative chunk width");
      off[c + 1] = off[c] + len[c] * chunk;
    }
    if (s == SPOPS_OK && off[nchunks] != stored)
      s = fail(SPOPS_ERR_INVALID, "chunk widths x C (%lld) differ from stored (%lld)", (long long)off[nchunks],
               (long long)stored);
    if (s == SPOPS_OK) s = P.chunk_off.alloc(off.size() * sizeof(int64_t));
    if (s == SPOPS_OK) {
      cudaError_t e = cudaMemcpyAsync(P.chunk_off.p, off.data(), off.size() * 8, cudaMemcpyHostToDevice, ctx->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
      if (e != cudaSuccess) s = cuda_fail(e, "upload chunk offsets", __FILE__, __LINE__);
    }
  }
  if (s == SPOPS_OK) s = padded_finish(ctx, A);
  if (s != SPOPS_OK) {
    A->release_all();
    delete A;
    return s;
  }
  *out = A;
  return SPOPS_OK;
}

spops_status_t spops_dia_create(spops_context_t ctx, spops_matrix_t* out, int64_t rows, int64_t cols, int64_t nnz,
                                int64_t ndiag, int64_t stride, const int64_t* diag_offsets, const void* diag_data,
                                spops_value_t vtype, spops_mem_t mem) {
  if (!ctx || !out) return fail(SPOPS_ERR_INVALID, "spops_dia_create: null context/output");
  if (rows < 0 || cols < 0 || ndiag < 0 || stride < rows) return fail(SPOPS_ERR_INVALID, "spops_dia_create: sizes");
  SPOPS_TRY(check_types(SPOPS_INDEX_I64, vtype));
  DeviceGuard g(ctx->device);
  spops_matrix_s* A = new spops_matrix_s();
  A->ctx = ctx;
  A->format = SPOPS_FMT_DIA;
  A->itype = SPOPS_INDEX_I64;
  A->vtype = vtype;
  A->rows = rows;
  A->cols = cols;
  A->nnz = nnz;
  A->dia.ndiag = ndiag;
  A->dia.stride = stride;
  spops_status_t s = place(ctx, A->dia.offsets, diag_offsets, (size_t)ndiag * 8, mem);
  if (s == SPOPS_OK) s = place(ctx, A->dia.data, diag_data, (size_t)ndiag * stride * A->vsize(), mem);
  if (s != SPOPS_OK) {
    A->release_all();
    delete A;
    return s;
  }
  *out = A;
  return SPOPS_OK;
}

spops_status_t spops_bsr_create(spops_context_t ctx, spops_matrix_t* out, int64_t rows, int64_t cols, int64_t nnz,
                                int64_t block_rows, int64_t block_cols, int64_t nnzb, const void* row_ptr,
                                const void* block_col, const void* block_data, spops_index_t itype,
                                spops_value_t vtype, spops_mem_t mem) {
  if (!ctx || !out) return fail(SPOPS_ERR_INVALID, "spops_bsr_create: null context/output");
  if (rows < 0 || cols < 0 || block_rows <= 0 || block_cols <= 0 || nnzb < 0)
    return fail(SPOPS_ERR_INVALID, "spops_bsr_create: sizes");
  if (block_rows * block_cols > 1024) return fail(SPOPS_ERR_UNSUPPORTED, "BSR blocks larger than 1024 elements");
  SPOPS_TRY(check_types(itype, vtype));
  DeviceGuard g(ctx->device);
  spops_matrix_s* A = new spops_matrix_s();
  A->ctx = ctx;
  A->format = SPOPS_FMT_BSR;
  A->itype = itype;
  A->vtype = vtype;
  A->rows = rows;
  A->cols = cols;
  A->nnz = nnz;
  BsrData& B = A->bsr;
  B.br = block_rows;
  B.bc = block_cols;
  B.mb = (rows + block_rows - 1) / block_rows;
  B.nb = (cols + block_cols - 1) / block_cols;
  B.nnzb = nnzb;
  spops_status_t s = place(ctx, B.row_ptr, row_ptr, (size_t)(B.mb + 1) * A->isize(), mem);
  if (s == SPOPS_OK) s = place(ctx, B.bcol, block_col, (size_t)nnzb * A->isize(), mem);
  if (s == SPOPS_OK) s = place(ctx, B.data, block_data, (size_t)nnzb * block_rows * block_cols * A->vsize(), mem);
  if (s == SPOPS_OK) s = validate_columns(ctx, B.bcol.p, nnzb, itype, B.nb, false);
  if (s != SPOPS_OK) {
    A->release_all();
    delete A;
    return s;
  }
  *out = A;
  return SPOPS_OK;
}

spops_status_t spops_matrix_array(spops_matrix_t A, spops_array_t which, const void** dev_ptr, int64_t* count,
                                  int32_t* elem_bytes) {
  if (!A) return fail(SPOPS_ERR_INVALID, "spops_matrix_array: null matrix");
  const void* p = nullptr;
  int64_t n = 0;
  int32_t eb = 0;
  const int32_t is = (int32_t)A->isize(), vs = (int32_t)A->vsize();
  switch (which) {
    case SPOPS_ARR_ROW:
      p = A->row.p; eb = is;
      n = A->format == SPOPS_FMT_CSR ? A->rows + 1 : A->format == SPOPS_FMT_COO ? A->nnz
          : A->format == SPOPS_FMT_VLCLUSTER ? A->clusters + 1 : 0;
      break;
    case SPOPS_ARR_COL:
      p = A->col.p; eb = is;
      n = (A->format == SPOPS_FMT_CSR || A->format == SPOPS_FMT_COO || A->format == SPOPS_FMT_VLCLUSTER) ? A->nnz
                                                                                                     : A->pad.stored;
      break;
    case SPOPS_ARR_VAL:
      eb = vs;
      if (A->format == SPOPS_FMT_DIA) { p = A->dia.data.p; n = A->dia.ndiag * A->dia.stride; }
      else if (A->format == SPOPS_FMT_VLCLUSTER) { p = A->val.p; n = A->cl_nnzv; }
      else if (A->format == SPOPS_FMT_BSR) { p = A->bsr.data.p; n = A->bsr.nnzb * A->bsr.br * A->bsr.bc; }
      else { p = A->val.p; n = (A->format == SPOPS_FMT_CSR || A->format == SPOPS_FMT_COO) ? A->nnz : A->pad.stored; }
      break;
    case SPOPS_ARR_REORDER: p = A->pad.reorder.p; eb = is; n = A->pad.sorted ? A->rows : 0; break;
    case SPOPS_ARR_CHUNK_LEN: p = A->pad.chunk_len.p; eb = is; n = A->pad.nchunks; break;
    case SPOPS_ARR_CHUNK_OFF: p = A->pad.chunk_off.p; eb = 8; n = A->pad.chunk_off.p ? A->pad.nchunks + 1 : 0; break;
    case SPOPS_ARR_ROW_LEN: p = A->pad.row_len.p; eb = 4; n = A->pad.row_len.p ? A->rows : 0; break;
    case SPOPS_ARR_DIAG_OFFSETS: p = A->dia.offsets.p; eb = 8; n = A->dia.ndiag; break;
    case SPOPS_ARR_BLOCK_ROW_PTR: p = A->bsr.row_ptr.p; eb = is; n = A->bsr.row_ptr.p ? A->bsr.mb + 1 : 0; break;
    case SPOPS_ARR_BLOCK_COL: p = A->bsr.bcol.p; eb = is; n = A->bsr.nnzb; break;
    case SPOPS_ARR_TILE_PTR: p = A->csr5.tile_ptr.p; eb = 4; n = A->csr5.tile_ptr.p ? A->csr5.tiles + 1 : 0; break;
    case SPOPS_ARR_TILE_DESC: p = A->csr5.desc.p; eb = 4; n = A->csr5.tiles * 32; break;
    case SPOPS_ARR_CLUSTER_SZ: p = A->cl_sz.p; eb = is; n = A->format == SPOPS_FMT_VLCLUSTER ? A->clusters : 0; break;
    case SPOPS_ARR_ROWPTR_VAL:
      p = A->cl_rpv.p; eb = is; n = A->format == SPOPS_FMT_VLCLUSTER ? A->clusters + 1 : 0;
      break;
    default: return fail(SPOPS_ERR_INVALID, "spops_matrix_array: unknown array %d", (int)which);
  }
  if (n > 0 && !p) return fail(SPOPS_ERR_INVALID, "spops_matrix_array: array %d not present", (int)which);
  if (dev_ptr) *dev_ptr = p;
  if (count) *count = n;
  if (elem_bytes) *elem_bytes = eb;
  return SPOPS_OK;
}

spops_status_t spops_matrix_download(spops_context_t ctx, spops_matrix_t A, spops_array_t which, void* host_dst,
                                     int64_t count) {
  if (!ctx || !A) return fail(SPOPS_ERR_INVALID, "spops_matrix_download: null argument");
  const void* p = nullptr;
  int64_t n = 0;
  int32_t eb = 0;
  SPOPS_TRY(spops_matrix_array(A, which, &p, &n, &eb));
  if (count < 0 || count > n) return fail(SPOPS_ERR_INVALID, "spops_matrix_download: count %lld > %lld",
                                          (long long)count, (long long)n);
  if (count == 0) return SPOPS_OK;
  if (!host_dst) return fail(SPOPS_ERR_INVALID, "spops_matrix_download: null destination");
  DeviceGuard g(ctx->device);
  return cuda_copy_to_host(ctx, host_dst, p, (size_t)count * eb);
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
  const PaddedData& P = A->pad;
  switch (A->format) {
    case SPOPS_FMT_SELL_C_SIGMA: {
      info->sigma = P.sigma; info->chunk = P.C; info->alignment = P.align;
      const int64_t nslice = P.sigma > 0 ? (A->rows + P.sigma - 1) / P.sigma : 0;
      const int64_t per = P.C > 0 ? P.sigma / P.C : 0;
      info->extra[0] = nslice; info->extra[1] = nslice * per; info->extra[2] = P.nchunks;
      info->extra[3] = per; info->extra[4] = P.stored;
      break;
    }
    case SPOPS_FMT_SELL_C_R:
    case SPOPS_FMT_SELL:
      info->sigma = P.sigma; info->chunk = P.C; info->alignment = P.align;
      info->extra[0] = P.nchunks; info->extra[1] = P.stored;
      break;
    case SPOPS_FMT_ELL:
      info->chunk = P.C; info->extra[0] = P.max_row; info->extra[1] = P.min_row;
      break;
    case SPOPS_FMT_DIA: info->extra[0] = A->dia.ndiag; info->extra[1] = A->dia.stride; break;
    case SPOPS_FMT_BSR:
      info->extra[0] = A->bsr.mb; info->extra[1] = A->bsr.nb; info->extra[2] = A->bsr.nnzb;
      info->extra[3] = A->bsr.br; info->extra[4] = A->bsr.bc;
      break;
    case SPOPS_FMT_CSR5:
      info->extra[0] = A->csr5.tiles; info->extra[1] = 32; info->extra[2] = 16; info->extra[3] = A->csr5.nempty;
      break;
    case SPOPS_FMT_VLCLUSTER:
      info->extra[0] = A->clusters; info->extra[1] = A->cl_nnzv; info->extra[2] = A->cl_max_sz;
      break;
    default: break;
  }
  return SPOPS_OK;
}

spops_status_t spops_matrix_touch(spops_matrix_t A) {
  if (!A) return fail(SPOPS_ERR_INVALID, "spops_matrix_touch: null matrix");
  A->tr.values_fresh = false;  // the row-ordered CSR plans depend on the pattern only
  A->plan.win.values_fresh = false;  // the window plan keeps a copy of the values
  A->pad.tails_fresh = false;        // the padded tails keep a copy of the values
  return SPOPS_OK;
}

spops_status_t spops_csr_set_values(spops_matrix_t A, const void* values) {
  if (!A) return fail(SPOPS_ERR_INVALID, "spops_csr_set_values: null matrix");
  if (A->format != SPOPS_FMT_CSR) return fail(SPOPS_ERR_INVALID, "spops_csr_set_values: not a CSR matrix");
  if (!values && A->nnz > 0) return fail(SPOPS_ERR_INVALID, "spops_csr_set_values: null values");
  A->val.borrow(values, (size_t)A->nnz * A->vsize());
  A->tr.values_fresh = false;
  A->plan.win.values_fresh = false;
  return SPOPS_OK;
}

spops_status_t spops_csr_upload_values(spops_context_t ctx, spops_matrix_t A, const void* host_values) {
  if (!ctx || !A) return fail(SPOPS_ERR_INVALID, "spops_csr_upload_values: null context/matrix");
  if (A->format != SPOPS_FMT_CSR) return fail(SPOPS_ERR_INVALID, "spops_csr_upload_values: not a CSR matrix");
  if (!A->val.own) return fail(SPOPS_ERR_INVALID, "spops_csr_upload_values: the handle borrows its values");
  if (A->nnz == 0) return SPOPS_OK;
  if (!host_values) return fail(SPOPS_ERR_INVALID, "spops_csr_upload_values: null values");
  DeviceGuard g(ctx->device);
  SPOPS_CUDA(cudaMemcpyAsync(A->val.p, host_values, (size_t)A->nnz * A->vsize(), cudaMemcpyHostToDevice,
                             ctx->stream));
  A->tr.values_fresh = false;
  A->plan.win.values_fresh = false;
  return SPOPS_OK;
}

spops_status_t spops_spmv_t(spops_context_t ctx, double alpha, spops_matrix_t A, const void* x, double beta,
                            void* y) {
  if (!ctx || !A) return fail(SPOPS_ERR_INVALID, "spops_spmv_t: null context/matrix");
  if ((!x && A->rows > 0) || (!y && A->cols > 0)) return fail(SPOPS_ERR_INVALID, "spops_spmv_t: null vector");
  DeviceGuard g(ctx->device);
  return csr_spmv_transpose(ctx, A, alpha, x, beta, y);
}

spops_status_t spops_sddmm(spops_context_t ctx, double alpha, spops_matrix_t A, const void* g, const void* x,
                           void* out) {
  if (!ctx || !A) return fail(SPOPS_ERR_INVALID, "spops_sddmm: null context/matrix");
  if (A->nnz > 0 && (!g || !x || !out)) return fail(SPOPS_ERR_INVALID, "spops_sddmm: null vector");
  DeviceGuard gd(ctx->device);
  return csr_sddmm(ctx, A, alpha, g, x, out);
}

spops_status_t spops_matrix_analyse(spops_context_t ctx, spops_matrix_t A) {
  if (!ctx || !A) return fail(SPOPS_ERR_INVALID, "spops_matrix_analyse: null argument");
  DeviceGuard g(ctx->device);
  switch (A->format) {
    case SPOPS_FMT_CSR: return csr_analyse(ctx, A);
    case SPOPS_FMT_COO: return A->csr_view ? SPOPS_OK : coo_analyse(ctx, A);
    default: return SPOPS_OK;  // other formats are complete when created
  }
}

spops_status_t spops_matrix_device_bytes(spops_matrix_t A, int64_t* bytes) {
  if (!A || !bytes) return fail(SPOPS_ERR_INVALID, "spops_matrix_device_bytes: null argument");
  auto own = [](const DevBuf& b) { return b.own ? (int64_t)b.bytes : 0; };
  const CsrPlan& P = A->plan;
  int64_t b = own(A->row) + own(A->col) + own(A->val) + own(P.blk_row) + own(P.blk_chunk) + own(P.partial) +
              own(P.counter) + own(P.seg);
  const PaddedData& D = A->pad;
  b += own(D.reorder) + own(D.chunk_len) + own(D.chunk_off) + own(D.row_len) + own(D.piece) + own(D.partial) +
       own(D.counter);
  b += own(A->dia.offsets) + own(A->dia.data) + own(A->bsr.row_ptr) + own(A->bsr.bcol) + own(A->bsr.data);
  b += own(A->tr.rp) + own(A->tr.ri) + own(A->tr.perm) + own(A->tr.val);
  const Csr5Data& F = A->csr5;
  b += own(F.tcol) + own(F.tval) + own(F.desc) + own(F.lane_row) + own(F.tile_ptr) + own(F.carry_in) +
       own(F.open_sum) + own(F.open_row) + own(F.empty);
  if (A->tr.view) {
    const CsrPlan& Q = A->tr.view->plan;
    b += own(Q.blk_row) + own(Q.blk_chunk) + own(Q.partial) + own(Q.counter) + own(Q.seg);
  }
  if (A->csr_view) {
    int64_t c = 0;
    spops_matrix_device_bytes(static_cast<spops_matrix_s*>(A->csr_view), &c);
    b += c;
  }
  *bytes = b;
  return SPOPS_OK;
}

spops_status_t spops_spmv(spops_context_t ctx, double alpha, spops_matrix_t A, const void* x, double beta, void* y) {
  if (!ctx || !A) return fail(SPOPS_ERR_INVALID, "spops_spmv: null context/matrix");
  if ((!x && A->cols > 0) || (!y && A->rows > 0)) return fail(SPOPS_ERR_INVALID, "spops_spmv: null vector");
  DeviceGuard g(ctx->device);
  switch (A->format) {
    case SPOPS_FMT_CSR: return csr_spmv(ctx, A, alpha, x, beta, y);
    case SPOPS_FMT_COO:
      if (!A->csr_view) SPOPS_TRY(coo_analyse(ctx, A));
      return csr_spmv(ctx, A->csr_view, alpha, x, beta, y);
    case SPOPS_FMT_SELL_C_SIGMA:
    case SPOPS_FMT_SELL_C_R:
    case SPOPS_FMT_SELL:
    case SPOPS_FMT_ELL: return padded_spmv(ctx, A, alpha, x, beta, y);
    case SPOPS_FMT_DIA: return dia_spmv(ctx, A, alpha, x, beta, y);
    case SPOPS_FMT_BSR: return bsr_spmv(ctx, A, alpha, x, beta, y);
    case SPOPS_FMT_CSR5: return csr5_spmv(ctx, A, alpha, x, beta, y);
    default: return fail(SPOPS_ERR_UNSUPPORTED, "SpMV for format %d", (int)A->format);
  }
}

spops_status_t spops_spmv_host_wait(spops_context_t ctx) {
  if (!ctx) return fail(SPOPS_ERR_INVALID, "spops_spmv_host_wait: null context");
  if (!ctx->a_pending) return SPOPS_OK;
  DeviceGuard g(ctx->device);
  cudaError_t e1 = ctx->in_stream ? cudaStreamSynchronize(ctx->in_stream) : cudaSuccess;
  cudaError_t e2 = cudaStreamSynchronize(ctx->stream);
  cudaError_t e3 = ctx->copy_stream ? cudaStreamSynchronize(ctx->copy_stream) : cudaSuccess;
  ctx->a_pending = false;
  SPOPS_CUDA(e1);
  SPOPS_CUDA(e2);
  SPOPS_CUDA(e3);
  return SPOPS_OK;
}

spops_status_t spops_spmv_host(spops_context_t ctx, double alpha, spops_matrix_t A, const void* x_host,
                               double beta, void* y_host) {
  if (!ctx || !A) return fail(SPOPS_ERR_INVALID, "spops_spmv_host: null context/matrix");
  SPOPS_TRY(spops_spmv_host_wait(ctx));
  DeviceGuard g(ctx->device);
  const size_t xb = (size_t)A->cols * A->vsize(), yb = (size_t)A->rows * A->vsize();
  if (ctx->xbuf.bytes < xb) SPOPS_TRY(ctx->xbuf.alloc(xb));
  if (ctx->ybuf.bytes < yb) SPOPS_TRY(ctx->ybuf.alloc(yb));
  cudaStream_t st = ctx->stream;
  if (xb) SPOPS_CUDA(cudaMemcpyAsync(ctx->xbuf.p, x_host, xb, cudaMemcpyHostToDevice, st));
  if (beta != 0.0 && yb) SPOPS_CUDA(cudaMemcpyAsync(ctx->ybuf.p, y_host, yb, cudaMemcpyHostToDevice, st));
  // Large CSR matrices on the default kernel: the SpMV runs in kHostParts row
  // ranges and each range's rows of y go back to the host on a second stream
  // while the next range computes, so only the last range's copy is exposed.
  constexpr int kHostParts = 8;
  // (only into page-locked y: a copy to pageable memory blocks the host and
  // would serialise the ranges)
  cudaPointerAttributes ya{};
  const bool y_pinned = y_host && cudaPointerGetAttributes(&ya, y_host) == cudaSuccess &&
                        ya.type == cudaMemoryTypeHost;
  cudaGetLastError();  // a pageable pointer may leave an error behind on some drivers
  const bool piped = y_pinned && A->format == SPOPS_FMT_CSR && A->rows >= (int64_t)1 << 20 && A->nnz > 0 &&
                     ctx->csr_variant == 0 && csr_tile_usable(A, 0);
  if (piped) {
    if (!ctx->copy_stream) SPOPS_CUDA(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    while ((int)ctx->part_events.size() < kHostParts) {
      cudaEvent_t e;
      SPOPS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      ctx->part_events.push_back(e);
    }
    if (!A->plan.ready) SPOPS_TRY(csr_analyse(ctx, A));
    const size_t vs = A->vsize();
    int used = 0;
    spops_status_t s = csr_tile_spmv_parts(
        ctx, A, kHostParts, alpha, ctx->xbuf.p, beta, ctx->ybuf.p, [&](int64_t r0, int64_t r1) -> spops_status_t {
          cudaEvent_t e = ctx->part_events[(size_t)(used++ % kHostParts)];
          SPOPS_CUDA(cudaEventRecord(e, st));
          SPOPS_CUDA(cudaStreamWaitEvent(ctx->copy_stream, e, 0));
          SPOPS_CUDA(cudaMemcpyAsync(static_cast<char*>(y_host) + r0 * vs, ctx->ybuf.as<char>() + r0 * vs,
                                     (size_t)(r1 - r0) * vs, cudaMemcpyDeviceToHost, ctx->copy_stream));
          return SPOPS_OK;
        });
    cudaError_t e1 = cudaStreamSynchronize(ctx->copy_stream);
    cudaError_t e2 = cudaStreamSynchronize(st);
    SPOPS_TRY(s);
    SPOPS_CUDA(e1);
    SPOPS_CUDA(e2);
    return SPOPS_OK;
  }
  SPOPS_TRY(spops_spmv(ctx, alpha, A, ctx->xbuf.p, beta, ctx->ybuf.p));
  if (yb) SPOPS_CUDA(cudaMemcpyAsync(y_host, ctx->ybuf.p, yb, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  (void)reserve_pinned;
  return SPOPS_OK;
}

spops_status_t spops_spmv_host_async(spops_context_t ctx, double alpha, spops_matrix_t A, const void* x_host,
                                     double beta, void* y_host) {
  if (!ctx || !A) return fail(SPOPS_ERR_INVALID, "spops_spmv_host_async: null context/matrix");
  const size_t vs = A->vsize(), xb = (size_t)A->cols * vs, yb = (size_t)A->rows * vs;
  if ((xb && !x_host) || (yb && !y_host)) return fail(SPOPS_ERR_INVALID, "spops_spmv_host_async: null vector");
  DeviceGuard g(ctx->device);
  auto pinned = [](const void* p) {
    cudaPointerAttributes a{};
    const bool ok = p && cudaPointerGetAttributes(&a, p) == cudaSuccess && a.type == cudaMemoryTypeHost;
    cudaGetLastError();
    return ok;
  };
  if ((xb && !pinned(x_host)) || (yb && !pinned(y_host)))  // copies from pageable memory block the host anyway
    return spops_spmv_host(ctx, alpha, A, x_host, beta, y_host);
  constexpr int kHostParts = 8;
  if (!ctx->in_stream) SPOPS_CUDA(cudaStreamCreateWithFlags(&ctx->in_stream, cudaStreamNonBlocking));
  if (!ctx->copy_stream) SPOPS_CUDA(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
  for (int i = 0; i < 2; ++i)
    for (cudaEvent_t* e : {&ctx->a_in[i], &ctx->a_read[i], &ctx->a_out[i]})
      if (!*e) SPOPS_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  while ((int)ctx->part_events.size() < kHostParts) {
    cudaEvent_t e;
    SPOPS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ctx->part_events.push_back(e);
  }
  const int s = ctx->a_next;
  ctx->a_next ^= 1;
  cudaStream_t st = ctx->stream, in = ctx->in_stream, out = ctx->copy_stream;
  if (ctx->axbuf[s].bytes < xb || ctx->aybuf[s].bytes < yb) {  // the slot grows: its last call must be done
    SPOPS_CUDA(cudaEventSynchronize(ctx->a_read[s]));
    SPOPS_CUDA(cudaEventSynchronize(ctx->a_out[s]));
    if (ctx->axbuf[s].bytes < xb) SPOPS_TRY(ctx->axbuf[s].alloc(xb));
    if (ctx->aybuf[s].bytes < yb) SPOPS_TRY(ctx->aybuf[s].alloc(yb));
  }
  void* xd = ctx->axbuf[s].p;
  char* yd = ctx->aybuf[s].as<char>();
  ctx->a_pending = true;
  // upload once the slot's previous SpMV has read x (and its download has read y)
  SPOPS_CUDA(cudaStreamWaitEvent(in, ctx->a_read[s], 0));
  if (beta != 0.0) SPOPS_CUDA(cudaStreamWaitEvent(in, ctx->a_out[s], 0));
  if (xb) SPOPS_CUDA(cudaMemcpyAsync(xd, x_host, xb, cudaMemcpyHostToDevice, in));
  if (beta != 0.0 && yb) SPOPS_CUDA(cudaMemcpyAsync(yd, y_host, yb, cudaMemcpyHostToDevice, in));
  SPOPS_CUDA(cudaEventRecord(ctx->a_in[s], in));
  // the SpMV after the upload and after the slot's previous download of y
  SPOPS_CUDA(cudaStreamWaitEvent(st, ctx->a_in[s], 0));
  SPOPS_CUDA(cudaStreamWaitEvent(st, ctx->a_out[s], 0));
  int used = 0;
  auto send = [&](int64_t r0, int64_t r1) -> spops_status_t {  // rows [r0, r1) of y back to the host
    cudaEvent_t e = ctx->part_events[(size_t)(used++ % kHostParts)];
    SPOPS_CUDA(cudaEventRecord(e, st));
    SPOPS_CUDA(cudaStreamWaitEvent(out, e, 0));
    if (r1 > r0)
      SPOPS_CUDA(cudaMemcpyAsync(static_cast<char*>(y_host) + r0 * vs, yd + r0 * vs, (size_t)(r1 - r0) * vs,
                                 cudaMemcpyDeviceToHost, out));
    return SPOPS_OK;
  };
  // One SpMV and one download of y: requests queued back to back already
  // overlap one request's download with the next one's upload and SpMV, and
  // cutting the SpMV into row ranges with a download each (as the blocking
  // spops_spmv_host does to shorten one request) measured slower here: 0.82
  // against 0.76 ms per request on the 4M-row power-law matrix, whose 64 MB
  // of x and y per request keep the host link busier than the 0.47 ms SpMV.
  SPOPS_TRY(spops_spmv(ctx, alpha, A, xd, beta, yd));
  SPOPS_TRY(send(0, A->rows));
  SPOPS_CUDA(cudaEventRecord(ctx->a_read[s], st));
  SPOPS_CUDA(cudaEventRecord(ctx->a_out[s], out));
  return SPOPS_OK;
}

}  // extern "C"
