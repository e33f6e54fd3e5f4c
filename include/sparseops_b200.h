/* sparseops_b200.h -- C ABI of the B200 (sm_100a) SparseOps hot path.
 *
 * Plain C: opaque handles, plain pointers and sizes, status codes.  No C++,
 * torch or CUDA types appear in the signatures (streams are passed as void*,
 * i.e. a cudaStream_t).  Every entry point names the reference interface it
 * replaces (lsl036/SparseOps, file:line).  The reference is a C++ template
 * library with no FFI of its own; these are the functions a cgo / ctypes /
 * JNI binding of its hot path binds, and the header-compatible C++ shim in
 * include/spops_b200/SpOps.h is built on them.
 *
 * Conventions
 *  - Every function returns spops_status_t; SPOPS_OK is 0.  On failure the
 *    library never exits the process (the reference calls exit()/assert:
 *    include/sparse_conversion.h:365-369, 728-743); spops_last_error() returns
 *    a message for the calling thread.
 *  - "device pointer" = memory of the context's device; "host pointer" =
 *    ordinary (pageable or pinned) host memory.
 *  - A matrix handle holds one storage format on the device plus whatever
 *    analysis its kernels need (row blocks, transposes), built once and reused.
 *  - Work is enqueued on the context's stream; functions that return host
 *    data synchronise that stream.
 */
#ifndef SPARSEOPS_B200_H
#define SPARSEOPS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPOPS_ABI_VERSION 1

typedef enum {
  SPOPS_OK = 0,
  SPOPS_ERR_INVALID = 1,     /* bad argument, shape or pointer */
  SPOPS_ERR_UNSUPPORTED = 2, /* type/format combination not provided */
  SPOPS_ERR_ALLOC = 3,       /* device or host allocation failed */
  SPOPS_ERR_CUDA = 4,        /* a CUDA runtime call failed */
  SPOPS_ERR_TOO_LARGE = 5,   /* result would exceed a stated limit (e.g. DIA diagonals, ELL bytes) */
  SPOPS_ERR_TIMEOUT = 6      /* a bounded device-side wait gave up (work queue) */
} spops_status_t;

typedef enum { SPOPS_INDEX_I32 = 0, SPOPS_INDEX_I64 = 1 } spops_index_t;
typedef enum { SPOPS_VALUE_F32 = 0, SPOPS_VALUE_F64 = 1 } spops_value_t;
typedef enum { SPOPS_MEM_DEVICE = 0, SPOPS_MEM_HOST = 1 } spops_mem_t;

/* Storage formats: the nine SpMV formats of include/sparse_format.h:49-295. */
typedef enum {
  SPOPS_FMT_CSR = 0,
  SPOPS_FMT_COO = 1,
  SPOPS_FMT_ELL = 2,
  SPOPS_FMT_SELL = 3,         /* S-ELL: sliced ELL, chunks of C consecutive rows */
  SPOPS_FMT_SELL_C_SIGMA = 4,
  SPOPS_FMT_SELL_C_R = 5,     /* SELL-C-sigma with one global sort */
  SPOPS_FMT_DIA = 6,
  SPOPS_FMT_BSR = 7,
  SPOPS_FMT_CSR5 = 8,
  SPOPS_FMT_VLCLUSTER = 9     /* CSR_VlengthCluster: clustered rows (LeSpGEMM_VLength operands) */
} spops_format_t;

/* Element layout inside an ELL matrix or a SELL chunk.  ROW_MAJOR is the
 * reference layout (include/sparse_conversion.h:237-249, 470-481); COL_MAJOR
 * is the device-native one (lane i of a warp reads row i: coalesced). */
typedef enum { SPOPS_ROW_MAJOR = 0, SPOPS_COL_MAJOR = 1 } spops_layout_t;

typedef struct spops_context_s* spops_context_t;
typedef struct spops_matrix_s* spops_matrix_t;
typedef struct spops_batch_s* spops_batch_t;
typedef struct spops_pairs_s* spops_pairs_t;

/* Parameters of a format conversion; zero means "reference default". */
typedef struct {
  int64_t sigma;      /* SELL-C-sigma slice height (reference SELL_SIGMA = 16384) */
  int64_t chunk;      /* C: rows per chunk (reference CHUNK_SIZE = 4) */
  int64_t alignment;  /* chunk width multiple (reference SIMD_WIDTH/8/sizeof(V)) */
  int64_t max_diags;  /* DIA limit (reference MAX_DIAG_NUM = 10240) */
  int64_t block_rows; /* BSR (reference BSR_BlockDimRow = 16) */
  int64_t block_cols; /* BSR (reference SIMD_WIDTH/8/sizeof(V)) */
  int32_t layout;     /* spops_layout_t for ELL / SELL variants */
  int32_t reserved;
} spops_format_params_t;

/* Scalar description of a matrix handle.  `extra` is format specific:
 *   SELL_C_SIGMA: [sliceNum, chunkNum, validchunkNum, chunk_num_per_slice, stored_elems]
 *   SELL_C_R / SELL: [chunks, stored_elems]
 *   ELL:  [max_row_width, min_row_width]
 *   DIA:  [complete_ndiags, stride]
 *   BSR:  [mb, nb, nnzb, blockDim_r, blockDim_c]
 *   CSR5: [tiles, omega, sigma]
 *   VLCLUSTER: [clusters, nnzv, max_cluster_sz] (rows = CSR rows, nnz = nnzc) */
typedef struct {
  int64_t rows, cols, nnz;
  int32_t format, index_type, value_type, layout;
  int64_t sigma, chunk, alignment;
  int64_t extra[8];
} spops_matrix_info_t;

/* ------------------------------------------------------------ context */
/* One context per (device, stream).  stream may be NULL (legacy default).
 * Matrices, batches and pair sets made with a context use its stream, and
 * their large arrays go back to its block cache when they are destroyed:
 * destroy them before the context. */
spops_status_t spops_create(spops_context_t* ctx, int device, void* stream);
spops_status_t spops_destroy(spops_context_t ctx);
spops_status_t spops_set_stream(spops_context_t ctx, void* stream);
spops_status_t spops_synchronize(spops_context_t ctx);
/* Synchronise and read (then clear) the context's device error word: bounded
 * device-side waits that ran out set bits there.  Returns SPOPS_ERR_TIMEOUT
 * when any bit was set; *flags (may be NULL) receives the bits. */
spops_status_t spops_check_device(spops_context_t ctx, int32_t* flags);
/* Tuning switches by name; unknown keys are rejected with SPOPS_ERR_INVALID.
 *   "csr_variant" 0..10: CSR SpMV kernel.  Tiles of 32*K entries summed in
 *   registers (K entries per lane / resident blocks per SM / next tile's
 *   loads issued early): 0 = 8/3/yes (default), 1 = 8/4/no, 5 = 4/4/no,
 *   6 = 8/5/no; they need the column and value arrays aligned to
 *   min(32, K * element size) bytes, otherwise variant 2 runs.  Row segments
 *   through shared memory (entries per lane per round / blocks per SM):
 *   2 = 8/4, 3 = 4/6, 4 = 16/2.  Column-sorted row windows whose partial y
 *   stays in shared memory (windows resident per SM): 7 = 1, 8 = 2, 9 = 4;
 *   they keep a copy of the values (refreshed after spops_csr_set_values or
 *   spops_matrix_touch), need cols and nnz below 2^31 (otherwise variant 2
 *   runs), and add a row's products in an order that can change from run to
 *   run at rounding level; variants 0-6 are bit-reproducible.  10: the tiles
 *   of variant 0 with each warp's columns, values and flags brought into
 *   shared memory by bulk copies two tiles ahead (measured slower than 0 on
 *   the power-law matrix: the x gathers need the L1 capacity the slots take);
 *   bit-reproducible, equal to variant 0 up to rounding. 
 *   "batch_band" 0 / 1: batched SpMV with one right-hand side stages each CSR
 *   segment's x window [r0 - H, r0 + rows + H) in shared memory, H in
 *   {16, 32, 64} from the matrix's band profile (0, the default: plain
 *   gathers).  Read when a batch is prepared and launched.
 *   "sell_tails" 0 / 1: SELL with C = 32, column-major: each 32-row chunk's
 *   slots beyond its fourth-longest row (held by at most three rows) are
 *   read in place (0, the default), or also kept row-contiguous and read from
 *   there (1).  Read when the matrix is converted or uploaded.
 *   "sell_order" 1 / 0: SELL with C = 32, column-major: the chunks' step
 *   windows are listed longest chunk first, so that warps running at the
 *   same time hold rows of like length (1, the default), or in chunk order
 *   (0).  The per-row results do not depend on it.  Read when the matrix is
 *   converted or uploaded.
 *   "adjoint_bands" 0 .. 8: spops_spmv_t right after a value change reads A's
 *   values through the transpose's permutation; it can do so in bands of
 *   source rows of about equal entry counts, each band's slice of the values
 *   small enough to stay in L2 while its gathers run, the bands adding into
 *   y in band order.  0 (the default): as many bands as keep each slice
 *   within 64 MB once the values pass 96 MB, else one pass; 1: one pass;
 *   2 .. 8: that many bands.  The bands' row offsets, columns and positions
 *   are built once per pattern and count (about 12 bytes per entry with
 *   int32 indices) and kept with the matrix.  Summation order changes with
 *   the count (rounding level); every count is bit-reproducible. */
spops_status_t spops_set_option(spops_context_t ctx, const char* key, int64_t value);
const char* spops_status_string(spops_status_t s);
const char* spops_last_error(void);
int spops_abi_version(void);

/* ------------------------------------------------------------- matrices */
/* CSR matrix from row_offset[rows+1], col_index[nnz], values[nnz].
 * SPOPS_MEM_DEVICE: the arrays are BORROWED (not copied); they must outlive
 *   the handle and must not change while analysis results are in use
 *   (call spops_matrix_touch after changing values in place).
 * SPOPS_MEM_HOST: the arrays are uploaded into device memory the handle owns.
 * Replaces the reference's host-side CSR_Matrix<I,V> (include/sparse_format.h:95-104)
 * as consumed by SpOps_csr (src/spmv_csr.cpp:165). */
spops_status_t spops_csr_create(spops_context_t ctx, spops_matrix_t* A, int64_t rows, int64_t cols, int64_t nnz,
                                const void* row_offset, const void* col_index, const void* values,
                                spops_index_t itype, spops_value_t vtype, spops_mem_t mem);
/* COO triplets; rows need not be sorted (include/sparse_format.h:72-81). */
spops_status_t spops_coo_create(spops_context_t ctx, spops_matrix_t* A, int64_t rows, int64_t cols, int64_t nnz,
                                const void* row_index, const void* col_index, const void* values,
                                spops_index_t itype, spops_value_t vtype, spops_mem_t mem);
/* Matrix Market text parsed on the device.  Replaces read_coo_matrix and
 * read_csr_matrix (utils/sparse_io.cpp:26-214; banner and size line as
 * mm_read_banner / mm_read_mtx_crd_size, utils/mmio.cpp:144-283): sparse
 * real, integer or pattern coordinate files; "symmetric" files expanded with
 * each off-diagonal entry followed by its mirror; values converted as
 * scanf("%lf") does (correctly rounded decimal to double) and then cast to
 * vtype; indices 1-based in the file.  _read_ take a file path (read on the
 * host, parsed on the device), _parse_ the file's bytes in host memory.  The
 * COO handle keeps the file's entry order; the CSR handle is coo_to_csr's
 * (compact: duplicates summed).  A file with zero rows gives a 0 x 0 matrix.
 * Malformed numbers, indices outside the size line and fewer entries than it
 * announces are refused with SPOPS_ERR_INVALID (the reference asserts). */
spops_status_t spops_mtx_read_coo(spops_context_t ctx, const char* path, spops_index_t itype, spops_value_t vtype,
                                  spops_matrix_t* coo);
spops_status_t spops_mtx_parse_coo(spops_context_t ctx, const char* text, int64_t len, spops_index_t itype,
                                   spops_value_t vtype, spops_matrix_t* coo);
spops_status_t spops_mtx_read_csr(spops_context_t ctx, const char* path, spops_index_t itype, spops_value_t vtype,
                                  int32_t compact, spops_matrix_t* csr);
spops_status_t spops_mtx_parse_csr(spops_context_t ctx, const char* text, int64_t len, spops_index_t itype,
                                   spops_value_t vtype, int32_t compact, spops_matrix_t* csr);
/* CSR handle (owned arrays) from a COO handle, on the device.  Replaces
 * coo_to_csr (include/sparse_conversion.h:37-99): rows in order, file order
 * kept within a row.  compact != 0 adds the reference's sum_csr_duplicates
 * (include/sparse_operation.h:21-69): equal columns of a row summed in file
 * order, distinct columns listed in reverse order of first appearance,
 * exact-zero sums dropped -- bit-identical to the reference. */
spops_status_t spops_coo_to_csr(spops_context_t ctx, spops_matrix_t coo, int32_t compact, spops_matrix_t* csr);
/* Rows of a CSR matrix in a new order: row i of *out is row perm[i] of csr
 * (csr_reorder_rows, include/sparse_conversion.h:1879-1998).  perm: host
 * array of csr's index type, a permutation of 0 .. rows-1; anything else is
 * refused with SPOPS_ERR_INVALID (the reference does not check). */
spops_status_t spops_csr_reorder_rows(spops_context_t ctx, spops_matrix_t csr, const void* perm, spops_matrix_t* out);
spops_status_t spops_matrix_destroy(spops_matrix_t A);
spops_status_t spops_matrix_info(spops_matrix_t A, spops_matrix_info_t* info);
/* Values changed in place (same pattern): drop value-derived caches. */
spops_status_t spops_matrix_touch(spops_matrix_t A);
/* Build the analysis a format's SpMV uses (lazily done by the first SpMV). */
spops_status_t spops_matrix_analyse(spops_context_t ctx, spops_matrix_t A);
/* Bytes of device memory the handle owns (arrays + analysis). */
spops_status_t spops_matrix_device_bytes(spops_matrix_t A, int64_t* bytes);

/* Point a CSR handle at new values (same pattern, same length, device
 * pointer, borrowed).  Keeps the analysis; marks derived values stale. */
spops_status_t spops_csr_set_values(spops_matrix_t A, const void* values);
/* Copy new values from host memory into a CSR handle that owns its values
 * (created from SPOPS_MEM_HOST arrays): same pattern, nnz values of the
 * handle's value type, queued on the context's stream.  Keeps the analysis;
 * marks derived values stale.  This is what the reference's per-call read of
 * A.values amounts to when the pattern is kept on the device (SpOps_csr,
 * src/spmv_csr.cpp:165, reads the host arrays on every call). */
spops_status_t spops_csr_upload_values(spops_context_t ctx, spops_matrix_t A, const void* host_values);

/* ------------------------------------------------------ format handles */
/* Device conversion of a CSR handle into another format (all work on the
 * device; integer layout arrays are bit-identical to the reference's):
 *   SELL_C_SIGMA  csr_to_sell_c_sigma  include/sparse_conversion.h:344
 *   SELL_C_R      csr_to_sell_c_R      include/sparse_conversion.h:490
 *   SELL (S-ELL)  csr_to_sell          include/sparse_conversion.h:265
 *   ELL           csr_to_ell           include/sparse_conversion.h:194
 *   DIA           csr_to_dia           include/sparse_conversion.h:619
 *   BSR           csr_to_bsr           include/sparse_conversion.h:776
 *   COO           csr_to_coo           include/sparse_conversion.h:152
 *   CSR5          csr_to_csr5          include/sparse_conversion.h:946 (device
 *                 tiles of 32 lanes x 16 entries; tile arrays differ from the
 *                 reference's CPU-SIMD tiles, SpMV results agree)
 * params may be NULL (reference defaults).  Errors the reference reports by
 * exit() come back as status codes: sigma not a multiple of C ->
 * SPOPS_ERR_INVALID; more than max_diags diagonals, or padded storage that
 * cannot fit in device memory -> SPOPS_ERR_TOO_LARGE. */
spops_status_t spops_convert(spops_context_t ctx, spops_matrix_t csr, spops_format_t format,
                             const spops_format_params_t* params, spops_matrix_t* out);

/* Padded-row matrix (SELL_C_SIGMA, SELL_C_R, SELL or ELL) from the arrays of
 * a reference struct, chunks concatenated in chunk order: chunk_len[nchunks]
 * (ELL: one chunk of width max_row_width), col[stored] (-1 = padding),
 * val[stored], reorder[rows] (SELL_C_SIGMA / SELL_C_R only, else NULL).
 * layout: SPOPS_ROW_MAJOR (reference) or SPOPS_COL_MAJOR.
 * Replaces the host structs of include/sparse_format.h:190-295 as consumed by
 * SpOps_sell_c_sigma / SpOps_sell_c_R / SpOps_sell / SpOps_ell. */
spops_status_t spops_padded_create(spops_context_t ctx, spops_matrix_t* A, spops_format_t format, int64_t rows,
                                   int64_t cols, int64_t nnz, int64_t chunk, int64_t sigma, int64_t alignment,
                                   spops_layout_t layout, const void* reorder, const void* chunk_len,
                                   int64_t nchunks, const void* col, const void* val, int64_t stored,
                                   spops_index_t itype, spops_value_t vtype, spops_mem_t mem);
/* DIA from diag_offsets[ndiag] (int64) and diag_data[ndiag * stride]
 * (include/sparse_format.h:172-184, consumed by SpOps_dia src/spmv_dia.cpp:177). */
spops_status_t spops_dia_create(spops_context_t ctx, spops_matrix_t* A, int64_t rows, int64_t cols, int64_t nnz,
                                int64_t ndiag, int64_t stride, const int64_t* diag_offsets, const void* diag_data,
                                spops_value_t vtype, spops_mem_t mem);
/* BSR from row_ptr[mb+1], block_colindex[nnzb], block_data[nnzb*br*bc]
 * (include/sparse_format.h:110-127, consumed by SpOps_bsr src/spmv_bsr.cpp:214). */
spops_status_t spops_bsr_create(spops_context_t ctx, spops_matrix_t* A, int64_t rows, int64_t cols, int64_t nnz,
                                int64_t block_rows, int64_t block_cols, int64_t nnzb, const void* row_ptr,
                                const void* block_col, const void* block_data, spops_index_t itype,
                                spops_value_t vtype, spops_mem_t mem);

/* Arrays of a handle, for export into the reference structs. */
typedef enum {
  SPOPS_ARR_ROW = 0,           /* CSR row_offset / COO row_index */
  SPOPS_ARR_COL = 1,           /* column indices (padded formats: slots, -1 = padding) */
  SPOPS_ARR_VAL = 2,           /* values; padded slots; DIA diag_data; BSR block_data */
  SPOPS_ARR_REORDER = 3,       /* SELL-C-sigma / SELL-C-R: stored row -> original row */
  SPOPS_ARR_CHUNK_LEN = 4,     /* chunk_len / S-ELL row_width / ELL max_row_width */
  SPOPS_ARR_CHUNK_OFF = 5,     /* int64 first slot of every chunk (nchunks + 1) */
  SPOPS_ARR_ROW_LEN = 6,       /* int32 slots up to each stored row's last entry */
  SPOPS_ARR_DIAG_OFFSETS = 7,  /* int64 DIA diag_offsets */
  SPOPS_ARR_BLOCK_ROW_PTR = 8, /* BSR row_ptr */
  SPOPS_ARR_BLOCK_COL = 9,     /* BSR block_colindex */
  SPOPS_ARR_TILE_PTR = 10,     /* CSR5 tile_ptr (uint32, bit 31: tile spans an empty row) */
  SPOPS_ARR_TILE_DESC = 11,    /* CSR5 per-lane row-start flags (uint32, tiles x 32) */
  SPOPS_ARR_CLUSTER_SZ = 12,   /* VLCLUSTER cluster_sz (rows per cluster) */
  SPOPS_ARR_ROWPTR_VAL = 13    /* VLCLUSTER rowptr_val (clusters + 1) */
} spops_array_t;
/* Device pointer, element count and element size of one array (no copy). */
spops_status_t spops_matrix_array(spops_matrix_t A, spops_array_t which, const void** dev_ptr, int64_t* count,
                                  int32_t* elem_bytes);
/* Copy one array into host memory (count elements; synchronises). */
spops_status_t spops_matrix_download(spops_context_t ctx, spops_matrix_t A, spops_array_t which, void* host_dst,
                                     int64_t count);

/* ---------------------------------------------------------------- SpMV */
/* y = alpha*A*x + beta*y on the device; x[cols], y[rows] device pointers of
 * A's value type.  beta == 0 overwrites y without reading it.
 * Replaces SpOps_<fmt>(alpha, A, x, beta, y) for every format:
 *   csr src/spmv_csr.cpp:165, coo src/spmv_coo.cpp:160, ell src/spmv_ell.cpp:225,
 *   sell src/spmv_s_ell.cpp:202, sell_c_sigma src/spmv_sell_c_sigma.cpp:189,
 *   sell_c_R src/spmv_sell_c_R.cpp:190, dia src/spmv_dia.cpp:177,
 *   bsr src/spmv_bsr.cpp:214, csr5 src/spmv_csr5.cpp:439. */
spops_status_t spops_spmv(spops_context_t ctx, double alpha, spops_matrix_t A, const void* x, double beta,
                          void* y);
/* Same with HOST x and y: uploads x (and y when beta != 0), downloads y.
 * The drop-in path of the header shim (host pointers in, host pointers out). */
spops_status_t spops_spmv_host(spops_context_t ctx, double alpha, spops_matrix_t A, const void* x_host,
                               double beta, void* y_host);
/* The same, queued: for a stream of independent requests (a server's SpMV
 * calls) whose host x and y are page-locked.  Returns once the upload, the
 * SpMV and the download are enqueued; the context alternates two device
 * slots, so request k + 1's upload runs while request k computes and its y
 * comes back.  x must stay unchanged and y unread until
 * spops_spmv_host_wait(ctx) returns (or a spops_spmv_host call, which waits
 * first).  With pageable x or y the call runs to completion as
 * spops_spmv_host does.  No reference counterpart: SpOps_<fmt> returns when
 * y is written. */
spops_status_t spops_spmv_host_async(spops_context_t ctx, double alpha, spops_matrix_t A, const void* x_host,
                                     double beta, void* y_host);
spops_status_t spops_spmv_host_wait(spops_context_t ctx);
/* Multi-RHS: Y = alpha*A*X + beta*Y with X [cols x k], Y [rows x k],
 * row-major with leading dimensions ldx, ldy (>= k).  No reference
 * counterpart (the reference has no SpMM); equals k SpOps_csr calls. */
spops_status_t spops_spmm(spops_context_t ctx, double alpha, spops_matrix_t A, const void* X, int64_t ldx,
                          int64_t k, double beta, void* Y, int64_t ldy);

/* ------------------------------------------------------------- batches */
/* Many CSR matrices (uneven sizes, same index/value types) run as ONE
 * persistent kernel launch: y_m = alpha * A_m x_m + beta * y_m for every m,
 * or with k > 1 right-hand sides Y_m = alpha * A_m X_m + beta * Y_m
 * (row-major X_m [cols_m x ldx_m], Y_m [rows_m x ldy_m]).
 * No reference counterpart: the reference calls SpOps_csr once per matrix
 * and column (the baseline these are compared with).
 * The handles must outlive the batch.  Work runs on the batch's own stream,
 * ordered after and before the context's stream with events. */
spops_status_t spops_batch_create(spops_context_t ctx, spops_batch_t* batch, int64_t count,
                                  const spops_matrix_t* mats, int64_t k);
spops_status_t spops_batch_destroy(spops_batch_t batch);
/* Device pointers of x/X and y/Y per matrix (host arrays of `count`
 * pointers); ldx / ldy may be NULL (= k). */
spops_status_t spops_batch_set_vectors(spops_batch_t batch, const void* const* X, const int64_t* ldx,
                                       void* const* Y, const int64_t* ldy);
/* Autotune: per matrix (k = 1) time CSR against SELL-C-sigma with C = 32,
 * sigma in {256, 4096}, row- and column-major chunks, on the device, and keep
 * the fastest; for k > 1 pick the right-hand-side tile (8 or 32 lanes).
 * flags bit 0: CSR only.  Needs the vectors set (it runs the products). */
spops_status_t spops_batch_tune(spops_context_t ctx, spops_batch_t batch, int32_t flags);
/* One persistent launch over all matrices (a captured graph is replayed
 * when alpha/beta match the captured ones). */
spops_status_t spops_batch_run(spops_context_t ctx, spops_batch_t batch, double alpha, double beta);
/* Capture the launch into a CUDA graph for later spops_batch_run calls. */
spops_status_t spops_batch_capture(spops_context_t ctx, spops_batch_t batch, double alpha, double beta);
/* items: work items of the launch; choice[count]: 0 = CSR, 1..4 = SELL-C-sigma
 * candidate (sigma 256/4096 x row/col-major); rhs_tile: lanes per RHS tile. */
spops_status_t spops_batch_info(spops_batch_t batch, int64_t* items, int32_t* choice, int32_t* rhs_tile);

/* ------------------------------------------------------------ LeSpGEMM */
/* MinHash signatures of A's rows: sig[rows x k] (device, uint64), row-major.
 * Replaces minhash_signatures_flat (include/spgemm_MinHashLSH.h:119);
 * bit-identical (same LCG coefficients from seed). */
spops_status_t spops_minhash(spops_context_t ctx, spops_matrix_t A, int32_t k, uint64_t seed, void* sig);
/* Same with a HOST output array sig_host[rows * k] (device scratch inside). */
spops_status_t spops_minhash_host(spops_context_t ctx, spops_matrix_t A, int32_t k, uint64_t seed, void* sig_host);
/* LSH candidate pairs (i < j, sorted, unique) with MinHash-estimated scores
 * (matches / k), on the device.  Replaces lsh_candidate_pairs_vector
 * (include/spgemm_MinHashLSH.h:777); constrain != 0: a bucket of more than
 * 256 rows pairs each row with its next 16 only. */
spops_status_t spops_lsh_pairs(spops_context_t ctx, spops_matrix_t A, int32_t k, int32_t bands, uint64_t seed,
                               int32_t constrain, spops_pairs_t* pairs);
/* Same from precomputed device signatures (lsh_candidate_pairs_from_flat_vector, :427). */
spops_status_t spops_lsh_pairs_from_signatures(spops_context_t ctx, const void* sig, int64_t rows, int32_t k,
                                               int32_t bands, int32_t constrain, spops_pairs_t* pairs);
/* A pair set from a caller's arrays i, j (int64) and score (double) of
 * `count` elements, host (SPOPS_MEM_HOST) or device (SPOPS_MEM_DEVICE) memory;
 * the arrays are copied.  The reference's clustering takes any such vector of
 * pairs (hierarchical_clustering_v0_fast, include/spgemm_utility.h:742). */
spops_status_t spops_pairs_create(spops_context_t ctx, const int64_t* i, const int64_t* j, const double* score,
                                  int64_t count, spops_mem_t mem, spops_pairs_t* pairs);
spops_status_t spops_pairs_count(spops_pairs_t pairs, int64_t* count);
/* Device arrays of the pairs: i, j (int64) and score (double). */
spops_status_t spops_pairs_arrays(spops_pairs_t pairs, const int64_t** i, const int64_t** j, const double** score);
/* Copy the pairs to host arrays of spops_pairs_count elements (any may be NULL). */
spops_status_t spops_pairs_download(spops_pairs_t pairs, int64_t* i, int64_t* j, double* score);
spops_status_t spops_pairs_destroy(spops_pairs_t pairs);
/* Hierarchical clustering of rows from sorted candidate pairs, on HOST arrays
 * (sequential merge order).  Replaces hierarchical_clustering_v0_fast
 * (include/spgemm_utility.h:742); bit-identical permutation[rows] (new row ->
 * original row) and offsets[nclusters + 1] (caller sizes it rows + 1). */
spops_status_t spops_hierarchical_clustering(const int64_t* row_ptr, const int64_t* col_index, int64_t rows,
                                             const int64_t* pi, const int64_t* pj, const double* score,
                                             int64_t npairs, int64_t cluster_size, int64_t* permutation,
                                             int64_t* offsets, int64_t* nclusters);

/* The same clustering on the device, from device pairs (spops_lsh_pairs) and
 * A's device pattern: bit-identical permutation[rows] and offsets[nclusters +
 * 1] (host arrays; offsets sized rows + 1).  Replaces
 * hierarchical_clustering_v0_fast (include/spgemm_utility.h:742-915): the
 * candidates run as prioritised tasks in rounds of root reservations, which
 * reproduce the sequential merge order; pair lists that are not sorted
 * i < j pairs take the host loop. */
spops_status_t spops_pairs_cluster(spops_context_t ctx, spops_matrix_t A, spops_pairs_t pairs, int64_t cluster_size,
                                   int64_t* permutation, int64_t* offsets, int64_t* nclusters);

typedef struct {
  int64_t flops;             /* 2 x intermediate products (get_spgemm_flop, src/spgemm.cpp:24) */
  int64_t clusters, dense_clusters, pairs;
  int64_t cluster_columns;   /* nnzc of the clustered A */
  int64_t c_cluster_columns; /* nnzc of the clustered C (before dropping zeros) */
  double minhash_ms, lsh_ms, hc_ms, cluster_ms, symbolic_ms, numeric_ms, to_csr_ms;
} spops_spgemm_stats_t;

/* C = A * B with the rows of A grouped into clusters (permutation / offsets
 * from the clustering), cluster-wise symbolic and numeric phases on the
 * device (hash / dense hybrid accumulator rules of kernel 3).  C is a new CSR
 * handle in A's original row order with ascending columns; entries whose
 * value is exactly zero are dropped as vlength_cluster2csr does.  Replaces
 * csr_reorder_rows + csr_to_vlength_cluster + LeSpGEMM_VLength(kernel 3) +
 * vlength_cluster2csr + inverse reorder (test/test_spgemm_hc_lsh.cpp:230-300,
 * src/spgemm.cpp:661).  l2_budget_bytes: the dense/hash classification
 * budget (the reference: CPU_L2CACHE_SIZE * 0.75); it only decides which
 * clusters drop all-below-1e-12 columns.  stats may be NULL. */
spops_status_t spops_spgemm_clustered(spops_context_t ctx, spops_matrix_t A, spops_matrix_t B,
                                      const int64_t* permutation, const int64_t* offsets, int64_t nclusters,
                                      int32_t sort_output, double l2_budget_bytes, spops_matrix_t* C,
                                      spops_spgemm_stats_t* stats);
/* Row-wise C = A * B: every structural entry of the product kept (exact
 * zeros included, no small-value drop), ascending columns in every row.
 * Replaces LeSpGEMM<sortOutput,I,V>(A, B, C, kernel_flag) (src/spgemm.cpp:683)
 * with its hash / array / sparse-accumulator row kernels (kernel_flag 1 / 2 /
 * 3, src/spgemm.cpp:44-235); they produce the same entries and differ only in
 * the unsorted column order of kernel 1, which ascending order satisfies. */
spops_status_t spops_spgemm_rowwise(spops_context_t ctx, spops_matrix_t A, spops_matrix_t B, int32_t kernel_flag,
                                    int32_t sort_output, spops_matrix_t* C, spops_spgemm_stats_t* stats);
/* Top-k Jaccard similarities of A's rows: for every row i, the top_k other
 * rows j (j != i) sharing a column with it, by |A_i n A_j| / |A_i u A_j|
 * (value type arithmetic, row lengths from A's offsets), ordered by
 * similarity descending then column ascending.  Replaces HashSpGEMMTopK
 * (src/spgemm.cpp:708-842, src/spgemm_hash.cpp:168-318). */
spops_status_t spops_spgemm_topk(spops_context_t ctx, spops_matrix_t A, int64_t top_k, spops_matrix_t* C);
/* The whole LeSpGEMM pipeline: MinHash + LSH (device), clustering (device),
 * cluster-wise SpGEMM (device). */
spops_status_t spops_spgemm_lsh(spops_context_t ctx, spops_matrix_t A, spops_matrix_t B, int32_t k, int32_t bands,
                                uint64_t seed, int64_t cluster_size, int32_t sort_output, double l2_budget_bytes,
                                spops_matrix_t* C, spops_spgemm_stats_t* stats);

/* ------------------------------------------------------------ adjoints */
/* y = alpha * A^T x + beta * y for a CSR handle: x[rows], y[cols] (device).
 * Replaces csr_transpose (include/sparse_conversion.h:2066) followed by
 * SpOps_csr on the transpose; the transpose pattern is built once on the
 * device (no atomics) and its values follow A's (spops_matrix_touch). */
spops_status_t spops_spmv_t(spops_context_t ctx, double alpha, spops_matrix_t A, const void* x, double beta,
                            void* y);
/* out[k] = alpha * g[row(k)] * x[col(k)] for every stored entry k of a CSR
 * handle (sampled dense-dense product on A's pattern): the gradient of
 * sum_i g_i * (alpha*A*x)_i with respect to A's values.  No reference
 * counterpart (the reference has no differentiation). */
spops_status_t spops_sddmm(spops_context_t ctx, double alpha, spops_matrix_t A, const void* g, const void* x,
                           void* out);

/* ------------------------------------------- features and format choice */
/* Structure features of a CSR matrix, computed on the device.  Replaces the
 * non-tile part of MTX::CalculateFeatures (src/sparse_features.cpp:643-775,
 * with the per-entry counts MTX::MtxLoad gathers, :336-478) for a general
 * (non-symmetric storage) matrix without duplicate entries:
 *   ndiags / diag_close_ratio: distinct diagonals; share of entries with
 *     |col - row| <= (rows + cols - 1) / 20
 *   p_ratio_*: smallest fraction p of rows (columns) holding at least 1 - p
 *     of the entries; gini_*: Gini coefficient of the per-row (per-column)
 *     counts by the trapezoid rule
 *   diagonal_dominant_ratio: rows whose |a_ii| exceeds the sum of their
 *     off-diagonal |a_ij|, over min(rows, cols)
 *   row_ / col_variability: largest log10 range of |a| over rows (columns)
 *     that hold a value below 1, with the reference's clamping at 0 (-1 if none)
 *   pattern_symm / value_symm (square only): share of off-diagonal entries
 *     whose mirror exists / exists with the same value printed to 6 decimals */
typedef struct {
  int64_t rows, cols, nnz;
  int64_t nnz_lower, nnz_upper, nnz_diagonal, ndiags;
  int64_t min_nnz_row, max_nnz_row, min_nnz_col, max_nnz_col;
  double nnz_ratio, diag_close_ratio, pattern_symm, value_symm;
  double nz_row_ratio, ave_nnz_row, var_nnz_row, std_nnz_row, p_ratio_row, gini_row;
  double nz_col_ratio, ave_nnz_col, var_nnz_col, std_nnz_col, p_ratio_col, gini_col;
  double diagonal_dominant_ratio, max_value_offdiag, max_value_diagonal, row_variability, col_variability;
} spops_features_t;
spops_status_t spops_matrix_features(spops_context_t ctx, spops_matrix_t csr, spops_features_t* features);

/* Tile features of a CSR matrix, computed on the device.  Replaces the tile
 * part of MTX::MtxLoad (src/sparse_features.cpp:181-265 per entry, :484-625
 * per tile and block), MTX::CalculateTilesFeatures (:783-846) and the
 * distance_per_row_ of MTX::CalculateTilesExtraFeatures (:943-965).
 * The matrix is cut into num_blocks x num_blocks tiles (MAT_TILE_SIZE = 256
 * in the reference; num_blocks <= 0 means 256, at most 2048): rows into
 * num_blocks row blocks (RB), of which the first rows % num_blocks hold
 * rows / num_blocks + 1 rows and the rest rows / num_blocks; columns into
 * column blocks (CB) alike.  The statistics over the tile, RB and CB entry
 * counts follow CalculateTilesFeatures, including its starting values:
 * nz_ratio_* = (non-empty count - 1) / length and var_* = (sum of squared
 * deviations - 1) / length, std_* = sqrt(max(var_*, 0)); min_* is at most
 * 100000000.  uniq_r / uniq_c: sum over tiles of the rows (columns) holding
 * an entry in the tile, over nnz; pot_reuse_r / _c: the same sums over rows
 * (columns).  distance_per_row: mean over rows of (last column - first
 * column in storage order) / row length (0 for empty rows), as the
 * reference's sum of neighbour distances telescopes to. */
typedef struct {
  int64_t num_blocks, rows_per_block, rows_mod, cols_per_block, cols_mod; /* t_num_blocks, t_num_RB, t_mod_RB, ... */
  int64_t min_nnz_tile, max_nnz_tile, min_nnz_rb, max_nnz_rb, min_nnz_cb, max_nnz_cb;
  double nz_ratio_tiles, ave_nnz_tile, var_nnz_tile, std_nnz_tile, p_ratio_tiles, gini_tiles;
  double nz_ratio_rb, ave_nnz_rb, var_nnz_rb, std_nnz_rb, p_ratio_rb, gini_rb;
  double nz_ratio_cb, ave_nnz_cb, var_nnz_cb, std_nnz_cb, p_ratio_cb, gini_cb;
  double uniq_r, uniq_c, pot_reuse_r, pot_reuse_c, distance_per_row;
} spops_tile_features_t;

/* Per-tile and per-block maps (the files MTX::FeaturesWrite writes,
 * src/sparse_features.cpp:1218-1330), host arrays filled when not NULL.
 * tile_* hold num_blocks^2 values, tile (i, j) at i * num_blocks + j; the
 * rb_* and cb_* arrays num_blocks values.  Row statistics of a tile run over
 * all rows of its row block, empty ones included (std: population standard
 * deviation); the RB / CB ones over the block's rows / columns. */
typedef struct {
  int64_t* tile_nnz;          /* nnz_by_Tiles_ */
  int64_t* tile_rows;         /* uniq_RB: rows with an entry in the tile */
  int64_t* tile_cols;         /* uniq_CB: columns with an entry in the tile */
  int64_t* tile_max_row_nnz;  /* max_rownnz_per_tile_ */
  double* tile_ave_row_nnz;   /* ave_rownnz_per_tile_ */
  double* tile_std_row_nnz;   /* std_rownnz_per_tile_ */
  int64_t* rb_nnz;            /* nnz_by_RB_ */
  int64_t* rb_max_row_nnz;    /* max_rownnz_per_RB_ */
  double* rb_ave_row_nnz;     /* ave_rownnz_per_RB_ */
  double* rb_std_row_nnz;     /* std_rownnz_per_RB_ */
  int64_t* cb_nnz;            /* nnz_by_CB_ */
  int64_t* cb_max_col_nnz;    /* max_colnnz_per_CB_ */
  double* cb_ave_col_nnz;     /* ave_colnnz_per_CB_ */
  double* cb_std_col_nnz;     /* std_colnnz_per_CB_ */
} spops_tile_maps_t;
spops_status_t spops_matrix_tile_features(spops_context_t ctx, spops_matrix_t csr, int64_t num_blocks,
                                          spops_tile_features_t* features, const spops_tile_maps_t* maps);

/* Storage format for y = A*x on this GPU.  No counterpart in the reference,
 * which computes features but leaves the choice to the caller.
 *   mode 0: rules on the features -- DIA when at most 64 diagonals hold at
 *     least half of the diagonal slots, otherwise CSR (the default CSR kernel
 *     needs no conversion and is within a few percent of the best padded
 *     format on irregular rows);
 *   mode 1: timed -- converts to each candidate (CSR, SELL-C-R and
 *     SELL-C-sigma with C = 32, CSR5, and DIA / BSR where the features allow
 *     them), runs a few SpMVs of each on the context stream, and returns the
 *     fastest;
 *   mode 2: learned -- a decision tree over derived features, fitted on
 *     seeded matrices whose SpMV time this library measured on a B200 in
 *     every mode-1 candidate (sparseops_b200/selector.py); the features'
 *     cost, no conversion or timing.  The model the reference's feature
 *     output (src/sparse_features.cpp:1225) is meant for.
 * *params receives the conversion parameters for spops_convert; ms (may be
 * NULL) the measured time per SpMV of the choice (mode 1; 0 in mode 0). */
spops_status_t spops_select_format(spops_context_t ctx, spops_matrix_t csr, int32_t mode, spops_format_t* format,
                                   spops_format_params_t* params, double* ms);
/* Mode 2's choice from features already computed (host only: no device
 * work), e.g. from spops_matrix_features or a stored feature file. */
spops_status_t spops_select_format_from_features(const spops_features_t* features, spops_format_t* format,
                                                 spops_format_params_t* params);

/* ------------------------------------------------ clustered (VLength) form */
/* CSR_VlengthCluster (spgemm_cluster.h:108-143) as a handle of format
 * SPOPS_FMT_VLCLUSTER: clusters of consecutive rows; cluster i holds the
 * union of its rows' columns, colids[rowptr[i] .. rowptr[i+1]), and for the
 * cluster's column p and its row k the value
 * values[rowptr_val[i] + p * cluster_sz[i] + k] (0 where the row lacks the
 * column).  Arrays: ROW = rowptr, COL = colids, VAL = values, CLUSTER_SZ,
 * ROWPTR_VAL; info: rows = CSR rows, nnz = nnzc, extra = [clusters, nnzv,
 * max_cluster_sz (at least 256, as the reference starts it)].  Replaces the
 * host struct consumed and produced by LeSpGEMM_VLength. */
spops_status_t spops_vlcluster_create(spops_context_t ctx, spops_matrix_t* M, int64_t csr_rows, int64_t clusters,
                                      int64_t cols, int64_t nnzc, int64_t nnzv, const void* cluster_sz,
                                      const void* rowptr, const void* colids, const void* rowptr_val,
                                      const void* values, spops_index_t itype, spops_value_t vtype, spops_mem_t mem);
/* csr_to_vlength_cluster (sparse_conversion.h:1640-1765): cluster i is rows
 * offsets[i] .. offsets[i+1] (host int64, from 0 to rows).  Each cluster's
 * columns are ascending (the reference lists them in hash-map order). */
spops_status_t spops_csr_to_vlength_cluster(spops_context_t ctx, spops_matrix_t csr, const int64_t* offsets,
                                            int64_t clusters, spops_matrix_t* cluster);
/* vlength_cluster2csr (sparse_conversion.h:1777-1862): rows in cluster
 * order, each row's entries in its cluster's column order, exact zeros
 * dropped. */
spops_status_t spops_vlength_cluster_to_csr(spops_context_t ctx, spops_matrix_t cluster, spops_matrix_t* csr);
/* LeSpGEMM_VLength (spgemm.h:175-180; kernel 3 rules, spgemm_Vlength_mixed.cpp)
 * C = A * B with A clustered: C in A's clusters, the cluster's columns
 * ascending, columns whose values all fall below 1e-12 dropped on the dense
 * and sorted paths, as the reference does.  l2_budget_bytes: the dense rule's
 * budget (the reference's CPU_L2CACHE_SIZE * mixed_l2_fraction).  A's exact
 * zeros take no part in C's structure. */
spops_status_t spops_spgemm_vlength(spops_context_t ctx, spops_matrix_t A_cluster, spops_matrix_t B,
                                    int32_t sort_output, double l2_budget_bytes, spops_matrix_t* C_cluster,
                                    spops_spgemm_stats_t* stats);

/* ------------------------------------------------------ no allocation */
/* y = alpha*A*x + beta*y for a CSR matrix given by device pointers, without
 * allocating any device memory.  No counterpart in the reference: it is for
 * callers that cannot call cudaMalloc at this point (a process whose device
 * memory is reserved up front by a pool, a plug-in or callback that must not
 * touch the allocator, a latency-bound loop that cannot take an allocation's
 * synchronisation).  Scratch lives in one fixed 4 MiB device array of the
 * library (held by every GPU that loads it until exit), which limits nnz to
 * 134,217,728 (larger: SPOPS_ERR_TOO_LARGE, nothing launched).  The first call
 * on a device (per CUDA context) looks that array up: make it before any
 * stream capture begins.  Calls whose work overlaps on the GPU race on the
 * array.  The row pointer is checked on the device first (row_offset[0] == 0,
 * non-decreasing, row_offset[rows] == nnz); a bad one is reported as
 * SPOPS_ERR_INVALID with y untouched.  Out-of-range column indices are
 * skipped and reported (SPOPS_ERR_INVALID).  Synchronises `stream` (a
 * cudaStream_t, may be NULL) before returning. */
spops_status_t spops_csr_spmv_noalloc(int64_t rows, int64_t cols, int64_t nnz, const void* row_offset,
                                      const void* col_index, const void* values, spops_index_t itype,
                                      spops_value_t vtype, double alpha, const void* x, double beta, void* y,
                                      void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SPARSEOPS_B200_H */
