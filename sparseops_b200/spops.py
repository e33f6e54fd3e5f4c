"""Host-side mirror of the reference's SpOps API over the C ABI.

Names, argument order and meaning follow the reference's include/SpOps.h
templates: ``SpOps_csr(alpha, A, x, beta, y)`` computes y = alpha*A*x + beta*y
(src/spmv_csr.cpp:165).  Matrices are the reference's structs
(include/sparse_format.h) with their arrays held either in host numpy arrays
(uploaded once, like the C++ shim's device cache) or in CUDA tensors
(borrowed, zero copy).  Vectors may be CUDA tensors (device path) or numpy
arrays (host path: x is uploaded, y downloaded, per call).

torch is used only for device memory and the current stream.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import call, dbl, i64, vp

try:  # torch is plumbing: device memory, streams
    import torch
except ImportError:  # pragma: no cover
    torch = None


def _is_cuda_tensor(a) -> bool:
    return torch is not None and isinstance(a, torch.Tensor) and a.is_cuda


def _ptr(a):
    if a is None:
        return None
    if _is_cuda_tensor(a) or (torch is not None and isinstance(a, torch.Tensor) and a.is_contiguous()):
        return vp(a.data_ptr())
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(vp)
    raise TypeError(f"unsupported array type {type(a)}")


def _itype(a) -> int:
    dt = a.dtype
    if dt in (np.int32, getattr(torch, "int32", None)):
        return 0
    if dt in (np.int64, getattr(torch, "int64", None)):
        return 1
    raise TypeError(f"index arrays must be int32 or int64, got {dt}")


def _vtype(a) -> int:
    dt = a.dtype
    if dt in (np.float32, getattr(torch, "float32", None)):
        return 0
    if dt in (np.float64, getattr(torch, "float64", None)):
        return 1
    raise TypeError(f"value arrays must be float32 or float64, got {dt}")


class Context:
    """A library context bound to one device and one stream (spops_create)."""

    def __init__(self, device: int = 0, stream: int | None = None):
        h = vp()
        call("spops_create", C.byref(h), int(device), vp(stream) if stream else None)
        self.handle = h
        self.device = int(device)
        self._stream = stream

    def set_stream(self, stream: int | None) -> None:
        if stream != self._stream:
            call("spops_set_stream", self.handle, vp(stream) if stream else None)
            self._stream = stream

    def follow_torch(self) -> "Context":
        """Enqueue on torch's current stream for this device."""
        if torch is not None and torch.cuda.is_available():
            self.set_stream(torch.cuda.current_stream(self.device).cuda_stream)
        return self

    def synchronize(self) -> None:
        call("spops_synchronize", self.handle)

    def check_device(self) -> int:
        """Raise SpOpsError(SPOPS_ERR_TIMEOUT) if a bounded device wait gave up."""
        f = C.c_int32()
        call("spops_check_device", self.handle, C.byref(f))
        return f.value

    def set_option(self, key: str, value: int) -> None:
        call("spops_set_option", self.handle, key.encode(), i64(int(value)))

    def close(self) -> None:
        if getattr(self, "handle", None):
            h, self.handle = self.handle, None
            _lib.release("spops_destroy", h)

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass


_CTX: dict[int, Context] = {}


def default_context(device: int | None = None) -> Context:
    if device is None:
        device = torch.cuda.current_device() if (torch is not None and torch.cuda.is_available()) else 0
    ctx = _CTX.get(device)
    if ctx is None:
        ctx = _CTX[device] = Context(device)
    return ctx.follow_torch()


class _Handle:
    """Owns one spops_matrix_t and keeps its borrowed arrays alive."""

    def __init__(self, ctx: Context, handle, keep=()):
        self.ctx, self.handle, self._keep = ctx, handle, keep

    def __del__(self):  # pragma: no cover
        try:
            _lib.release("spops_matrix_destroy", self.handle, self.ctx)
        except Exception:
            pass

    def info(self) -> _lib.MatrixInfo:
        out = _lib.MatrixInfo()
        call("spops_matrix_info", self.handle, C.byref(out))
        return out

    def device_bytes(self) -> int:
        b = C.c_int64()
        call("spops_matrix_device_bytes", self.handle, C.byref(b))
        return b.value


class Matrix_Features:
    """Common fields of every reference format (include/sparse_format.h:49-69)."""

    num_rows: int
    num_cols: int
    num_nnzs: int
    kernel_flag: int = 1

    def __init__(self):
        self._h: _Handle | None = None
        self.kernel_flag = 1


class CSR_Matrix(Matrix_Features):
    """Compressed sparse row matrix (include/sparse_format.h:95-104).

    Arrays may be numpy (host, uploaded on first use) or CUDA tensors
    (device, borrowed).  ``kernel_flag`` is accepted for API compatibility;
    every value selects the same device kernel.
    """

    def __init__(self, num_rows, num_cols, row_offset, col_index, values, kernel_flag: int = 1):
        super().__init__()
        self.num_rows, self.num_cols = int(num_rows), int(num_cols)
        self.row_offset, self.col_index, self.values = row_offset, col_index, values
        self.num_nnzs = int(len(col_index))
        self.kernel_flag = kernel_flag

    def device(self, ctx: Context | None = None) -> _Handle:
        """The device-resident handle (created, and analysed, on first use)."""
        if self._h is None:
            ctx = ctx or default_context()
            on_dev = _is_cuda_tensor(self.values)
            h = vp()
            call("spops_csr_create", ctx.handle, C.byref(h), i64(self.num_rows), i64(self.num_cols),
                 i64(self.num_nnzs), _ptr(self.row_offset), _ptr(self.col_index), _ptr(self.values),
                 _itype(self.col_index), _vtype(self.values), 0 if on_dev else 1)
            self._h = _Handle(ctx, h, (self.row_offset, self.col_index, self.values) if on_dev else ())
            call("spops_matrix_analyse", ctx.handle, h)
        return self._h

    def touch(self) -> None:
        """Values were changed in place (same pattern)."""
        if self._h is not None:
            call("spops_matrix_touch", self._h.handle)


def _spmv(alpha, A: Matrix_Features, x, beta, y):
    h = A.device()
    ctx = h.ctx
    if _is_cuda_tensor(x):
        if not _is_cuda_tensor(y):
            raise TypeError("x is a CUDA tensor but y is not")
        ctx.follow_torch()
        call("spops_spmv", ctx.handle, dbl(alpha), h.handle, _ptr(x), dbl(beta), _ptr(y))
    else:
        if not (isinstance(x, np.ndarray) and isinstance(y, np.ndarray)):
            raise TypeError("x and y must both be CUDA tensors or both numpy arrays")
        call("spops_spmv_host", ctx.handle, dbl(alpha), h.handle, _ptr(np.ascontiguousarray(x)), dbl(beta),
             _ptr(y))
    return y


def spmv_host_async(alpha, A: Matrix_Features, x, beta, y):
    """y = alpha*A*x + beta*y with host x and y, queued (spops_spmv_host_async):
    returns before y is written.  For a stream of independent requests with
    page-locked x and y (torch CPU tensors from pin_memory()), consecutive
    calls overlap one request's upload with the previous one's SpMV and
    download.  Keep x unchanged and y unread until spmv_host_wait()."""
    h = A.device()
    call("spops_spmv_host_async", h.ctx.handle, dbl(alpha), h.handle, _ptr(x), dbl(beta), _ptr(y))
    return y


def spmv_host_wait(A: Matrix_Features = None, ctx=None):
    """Completes every spmv_host_async call queued on the matrix's (or the
    given, or the default) context."""
    ctx = A.device().ctx if A is not None else (ctx or default_context())
    call("spops_spmv_host_wait", ctx.handle)


class DeviceCSR(CSR_Matrix):
    """A CSR matrix produced on the device (conversion or product result),
    held by its handle; host copies of the arrays are made on first access."""

    def __init__(self, handle: _Handle, rows: int, cols: int):
        info = handle.info()
        super().__init__(rows, cols, None, np.zeros(0, np.int64), None)
        self.num_nnzs = int(info.nnz)
        self._h = handle
        self._it, self._vt = int(info.index_type), int(info.value_type)
        self._host = None

    def host(self):
        """(row_offset, col_index, values) as numpy arrays."""
        if self._host is None:
            h = self._h
            idx = np.int32 if self._it == 0 else np.int64
            val = np.float32 if self._vt == 0 else np.float64
            arrs = (np.empty(self.num_rows + 1, idx), np.empty(self.num_nnzs, idx), np.empty(self.num_nnzs, val))
            for arr, which in zip(arrs, (0, 1, 2)):
                if len(arr):
                    call("spops_matrix_download", h.ctx.handle, h.handle, which, vp(arr.ctypes.data), i64(len(arr)))
            self._host = arrs
        return self._host

    row_offset = property(lambda self: self.host()[0], lambda self, v: None)
    col_index = property(lambda self: self.host()[1] if self._h is not None else np.zeros(0), lambda self, v: None)
    values = property(lambda self: self.host()[2] if self._h is not None else None, lambda self, v: None)

    def device(self, ctx=None):
        return self._h


def SpOps_csr(alpha, csr: CSR_Matrix, x, beta, y):
    """y = alpha*A*x + beta*y for a CSR matrix (reference src/spmv_csr.cpp:165)."""
    return _spmv(alpha, csr, x, beta, y)


def SpMM_csr(alpha, csr: CSR_Matrix, X, beta, Y):
    """Y = alpha*A*X + beta*Y for row-major X [cols x k], Y [rows x k] (CUDA
    tensors).  No reference counterpart; equals k SpOps_csr calls."""
    h = csr.device()
    ctx = h.ctx.follow_torch()
    k = X.shape[1]
    call("spops_spmm", ctx.handle, dbl(alpha), h.handle, _ptr(X), i64(X.stride(0)), i64(k), dbl(beta), _ptr(Y),
         i64(Y.stride(0)))
    return Y


class Batch:
    """Many CSR matrices in one persistent launch (spops_batch_*).

    ``X`` / ``Y`` are lists of CUDA tensors: vectors for k = 1, row-major
    [n x k] matrices otherwise.  ``tune()`` picks the form per matrix on the
    device; ``capture()`` records the launch in a CUDA graph that ``run()``
    replays."""

    def __init__(self, matrices, k: int = 1, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self.matrices = list(matrices)
        self.handles = [m.device(self.ctx) for m in self.matrices]
        arr = (vp * len(self.handles))(*[h.handle for h in self.handles])
        self.k = int(k)
        h = vp()
        call("spops_batch_create", self.ctx.handle, C.byref(h), i64(len(self.handles)), arr, i64(self.k))
        self.handle = h
        self._vecs = None

    def __del__(self):  # pragma: no cover
        try:
            _lib.release("spops_batch_destroy", getattr(self, "handle", None), self.ctx)
        except Exception:
            pass

    def set_vectors(self, X, Y):
        n = len(self.handles)
        xs = (vp * n)(*[vp(x.data_ptr()) for x in X])
        ys = (vp * n)(*[vp(y.data_ptr()) for y in Y])
        ldx = (C.c_int64 * n)(*[(x.stride(0) if x.dim() == 2 else 1) for x in X])
        ldy = (C.c_int64 * n)(*[(y.stride(0) if y.dim() == 2 else 1) for y in Y])
        call("spops_batch_set_vectors", self.handle, xs, ldx, ys, ldy)
        self._vecs = (list(X), list(Y))

    def tune(self, csr_only: bool = False):
        self.ctx.follow_torch()
        call("spops_batch_tune", self.ctx.handle, self.handle, C.c_int32(1 if csr_only else 0))

    def run(self, alpha: float = 1.0, beta: float = 0.0):
        self.ctx.follow_torch()
        call("spops_batch_run", self.ctx.handle, self.handle, dbl(alpha), dbl(beta))

    def capture(self, alpha: float = 1.0, beta: float = 0.0):
        self.ctx.follow_torch()
        call("spops_batch_capture", self.ctx.handle, self.handle, dbl(alpha), dbl(beta))

    def info(self):
        items = C.c_int64()
        ch = (C.c_int32 * len(self.handles))()
        kt = C.c_int32()
        call("spops_batch_info", self.handle, C.byref(items), ch, C.byref(kt))
        return items.value, list(ch), kt.value
