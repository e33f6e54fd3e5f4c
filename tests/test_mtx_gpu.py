"""Matrix Market files read on the device (spops_mtx_*) against the
reference's own read_csr_matrix (golden fixtures: compact 0/1, FP64/FP32
values, bit for bit), the COO entry order against a plain restatement of the
reference's reading rules with Python's correctly rounded float(), a large
random file, and the refusals."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NCASES = 7


def _write(tmp_path, text, name="m.mtx"):
    p = tmp_path / name
    p.write_bytes(text if isinstance(text, bytes) else text.encode())
    return str(p)


def _py_coo(text):
    """The reference's reading rules: banner, '%' lines, size line (or the next
    three numbers after a blank one), nnz entries, symmetric expansion."""
    lines = text.split("\n")
    words = lines[0].split()
    field, symm = words[3].lower(), words[4].lower()
    i = 1
    while i < len(lines) and lines[i].startswith("%"):
        i += 1
    size = lines[i].split()
    if len(size) >= 3:
        rows, cols, nnz = (int(t) for t in size[:3])
        rest = "\n".join(lines[i + 1:]).split()
    else:
        toks = "\n".join(lines[i + 1:]).split()
        rows, cols, nnz = (int(t) for t in toks[:3])
        rest = toks[3:]
    per = 2 if field == "pattern" else 3
    r, c, v = [], [], []
    for e in range(nnz):
        a, b = int(rest[per * e]) - 1, int(rest[per * e + 1]) - 1
        x = 1.0 if per == 2 else float(rest[per * e + 2])
        r.append(a), c.append(b), v.append(x)
        if symm == "symmetric" and a != b:
            r.append(b), c.append(a), v.append(x)
    return rows, cols, np.array(r, np.int64), np.array(c, np.int64), np.array(v)


@pytest.mark.parametrize("k", range(NCASES))
@pytest.mark.parametrize("compact", [0, 1])
@pytest.mark.parametrize("f32", [0, 1])
def test_golden_csr(cuda, golden, tmp_path, k, compact, f32):
    from sparseops_b200 import read_csr_matrix
    g = golden
    text = g[f"mtx{k}_text"].tobytes()
    path = _write(tmp_path, text)
    vt = np.float32 if f32 else np.float64
    for it in (np.int32, np.int64):
        rp, ci, v = read_csr_matrix(path, bool(compact), it, vt).host()
        assert np.array_equal(rp.astype(np.int64), g[f"mtx{k}_{compact}{f32}_rp"])
        assert np.array_equal(ci.astype(np.int64), g[f"mtx{k}_{compact}{f32}_ci"])
        # duplicates of +inf and -inf sum to NaN (whose sign the host and the GPU choose differently)
        assert np.array_equal(v.astype(np.float64), g[f"mtx{k}_{compact}{f32}_v"], equal_nan=True)


@pytest.mark.parametrize("k", range(NCASES))
def test_parse_from_memory_and_coo_order(cuda, golden, k):
    import ctypes as C
    from sparseops_b200 import DeviceCSR, default_context
    from sparseops_b200._lib import call, i64, vp
    from sparseops_b200.spops import _Handle
    text = golden[f"mtx{k}_text"].tobytes()
    ctx = default_context()
    out = vp()
    call("spops_mtx_parse_coo", ctx.handle, text, i64(len(text)), C.c_int(1), C.c_int(1), C.byref(out))
    h = _Handle(ctx, out)
    info = h.info()
    rows, cols, r, c, v = _py_coo(text.decode())
    assert (info.rows, info.cols, info.nnz) == (rows, cols, len(r)) or rows == 0
    got = [np.empty(info.nnz, np.int64), np.empty(info.nnz, np.int64), np.empty(info.nnz)]
    for arr, which in zip(got, (0, 1, 2)):
        if len(arr):
            call("spops_matrix_download", ctx.handle, h.handle, which, vp(arr.ctypes.data), i64(len(arr)))
    assert np.array_equal(got[0], r) and np.array_equal(got[1], c) and np.array_equal(got[2], v, equal_nan=True)
    out2 = vp()
    call("spops_mtx_parse_csr", ctx.handle, text, i64(len(text)), C.c_int(1), C.c_int(1), C.c_int32(0),
         C.byref(out2))
    m = DeviceCSR(_Handle(ctx, out2), int(info.rows), int(info.cols))
    assert np.array_equal(m.host()[0], golden[f"mtx{k}_00_rp"])
    assert np.array_equal(m.host()[2], golden[f"mtx{k}_00_v"], equal_nan=True)


def test_large_random_file(cuda, tmp_path):
    """300,000 entries written at several precisions, general and symmetric."""
    from sparseops_b200 import read_coo_matrix
    rng = np.random.default_rng(8)
    n, nnz = 5000, 300000
    r = rng.integers(1, n + 1, nnz)
    c = rng.integers(1, n + 1, nnz)
    x = rng.standard_normal(nnz) * 10.0 ** rng.integers(-200, 200, nnz)
    fmts = ["%.17g", "%.6g", "%.25e", "%.3f"]
    body = "\n".join("%d %d %s" % (a, b, fmts[i % 4] % y) for i, (a, b, y) in enumerate(zip(r, c, x)))
    for symm in ("general", "symmetric"):
        if symm == "symmetric":
            lo, hi = np.minimum(r, c), np.maximum(r, c)
            body = "\n".join("%d %d %s" % (a, b, fmts[i % 4] % y) for i, (a, b, y) in enumerate(zip(hi, lo, x)))
        text = "%%%%MatrixMarket matrix coordinate real %s\n%d %d %d\n%s\n" % (symm, n, n, nnz, body)
        path = _write(tmp_path, text, symm + ".mtx")
        m = read_coo_matrix(path, np.int64, np.float64)
        rows, cols, er, ec, ev = _py_coo(text)
        assert m.num_nnzs == len(er)
        assert np.array_equal(m.row_index, er) and np.array_equal(m.col_index, ec)
        assert np.array_equal(m.values.view(np.uint64), ev.view(np.uint64))


@pytest.mark.parametrize("order", ["random", "rows_sorted", "symmetric"])
def test_large_csr_no_compact(cuda, tmp_path, order):
    """CSR without the duplicate summation, built straight from the parsed
    entries: row offsets from counts, entries in file order within a row (a
    stable sort by row), for files in random row order, already sorted by row
    (no sort needed) and symmetric (mirror copies placed after their entry)."""
    from sparseops_b200 import read_csr_matrix
    rng = np.random.default_rng(31)
    n, nnz = 7000, 250000
    r, c = rng.integers(1, n + 1, nnz), rng.integers(1, n + 1, nnz)
    if order == "rows_sorted":
        r = np.sort(r)
    if order == "symmetric":
        r, c = np.maximum(r, c), np.minimum(r, c)
    x = rng.standard_normal(nnz)
    symm = "symmetric" if order == "symmetric" else "general"
    body = "\n".join("%d %d %.17g" % (a, b, y) for a, b, y in zip(r, c, x))
    text = "%%%%MatrixMarket matrix coordinate real %s\n%d %d %d\n%s\n" % (symm, n + 3, n, nnz, body)
    path = _write(tmp_path, text, order + ".mtx")
    _, _, er, ec, ev = _py_coo(text)
    perm = np.argsort(er, kind="stable")
    want_rp = np.zeros(n + 4, np.int64)
    np.cumsum(np.bincount(er, minlength=n + 3), out=want_rp[1:])
    for it, vt in ((np.int32, np.float64), (np.int64, np.float32)):
        rp, ci, v = read_csr_matrix(path, False, it, vt).host()
        assert np.array_equal(rp.astype(np.int64), want_rp)
        assert np.array_equal(ci.astype(np.int64), ec[perm])
        assert np.array_equal(v, ev[perm].astype(vt))


@pytest.mark.parametrize("text,status", [
    ("%%MatrixMarket matrix coordinate real\n2 2 1\n1 1 1\n", 1),           # banner of four words
    ("%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 1\n", 1),   # no banner
    ("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n", 2),     # dense arrays are not read
    ("%%MatrixMarket matrix coordinate complex general\n2 2 1\n1 1 1 0\n", 2),
    ("%%MatrixMarket matrix coordinate real hermitian\n2 2 1\n1 1 1\n", 1),  # invalid as mm_is_valid says
    ("%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1.5\n", 1),  # fewer entries than announced
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 3 1.5\n", 1),  # column outside the size
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 1.5x\n", 1),  # not a number
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 0x1p3\n", 1),  # hexadecimal values refused
])
def test_refusals(cuda, tmp_path, text, status):
    from sparseops_b200 import SpOpsError, read_csr_matrix
    with pytest.raises(SpOpsError) as e:
        read_csr_matrix(_write(tmp_path, text))
    assert e.value.status == status


def test_missing_file(cuda, tmp_path):
    from sparseops_b200 import SpOpsError, read_csr_matrix
    with pytest.raises(SpOpsError):
        read_csr_matrix(str(tmp_path / "absent.mtx"))


def _coo_from_memory(text):
    import ctypes as C
    from sparseops_b200._lib import call, i64, vp
    from sparseops_b200.formats import _Handle, default_context
    ctx = default_context()
    out = vp()
    call("spops_mtx_parse_coo", ctx.handle, text, i64(len(text)), C.c_int(1), C.c_int(1), C.byref(out))
    h = _Handle(ctx, out)
    n = int(h.info().nnz)
    got = [np.empty(n, np.int64), np.empty(n, np.int64), np.empty(n)]
    for arr, which in zip(got, (0, 1, 2)):
        if n:
            call("spops_matrix_download", ctx.handle, h.handle, which, vp(arr.ctypes.data), i64(n))
    return got


@pytest.mark.parametrize("case", ["long_comments", "size_line_at_prefix_end", "many_chunks"])
def test_path_read_matches_memory(cuda, tmp_path, case):
    """Reading from a path (header from a growing prefix, entries streamed in
    4 MiB chunks by several reader threads) gives the same COO as parsing the
    same bytes from host memory: a header longer than the first 64 KiB
    prefix, a size line cut by that prefix, and a 20 MB file of many chunks."""
    from sparseops_b200 import read_coo_matrix
    rng = np.random.default_rng(21)
    head = "%%MatrixMarket matrix coordinate real general\n"
    if case == "long_comments":
        head += "".join("%% comment line %06d %s\n" % (i, "x" * 60) for i in range(1500))
        nnz = 2000
    elif case == "size_line_at_prefix_end":
        pad = 65536 - len(head) - 4  # the size line starts 4 bytes before the prefix ends
        head += "%" + "y" * (pad - 2) + "\n"
        nnz = 2000
    else:
        nnz = 700_000
    n = 100_000
    r, c = rng.integers(1, n + 1, nnz), rng.integers(1, n + 1, nnz)
    x = rng.standard_normal(nnz) * 10.0 ** rng.integers(-30, 30, nnz)
    import io
    buf = io.StringIO()
    np.savetxt(buf, np.column_stack([r, c, x]), fmt="%d %d %.17g")
    text = (head + "%d %d %d\n" % (n, n, nnz) + buf.getvalue()).encode()
    if case == "size_line_at_prefix_end":
        assert text.index(b"%d %d %d\n" % (n, n, nnz)) == 65532
    path = _write(tmp_path, text)
    m = read_coo_matrix(path, np.int64, np.float64)
    er, ec, ev = _coo_from_memory(text)
    assert m.num_nnzs == nnz
    assert np.array_equal(m.row_index, er) and np.array_equal(m.col_index, ec)
    assert np.array_equal(m.values.view(np.uint64), ev.view(np.uint64))
    assert np.array_equal(er, r - 1) and np.array_equal(ec, c - 1)
    assert np.array_equal(ev, x)
