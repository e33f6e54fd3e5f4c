"""Write the golden fixtures in this directory from the REFERENCE itself.

    python tests/golden/make_golden.py      (needs oracle/_ref, i.e. `make -C oracle ref`)

Every array in golden.npz is an output of the reference SparseOps library,
compiled from its own sources (oracle/Makefile) and called through
oracle/ref_harness.cpp, on small seeded synthetic inputs (sparseops_b200.synth).
The reference ships no golden vectors or known-answer tests of its own
(its SpGEMM goldens and SuiteSparse inputs are not part of the repository), so
these fixtures pin the oracle's restatement (tests/test_oracle_golden.py) and,
through the oracle, the device kernels.
"""
from __future__ import annotations

import os
import tempfile
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import Reference  # noqa: E402
from sparseops_b200 import synth  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz")


def sort_rows(rp, ci, v):
    ci, v = ci.copy(), v.copy()
    for r in range(len(rp) - 1):
        a, b = rp[r], rp[r + 1]
        o = np.argsort(ci[a:b], kind="stable")
        ci[a:b], v[a:b] = ci[a:b][o], v[a:b][o]
    return ci, v


def mtx_cases():
    """Matrix Market texts covering the reader's rules (banner case, comment
    lines, a size line after a blank line, CRLF, symmetric / skew / pattern /
    integer fields, duplicates, zero rows) and values that take every
    conversion path (exact fast path, double-double, exact midpoints)."""
    rng = np.random.default_rng(77)
    cases = []
    vals = ["1", "-2.5", "+3e2", "4.0E-3", "0.1", "1e-320", "2.4703282292062328e-324", "9007199254740993",
            "1.7976931348623157e308", "123456789012345678901234567890e-10", "-0", "7.0000000000000000000001",
            "1.00000000000000011102230246251565404236316680908203125", "6.02214076e23", ".5", "5."]
    lines = ["%%MatrixMarket matrix coordinate real general", "% a comment", "%", "6 5 %d" % (len(vals) + 4)]
    ents = [(1 + (i % 6), 1 + (i * 3 % 5), v) for i, v in enumerate(vals)]
    ents += [(2, 2, "1.5"), (2, 2, "-1.5"), (6, 5, "%.17g" % rng.standard_normal()), (1, 1, "0.25")]
    lines += ["%d %d %s" % e for e in ents]
    cases.append("\n".join(lines) + "\n")
    # symmetric, upper-case words, CRLF, a blank line before a split size line
    n, ent = 40, []
    for i in range(120):
        r, c = int(rng.integers(1, n + 1)), int(rng.integers(1, n + 1))
        r, c = max(r, c), min(r, c)
        ent.append("%d %d %.17g" % (r, c, rng.standard_normal() * 10.0 ** rng.integers(-30, 30)))
    cases.append("%%MatrixMarket MATRIX Coordinate REAL Symmetric\r\n%c\r\n\r\n  40 40\r\n120\r\n" +
                 "\r\n".join(ent) + "\r\n")
    # pattern general with duplicates and extra trailing tokens after the last entry
    pat = ["%d %d" % (int(rng.integers(1, 30)), int(rng.integers(1, 25))) for _ in range(200)]
    cases.append("%%MatrixMarket matrix coordinate pattern general\n29 24 200\n" + "\n".join(pat) + "\n7 7\n")
    # integer symmetric, tabs
    it = ["%d\t%d\t%d" % (max(a, b), min(a, b), v) for a, b, v in
          zip(rng.integers(1, 20, 60), rng.integers(1, 20, 60), rng.integers(-50, 50, 60))]
    cases.append("%%MatrixMarket matrix coordinate integer symmetric\n19 19 60\n" + "\n".join(it) + "\n")
    # skew-symmetric (not expanded by the reference)
    sk = ["%d %d %.6e" % (i + 2, i + 1, (i + 1) * 0.37) for i in range(10)]
    cases.append("%%MatrixMarket matrix coordinate real skew-symmetric\n11 11 10\n" + "\n".join(sk) + "\n")
    # no rows
    cases.append("%%MatrixMarket matrix coordinate real general\n0 0 0\n")
    # values around rounding midpoints and extremes, written with many digits
    mid = []
    for i in range(80):
        x = float(rng.standard_normal()) * 10.0 ** int(rng.integers(-300, 300))
        y = np.nextafter(x, np.inf)
        m = (np.longdouble(x) + np.longdouble(y)) / 2
        mid.append("%d %d %s" % (1 + i % 9, 1 + i % 7, np.format_float_scientific(m, unique=False, precision=60)))
    cases.append("%%MatrixMarket matrix coordinate real general\n9 7 80\n" + "\n".join(mid) + "\n")
    return cases


def main():
    R = Reference(threads=4)
    g = {}

    # ---- CSR SpMV: y = 0.8*A*x + 0.7*y0 (the reference's own test alpha/beta,
    # include/sparse_operation.h:123-124), kernel_flag 2
    for name, (rp, ci, v) in {
        "lap": synth.laplacian_2d(32),
        "pl": synth.powerlaw(2000, hi=300, seed=11),
    }.items():
        n = len(rp) - 1
        x = synth.uniform(n, 0)
        y0 = synth.uniform(n, 1)
        g[f"{name}_rp"], g[f"{name}_ci"], g[f"{name}_v"], g[f"{name}_x"], g[f"{name}_y0"] = rp, ci, v, x, y0
        g[f"{name}_y"] = R.spmv_csr(rp, ci, v, x, 0.8, 0.7, y0, flag=2)

    # ---- layouts on the power-law matrix
    rp, ci, v = g["pl_rp"], g["pl_ci"], g["pl_v"]
    n = len(rp) - 1
    for tag, (sig, C_, al) in {"a": (512, 32, 8), "b": (64, 4, 4), "c": (16384, 4, 4)}.items():
        h = R.fmt_build("sell_c_sigma", rp, ci, v, n, sig, C_, al)
        info = R.fmt_info(h)
        ro, cl = np.zeros(n, np.int32), np.zeros(info[2], np.int32)
        col, val = np.zeros(info[5], np.int32), np.zeros(info[5])
        R.fmt_copy(h, ro, cl, col, val)
        g[f"scs_{tag}_reorder"], g[f"scs_{tag}_chunk_len"] = ro, cl
        R.fmt_free(h)
    h = R.fmt_build("sell_c_R", rp, ci, v, n, 0, 32, 8)
    info = R.fmt_info(h)
    ro, cl = np.zeros(n, np.int32), np.zeros(info[0], np.int32)
    R.fmt_copy(h, ro, cl)
    g["scr_reorder"], g["scr_chunk_len"] = ro, cl
    R.fmt_free(h)
    h = R.fmt_build("sell", rp, ci, v, n, 0, 4, 4)
    info = R.fmt_info(h)
    w = np.zeros(info[0], np.int32)
    R.fmt_copy(h, w)
    g["sell_row_width"] = w
    R.fmt_free(h)

    # ---- DIA on the Laplacian and on a banded matrix
    for name, (brp, bci, bv) in {"lap": (g["lap_rp"], g["lap_ci"], g["lap_v"]),
                                 "band": synth.banded_random(1500, mean=6, band=8, seed=12)}.items():
        nn = len(brp) - 1
        h = R.fmt_build("dia", brp, bci, bv, nn, 10240, 0, 4)
        info = R.fmt_info(h)
        off = np.zeros(info[0], np.int64)
        data = np.zeros(info[0] * info[1])
        R.fmt_copy(h, off, None, None, data)
        g[f"dia_{name}_offsets"], g[f"dia_{name}_stride"] = off, np.int64(info[1])
        if name == "band":
            g["band_rp"], g["band_ci"], g["band_v"] = brp, bci, bv
        R.fmt_free(h)

    # ---- BSR structure
    for name, (brp, bci, bv, br, bc) in {"lap": (g["lap_rp"], g["lap_ci"], g["lap_v"], 16, 4),
                                         "pl": (rp, ci, v, 16, 8)}.items():
        nn = len(brp) - 1
        h = R.fmt_build("bsr", brp, bci, bv, nn, br, bc)
        info = R.fmt_info(h)
        brow, bcol = np.zeros(info[0] + 1, np.int32), np.zeros(info[2], np.int32)
        bdata = np.zeros(info[2] * br * bc)
        R.fmt_copy(h, brow, bcol, None, bdata)
        g[f"bsr_{name}_row_ptr"], g[f"bsr_{name}_col"] = brow, bcol
        R.fmt_free(h)

    # ---- LeSpGEMM preprocessing and kernel 3 on a planted-community matrix
    arp, aci, av = synth.planted_communities(1024, ncomm=32, mean=12.0, seed=13)
    brp, bci, bv = synth.transpose(arp, aci, av, 1024)
    g["sp_arp"], g["sp_aci"], g["sp_av"] = arp, aci, av
    sig = R.minhash(arp, aci, 64, 7)
    g["sp_sig"] = sig
    pi, pj, ps = R.lsh_pairs(arp, aci, 64, 16, 7, True)
    g["sp_pi"], g["sp_pj"], g["sp_ps"] = pi, pj, ps
    perm, offs = R.hc(arp, aci, pi, pj, ps, 8)
    g["sp_perm"], g["sp_offsets"] = perm, offs
    for so in (0, 1):
        c = R.spgemm_kernel3((arp, aci, av), (brp, bci, bv, 1024), perm, offs, sort_output=bool(so))
        cci, cv = sort_rows(c["rp"], c["ci"], c["v"])
        g[f"sp_c{so}_rp"], g[f"sp_c{so}_ci"], g[f"sp_c{so}_v"] = c["rp"], cci, cv
        g[f"sp_c{so}_dense"] = np.int64(c["dense_clusters"])
    # row-wise LeSpGEMM (kernels 1-3, sorted) and HashSpGEMMTopK on the same matrix
    for kf in (1, 2, 3):
        c = R.spgemm_rowwise((arp, aci, av), (brp, bci, bv, 1024), kf, True)
        g[f"rw{kf}_rp"], g[f"rw{kf}_ci"], g[f"rw{kf}_v"] = c["rp"], c["ci"], c["v"]
    for f32 in (0, 1):
        c = R.spgemm_topk(arp, aci, 1024, 6, bool(f32))
        g[f"topk{f32}_rp"], g[f"topk{f32}_ci"], g[f"topk{f32}_v"] = c["rp"], c["ci"], c["v"]
    # a bucket larger than 256 rows (window rule): 400 identical rows
    rp2 = np.arange(0, 401 * 3, 3, dtype=np.int64)
    ci2 = np.tile(np.array([5, 17, 99], np.int64), 400)
    pi2, pj2, ps2 = R.lsh_pairs(rp2, ci2, 64, 16, 7, True)
    g["big_pi"], g["big_pj"], g["big_ps"] = pi2, pj2, ps2

    # ---- transpose (csr_transpose: duplicates summed, exact zeros dropped)
    brp, bci, bv = g["band_rp"], g["band_ci"], g["band_v"]
    trp, tci, tv = R.csr_transpose(brp.astype(np.int64), bci.astype(np.int64), bv, len(brp) - 1)
    tci, tv = sort_rows(trp, tci, tv)
    g["tr_rp"], g["tr_ci"], g["tr_v"] = trp, tci, tv

    # ---- COO -> CSR (coo_to_csr, plain and with sum_csr_duplicates):
    # duplicates in random file order, values that cancel exactly
    rng = np.random.default_rng(77)
    n, nc, m = 300, 60, 4000
    ri = rng.integers(0, n, m).astype(np.int64)
    ci = rng.integers(0, nc, m).astype(np.int64)
    cv = rng.integers(-3, 4, m).astype(np.float64) * 0.25
    g["coo_ri"], g["coo_ci"], g["coo_v"], g["coo_shape"] = ri, ci, cv, np.array([n, nc], np.int64)
    for compact in (0, 1):
        crp, cci, ccv = R.coo_to_csr(n, nc, ri, ci, cv, bool(compact))
        g[f"coo_rp{compact}"], g[f"coo_csr_ci{compact}"], g[f"coo_csr_v{compact}"] = crp, cci, ccv

    # ---- structure features (MTX::MtxLoad + CalculateFeatures on the matrix
    # written as a general real Matrix Market file): rectangular random,
    # square with partly mirrored entries, banded with mixed magnitudes
    rng = np.random.default_rng(91)
    cases = []
    rp, ci, cv = [0], [], []
    for r in range(180):
        cols = np.sort(rng.choice(150, int(rng.integers(0, 9)), replace=False))
        ci += list(cols)
        cv += list(rng.choice([-4.0, -0.5, 0.125, 1.0, 3.0, 250.0, 0.0], len(cols)))
        rp.append(len(ci))
    cases.append((np.array(rp), np.array(ci), np.array(cv), 150))
    ent = {}
    for _ in range(900):
        r, c = int(rng.integers(0, 120)), int(rng.integers(0, 120))
        x = float(rng.choice([-3.0, -0.5, 0.25, 1.0, 7.0]))
        ent[(r, c)] = x
        if rng.random() < 0.6:
            ent[(c, r)] = x if rng.random() < 0.75 else x + 0.5
    for i in range(0, 120, 2):
        ent[(i, i)] = 40.0
    keys = sorted(ent)
    rp = np.zeros(121, np.int64)
    for r, _ in keys:
        rp[r + 1] += 1
    cases.append((np.cumsum(rp), np.array([c for _, c in keys]), np.array([ent[k] for k in keys]), 120))
    rp, ci, cv = [0], [], []
    for r in range(400):
        for d in (-3, -1, 0, 1, 7):
            if 0 <= r + d < 400 and rng.random() < 0.9:
                ci.append(r + d)
                cv.append(float(rng.choice([0.001, 0.5, 2.0, 1000.0])) * (1 if d else 5))
        rp.append(len(ci))
    cases.append((np.array(rp), np.array(ci), np.array(cv), 400))
    for k, (frp, fci, fv, fnc) in enumerate(cases):
        g[f"feat{k}_rp"], g[f"feat{k}_ci"], g[f"feat{k}_v"] = frp.astype(np.int64), fci.astype(np.int64), fv
        g[f"feat{k}_nc"] = np.int64(fnc)
        g[f"feat{k}_out"] = R.features(frp, fci, fv, fnc)

    # ---- tile features (MtxLoad's tile counts, CalculateTilesFeatures and
    # CalculateTilesExtraFeatures on the 256 x 256 grid): the three matrices
    # above and a 3000 x 2500 one with uneven blocks, unsorted rows and
    # repeated entries
    rng = np.random.default_rng(92)
    rp, ci = [0], []
    for r in range(3000):
        k = int(rng.integers(0, 30)) if rng.random() < 0.9 else int(rng.integers(100, 400))
        cols = list(rng.integers(0, 2500, k))
        if k and rng.random() < 0.2:
            cols.append(cols[0])
        ci += cols
        rp.append(len(ci))
    tcases = cases + [(np.array(rp), np.array(ci), np.ones(len(ci)), 2500)]
    g["tile3_rp"], g["tile3_ci"] = np.array(rp, np.int64), np.array(ci, np.int64)
    g["tile3_nc"] = np.int64(2500)
    for k, (frp, fci, fv, fnc) in enumerate(tcases):
        sc, ti, td, bi, bd = R.tile_features(frp, fci, fv, fnc)
        g[f"tile{k}_sc"], g[f"tile{k}_ti"], g[f"tile{k}_td"], g[f"tile{k}_bi"], g[f"tile{k}_bd"] = sc, ti, td, bi, bd

    # ---- Matrix Market files through the reference's read_csr_matrix
    for k, text in enumerate(mtx_cases()):
        with tempfile.NamedTemporaryFile("wb", suffix=".mtx", delete=False) as f:
            f.write(text.encode())
            path = f.name
        g[f"mtx{k}_text"] = np.frombuffer(text.encode(), np.uint8)
        for compact in (0, 1):
            for f32 in (0, 1):
                c = R.read_csr(path, compact=bool(compact), f32=bool(f32))
                for key in ("rp", "ci", "v"):
                    g[f"mtx{k}_{compact}{f32}_{key}"] = c[key]
        os.unlink(path)

    np.savez_compressed(OUT, **g)
    print(OUT, os.path.getsize(OUT), "bytes,", len(g), "arrays")


if __name__ == "__main__":
    main()
