"""The learned storage-format selector: corpus, measurements and model fit.

    python -m sparseops_b200.selector collect DATA.json   # on a GPU: features + SpMV time of every candidate
    python -m sparseops_b200.selector fit DATA.json       # fit the tree, write csrc/selector_tree.h

The reference computes structure features and writes them out for a model
that lives outside the repository (src/sparse_features.cpp:642-1093, 1225);
this module is that model for this GPU.  The corpus is a fixed list of
seeded synthetic matrices of varied structure -- power-law rows of several
means and spreads, banded-plus-random rows, pure bands, 2-D Laplacians,
planted column communities, symmetric random graphs and grouped near-duplicate
rows.  For each one `collect` records the device features
(spops_matrix_features) and the time of one FP64 SpMV in every candidate
format of spops_select_format's timed mode: CSR, SELL-C-R (C = 32),
SELL-C-sigma (C = 32, sigma = 4096), CSR5, and DIA where its diagonals are
dense enough.  `fit` labels every matrix with its fastest format, fits a
small decision tree on the derived features below (every third matrix held
out), reports agreement with the timed choice and the time lost on the
held-out matrices, and writes the tree as a C table that
spops_select_format's mode 2 walks.
"""
from __future__ import annotations

import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TREE_HEADER = os.path.join(HERE, "csrc", "selector_tree.h")

# candidate formats (spops_format_t values) and their spops_convert parameters
CANDIDATES = {
    "csr": (0, {}),
    "sell_c_R": (5, {"chunk": 32, "alignment": 1, "layout": 1}),
    "sell_c_sigma": (4, {"chunk": 32, "sigma": 4096, "alignment": 1, "layout": 1}),
    "csr5": (8, {}),
    "dia": (6, {"alignment": 1}),
}

DERIVED = ("log2_rows", "log2_nnz", "ave_nnz_row", "cv_nnz_row", "max_over_ave_row", "gini_row", "diag_close_ratio",
           "dia_fill", "log2_ndiags", "nz_row_ratio", "p_ratio_row")


def derived(f: dict) -> list[float]:
    """The tree's inputs from spops_features_t (the C side computes the same,
    csrc/selector.cpp: derived_features)."""
    rows, cols, nnz, nd = float(f["rows"]), float(f["cols"]), float(f["nnz"]), float(f["ndiags"])
    ave = float(f["ave_nnz_row"])
    mn = min(rows, cols)
    return [
        math.log2(rows + 1.0),
        math.log2(nnz + 1.0),
        ave,
        float(f["std_nnz_row"]) / max(ave, 1e-12),
        float(f["max_nnz_row"]) / max(ave, 1e-12),
        float(f["gini_row"]),
        float(f["diag_close_ratio"]),
        nnz / (nd * mn) if nd > 0 and mn > 0 else 0.0,
        math.log2(nd + 1.0),
        float(f["nz_row_ratio"]),
        float(f["p_ratio_row"]),
    ]


def dia_allowed(f: dict) -> bool:
    """The timed mode's condition for trying DIA (csrc/features.cu)."""
    mn = min(f["rows"], f["cols"])
    return 0 < f["ndiags"] <= 10240 and f["nnz"] >= 0.25 * f["ndiags"] * mn


def _band(n: int, half: int, seed: int):
    """Pure band |i - j| <= half, values N(0, 1) (int32 indices)."""
    rng = np.random.default_rng(seed)
    i = np.repeat(np.arange(n, dtype=np.int64), 2 * half + 1)
    j = i + np.tile(np.arange(-half, half + 1, dtype=np.int64), n)
    keep = (j >= 0) & (j < n)
    i, j = i[keep], j[keep]
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(i, minlength=n), out=rp[1:])
    return rp.astype(np.int32), j.astype(np.int32), rng.standard_normal(len(j))


def corpus():
    """(name, generator) pairs; each generator returns (rp, ci, v, ncols)."""
    from . import synth
    out = []
    for n in (65536, 262144, 1048576):
        for m in (4, 16, 48):
            for s in (0.2, 0.7, 1.2):
                out.append((f"powerlaw n={n} mean={m} sigma={s}",
                            lambda n=n, m=m, s=s: (*synth.powerlaw(n, mu=math.log(m), sigma=s, lo=1, hi=20000,
                                                                   seed=int(1000 * s) + m), n)))
    for n in (65536, 524288):
        for mean in (8, 32):
            for band in (16, 512):
                out.append((f"banded_random n={n} mean={mean} band={band}",
                            lambda n=n, mean=mean, band=band: (*synth.banded_random(n, float(mean), band,
                                                                                    seed=mean + band), n)))
    for n, half in ((262144, 1), (262144, 4), (131072, 16), (65536, 64)):
        out.append((f"band n={n} half={half}", lambda n=n, half=half: (*_band(n, half, half), n)))
    for nx in (128, 256, 512, 1024, 2048):
        out.append((f"laplacian {nx}x{nx}", lambda nx=nx: (*synth.laplacian_2d(nx), nx * nx)))
    for n, ncomm in ((65536, 256), (524288, 2048)):
        out.append((f"planted n={n} ncomm={ncomm}",
                    lambda n=n, ncomm=ncomm: tuple(a.astype(np.int32) if a.dtype == np.int64 else a
                                                   for a in synth.planted_communities(n, ncomm=ncomm, seed=3)) + (n,)))
    for n, deg in ((131072, 8.0), (1048576, 32.0)):
        out.append((f"graph n={n} degree={deg}", lambda n=n, deg=deg: (*synth.symmetric_graph(n, deg, seed=11), n)))
    for group, width in ((32, 12), (8, 64), (64, 128)):
        def gen(group=group, width=width):
            rp, ci, v, nc = synth.grouped_rows(262144, group=group, width=width, mean=min(width, 24.0), seed=width)
            return rp.astype(np.int32), ci.astype(np.int32), v, nc
        out.append((f"grouped group={group} width={width}", gen))
    return out


def _time_spmv(op, reps=30, warm=3):
    import torch
    for _ in range(warm):
        op()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        op()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def collect(path: str) -> None:
    """Features and per-format SpMV times (ms) of every corpus matrix."""
    import torch
    from . import CSR_Matrix, default_context, synth
    from ._lib import call, dbl, vp
    from .formats import convert_to, matrix_features
    dev = torch.device("cuda", 0)
    ctx = default_context(0)
    rows = []
    for name, gen in corpus():
        rp, ci, v, nc = gen()
        n = len(rp) - 1
        A = CSR_Matrix(n, nc, torch.from_numpy(rp).to(dev), torch.from_numpy(ci).to(dev), torch.from_numpy(v).to(dev))
        f = matrix_features(A)
        x = torch.from_numpy(synth.uniform(nc, 7)).to(dev)
        y = torch.zeros(n, dtype=torch.float64, device=dev)
        times = {}
        for fmt, (_, params) in CANDIDATES.items():
            if fmt == "dia" and not dia_allowed(f):
                continue
            try:
                M = convert_to(A, fmt, **params)
                h = M.device(ctx)
                times[fmt] = _time_spmv(lambda: call("spops_spmv", ctx.handle, dbl(1.0), h.handle,
                                                     vp(x.data_ptr()), dbl(0.0), vp(y.data_ptr())))
                del M, h
            except Exception as e:  # a conversion refused (too large): not a candidate
                print(f"{name}: {fmt} skipped: {e}", file=sys.stderr)
        rows.append({"name": name, "features": f, "ms": times})
        print(f"{name}: " + ", ".join(f"{k} {t:.4f}" for k, t in times.items()), file=sys.stderr, flush=True)
        del A, x, y
        torch.cuda.empty_cache()
    with open(path, "w") as fh:
        json.dump({"device": torch.cuda.get_device_name(0), "rows": rows}, fh, indent=0)


def _labels(rows):
    return [min(r["ms"], key=r["ms"].get) for r in rows]


def fit(path: str, max_depth: int = 4, header: str = TREE_HEADER) -> dict:
    """Fit on two thirds of the corpus, evaluate on the rest, write the C table."""
    from sklearn.tree import DecisionTreeClassifier
    with open(path) as fh:
        data = json.load(fh)
    rows = data["rows"]
    X = np.array([derived(r["features"]) for r in rows])
    y = np.array([CANDIDATES[l][0] for l in _labels(rows)])
    held = np.arange(len(rows)) % 3 == 2
    clf = DecisionTreeClassifier(max_depth=max_depth, min_samples_leaf=2, random_state=0)
    clf.fit(X[~held], y[~held])
    code_of = {v[0]: k for k, v in CANDIDATES.items()}

    def report(mask):
        agree, regret = 0, []
        for r, xv, lab in zip(np.array(rows, dtype=object)[mask], X[mask], y[mask]):
            pred = code_of[int(clf.predict(xv[None, :])[0])]
            best = min(r["ms"].values())
            t = r["ms"].get(pred, float("inf"))
            agree += int(CANDIDATES[pred][0] == lab)
            regret.append(t / best)
        return {"matrices": int(mask.sum()), "agree": agree, "mean_time_over_best": float(np.mean(regret)),
                "max_time_over_best": float(np.max(regret))}
    ev = {"train": report(~held), "held_out": report(held), "device": data.get("device", ""),
          "labels": {k: int(np.sum(y == v[0])) for k, v in CANDIDATES.items()}}
    _write_header(clf, ev, header)
    return ev


def _write_header(clf, ev: dict, header: str) -> None:
    t = clf.tree_
    classes = clf.classes_
    nodes = []
    for k in range(t.node_count):
        if t.children_left[k] < 0:
            nodes.append((-1, 0.0, -1, -1, int(classes[int(np.argmax(t.value[k][0]))])))
        else:
            nodes.append((int(t.feature[k]), float(t.threshold[k]), int(t.children_left[k]),
                          int(t.children_right[k]), -1))
    ho = ev["held_out"]
    lines = [
        "// Decision tree of the learned format selector (spops_select_format mode 2).",
        "// Generated by sparseops_b200/selector.py from measured SpMV times; do not edit.",
        f"// Inputs: derived features {', '.join(DERIVED)}.",
        f"// Fitted on {ev['train']['matrices']} seeded matrices ({ev['device']}); on the "
        f"{ho['matrices']} held-out ones it picks the",
        f"// timed choice for {ho['agree']} and its SpMV takes {ho['mean_time_over_best']:.3f}x the best on average "
        f"({ho['max_time_over_best']:.3f}x at worst).",
        "#pragma once",
        "",
        "namespace spops {",
        "",
        "struct SelectorNode {",
        "  int feature;      // derived feature index, -1 for a leaf",
        "  double threshold; // go left when feature <= threshold",
        "  int left, right;  // child nodes",
        "  int format;       // spops_format_t of a leaf",
        "};",
        "",
        f"constexpr int kSelectorNodes = {len(nodes)};",
        "constexpr SelectorNode kSelectorTree[kSelectorNodes] = {",
    ]
    for f_, th, l, r, c in nodes:
        lines.append(f"    {{{f_}, {th!r}, {l}, {r}, {c}}},")
    lines += ["};", "", "}  // namespace spops", ""]
    with open(header, "w") as fh:
        fh.write("\n".join(lines))


def predict_table(xv) -> int:
    """Walk the committed C table (parsed from the header) for one derived
    feature vector: the format code the library's mode 2 returns."""
    nodes = []
    with open(TREE_HEADER) as fh:
        for line in fh:
            line = line.strip()
            if line.startswith("{") and line.endswith("},"):
                a = line[1:-2].split(",")
                nodes.append((int(a[0]), float(a[1]), int(a[2]), int(a[3]), int(a[4])))
    k = 0
    while nodes[k][0] >= 0:
        k = nodes[k][2] if xv[nodes[k][0]] <= nodes[k][1] else nodes[k][3]
    return nodes[k][4]


if __name__ == "__main__":
    if len(sys.argv) != 3 or sys.argv[1] not in ("collect", "fit"):
        raise SystemExit(__doc__)
    if sys.argv[1] == "collect":
        collect(sys.argv[2])
    else:
        print(json.dumps(fit(sys.argv[2]), indent=1))
