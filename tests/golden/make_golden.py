"""Generate tests/golden/golden.json from the reference itself.

    WMD_REFERENCE_DIR=<reference checkout> make -C oracle   # builds oracle/_ref/
    WMD_REFERENCE_DIR=<reference checkout> python tests/golden/make_golden.py

Needs the reference checkout (its data/ directory and its sources, compiled
in place into oracle/_ref/).  Records, at full FP64 precision:

* the d=3 known-answer sample (data/sample.mtx, data/v2.txt, data/r2.txt,
  the "small input" of the reference README) with the inputs themselves,
  through the fused solver, the nonfused solver (both lambda signs) and the
  Python reference main.py;
* every synthetic case of tests/golden/cases.py: generator digest plus the
  fused reference's output on one OpenMP thread (deterministic order), and
  main.py's output on the smaller ones.
"""
from __future__ import annotations

import importlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("WMD_REFERENCE_DIR", "")
if not REF or not os.path.isdir(REF):
    raise SystemExit("set WMD_REFERENCE_DIR to the reference checkout "
                     "(the directory holding sinkhorn_wmd_fused.cpp)")
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

import oracle  # noqa: E402
from oracle import oracle as O  # noqa: E402
from cases import SYNTH_CASES  # noqa: E402

synth = importlib.import_module(
    "optimized-implementation-of-word-movers-distance_b200.synth")


def read_sample():
    lines = open(os.path.join(REF, "data/sample.mtx")).read().split("\n")
    V, N, nnz = map(int, lines[0].split())
    edges = [l.split() for l in lines[1:] if l.strip()][:nnz]
    rows = [int(e[0]) - 1 for e in edges]
    cols = [int(e[1]) - 1 for e in edges]
    w = [float(e[2]) for e in edges]
    vecs = np.loadtxt(os.path.join(REF, "data/v2.txt")).reshape(V, -1)
    r = np.loadtxt(os.path.join(REF, "data/r2.txt")).reshape(-1)
    return V, N, rows, cols, w, vecs, r


def main_py():
    sys.path.insert(0, REF)
    import main  # the reference's Python solver (main.py:37)
    return main


def main():
    if not oracle.reference_available("fused"):
        raise SystemExit("oracle/_ref is not built (make -C oracle)")
    out = {"sample_d3": {}, "synthetic": {}}

    V, N, rows, cols, w, vecs, r = read_sample()
    row_ptr, ci, cv = oracle.counting_sort(V, rows, cols, w)
    col_ptr, ri, rv = oracle.counting_sort(N, cols, rows, w)
    from scipy import sparse
    c = sparse.csr_matrix((w, (rows, cols)), shape=(V, N))
    mp = main_py()
    s = {"V": V, "N": N, "edges": [rows, cols, w], "vecs": vecs.tolist(),
         "r": r.tolist(), "max_iter": 15, "outputs": {}}
    for lam in (1.0, 10.0):
        s["outputs"][f"fused_lam{lam:g}"] = O.reference_sinkhorn(
            r, vecs, row_ptr, ci, cv, N, lam, 15, "fused", 1).tolist()
        s["outputs"][f"nonfused_lam{lam:g}"] = O.reference_sinkhorn(
            r, vecs, row_ptr, ci, cv, N, lam, 15, "nonfused", 1).tolist()
        s["outputs"][f"mainpy_lam{lam:g}"] = np.asarray(
            mp.sinkhorn_wmd(r, c, vecs, -lam, 15)).ravel().tolist()
    # The nonfused binary as shipped (lamda = -1 with exp(-M*lamda)).
    s["outputs"]["nonfused_shipped_sign"] = O.reference_sinkhorn(
        r, vecs, row_ptr, ci, cv, N, -1.0, 15, "nonfused", 1).tolist()
    out["sample_d3"] = s

    for name, prm in SYNTH_CASES.items():
        V, d, N, vr, lo, hi, nc, seed, lam, it, empty = prm
        p = synth.case(V, d, N, vr, lo, hi, nc, seed, lam, it, empty)
        csr_ptr, csr_ci, csr_v = oracle.csr_from_csc(
            V, N, p.col_ptr, p.row_inds, p.vals)
        vecs64 = p.vecs.astype(np.float64)
        ref = O.reference_sinkhorn(p.r, vecs64, csr_ptr, csr_ci, csr_v, N, lam,
                                   it, "fused", 1)
        entry = {"params": list(prm), "digest": synth.digest(p),
                 "v_r": p.v_r, "nnz": p.nnz, "fused": ref.tolist()}
        if V * N <= 2_000_000 and p.nnz and np.all(np.diff(p.col_ptr) > 0):
            cs = sparse.csc_matrix((p.vals, p.row_inds, p.col_ptr),
                                   shape=(V, N))
            entry["mainpy"] = np.asarray(
                mp.sinkhorn_wmd(p.r, cs.tocsr(), vecs64, -lam, it)).ravel().tolist()
        out["synthetic"][name] = entry
        print(name, "v_r", p.v_r, "nnz", p.nnz, flush=True)

    path = os.path.join(HERE, "golden.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main()
