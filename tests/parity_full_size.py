"""Parity of the product's matvec with the reference's at full size (the
245,760-unknown lossy sphere: radius 5 lambda, icosphere sub 6, eps_r
2.5-0.1j, leaf 0.25 lambda), on a B200 with the reference built in
oracle/_ref. Not collected by pytest (about two minutes, most of it the
reference's own setup on the host cores).

    python tests/parity_full_size.py [--sub 6] [--radius-lambda 5]

Reports:
  * the relative 2-norm difference of A x (x uniform on the unit disk,
    mt19937_64 seed 0) between product and reference;
  * the near-field entries that differ beyond 1e-11 of the largest entry,
    and whether every one of them is a K-type entry (z12 = -z21) of two
    RWGs sharing a triangle. These are the same-triangle terms whose
    reference evaluation takes the 1/|D| branch on a rounding-noise height
    (Code/Operator.h:637-652); the product evaluates them at height 0;
  * the matvec difference once those entries of the reference are replaced
    by the product's. That number is the parity of everything else.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--sub", type=int, default=6)
    ap.add_argument("--radius-lambda", type=float, default=5.0)
    ap.add_argument("--eps", type=complex, default=complex(2.5, -0.1))
    ap.add_argument("--leaf", type=float, default=0.25)
    args = ap.parse_args(argv)
    from mlfma_pmchwt_b200 import MLFMM
    from mlfma_pmchwt_b200 import mesh as M
    from oracle import oracle as O

    O.set_threads(os.cpu_count() or 1)
    lam = M.wavelength(3e8)
    m = M.icosphere(args.sub, args.radius_lambda * lam)
    nas = M.write_nas(m, Path("/tmp") / f"parity_full_{os.getpid()}.nas")
    op = MLFMM(m, eps_r=args.eps, leaf_coeff=args.leaf, device=0)
    t0 = time.perf_counter()
    ref = O.RefOperator(nas, eps_r=args.eps, leaf_coeff=args.leaf)
    ref_setup = time.perf_counter() - t0
    N, n = op.N, op.n
    x = M.unit_disk_vector(n, 0)
    w = op.apply_ax(x)
    wr = ref.apply(x)
    out = {"unknowns": n, "reference_setup_s": round(ref_setup, 1), "matvec_rel_raw": rel(w, wr)}

    # near-field entries, aligned by (target, source)
    nr = op.near(values=True)
    mk = nr["target"].astype(np.int64) * N + nr["source"]
    ptr, ids, vals = ref.znear()
    lens = np.diff(ptr[: N + 1]) // 2
    rt = np.repeat(np.arange(N, dtype=np.int64), lens)
    rs = ids[ptr[0]:ptr[N]][0::2].astype(np.int64)
    rz11 = vals[ptr[0]:ptr[N]][0::2]
    rz12 = vals[ptr[0]:ptr[N]][1::2]
    rz22 = vals[ptr[N]:ptr[2 * N]][1::2]
    rk = rt * N + rs
    om, orf = np.argsort(mk), np.argsort(rk)
    assert np.array_equal(mk[om], rk[orf]), "near pair sets differ"
    z11, z12, z22 = nr["z11"][om], nr["z12"][om], nr["z22"][om]
    rz11, rz12, rz22 = rz11[orf], rz12[orf], rz22[orf]
    t, s = rt[orf], rs[orf]
    scale = np.abs(rz11).max()
    tol = 1e-11 * scale
    off11 = np.abs(z11 - rz11) > tol
    off22 = np.abs(z22 - rz22) > tol
    off12 = np.abs(z12 - rz12) > tol
    r = op.rwgs()
    fp, fn = r["face_pos"], r["face_neg"]
    shares = (fp[t] == fp[s]) | (fp[t] == fn[s]) | (fn[t] == fp[s]) | (fn[t] == fn[s])
    out.update(near_pairs=int(len(t)), differing_z11=int(off11.sum()), differing_z22=int(off22.sum()),
               differing_z12=int(off12.sum()), differing_z12_all_share_a_triangle=bool(shares[off12].all()),
               max_z12_difference_over_median_z12=float(np.abs(z12 - rz12)[off12].max() / np.median(np.abs(rz12)))
               if off12.any() else 0.0)
    clean = ~(off11 | off12 | off22)
    out["near_rel_of_other_entries"] = float(
        np.sqrt((np.abs(z11 - rz11)[clean] ** 2 + np.abs(z12 - rz12)[clean] ** 2 + np.abs(z22 - rz22)[clean] ** 2).sum()
                / (np.abs(rz11[clean]) ** 2 + np.abs(rz12[clean]) ** 2 + np.abs(rz22[clean]) ** 2).sum()))
    # reference matvec with the flagged K entries exchanged for the product's
    d = (z12 - rz12)[off12]
    wf = wr.copy()
    np.add.at(wf, t[off12], d * x[N + s[off12]])
    np.add.at(wf, N + t[off12], -d * x[s[off12]])
    out["matvec_rel_after_exchange"] = rel(w, wf)
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
