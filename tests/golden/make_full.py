"""Full-matrix fixtures of libgrpp's heavy-element tests (tests/golden/full_<name>.npz).

Run here, where the reference tree exists:

    python tests/golden/make_full.py [--ref-root <libgrpp source tree>]   (default: $LIBGRPP_REFERENCE)

For test/ThO, test/UO2 and test/KCs the molecule, basis and GRPP inputs are read with
libgrpp_b200.formats (the C driver's shell and centre order, test_libgrpp_c/main.c:196-254)
and stored flat (b_* arrays, no task list: every ordered pair of the n_shells basis
shells x every centre is a task; the outercore shells follow the basis shells), together with libgrpp's shipped matrices arep.txt, so_x.txt, so_y.txt, so_z.txt as
dense lower triangles. These are the matrices libgrpp's own ctest compares its output with
(test/compare_matrices.c:129-148, CMakeLists.txt:53-59).

libgrpp compiled here (oracle/_ref, the C driver's full-GRPP calls) reproduces the shipped
ThO and UO2 matrices to 1e-13. The shipped KCs matrices come from libgrpp's Fortran driver
(test/KCs/run_test.sh), which sums type 1, type 2 per L and outercore terms from separate
calls, each with its own radial-grid convergence; five of its arep elements sit 1.7e-10 to
2.1e-10 from the C path. For every element where the C path and the shipped matrix differ
beyond the tolerance of record, the fixture holds the binary128 value (oracle/truth_quad.c,
summed over the element's tasks) as truth_<comp>[truth_idx], and refdev_<comp> = the larger
of the two libgrpp paths' distances from it.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from libgrpp_b200.formats import read_lower_triangle, read_system  # noqa: E402
from tests.util import (assemble_lower, full_system, load_ref, strict_tol,  # noqa: E402
                        truth_full_batch)

COMPS = ("arep", "so_x", "so_y", "so_z")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=os.environ.get("LIBGRPP_REFERENCE", "/root/reference"))
    args = ap.parse_args()
    for name in ("ThO", "UO2", "KCs"):
        d = os.path.join(args.ref_root, "test", name)
        S = read_system(d)
        b = S.batch(np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32))
        data = {"b_" + k: v for k, v in b.__dict__.items() if not k.startswith("_") and not k.startswith("task_")}
        n = S.n_basis()
        tri = np.tril_indices(n)
        for c in COMPS:
            data["shipped_" + c] = read_lower_triangle(os.path.join(d, c + ".txt"))[tri]
        data["cart_order"] = S.cart_order
        data["n_basis"] = n
        data["n_shells"] = len(S.shells)  # basis shells come first; outercore shells follow
        out = os.path.join(HERE, f"full_{name.lower()}.npz")
        np.savez_compressed(out, **data)
        add_truth(out, n)
        print(f"{name}: {len(S.shells)} shells, {n} basis functions, {len(S.centres)} centres -> "
              f"{os.path.relpath(out, ROOT)} ({os.path.getsize(out) / 1e6:.1f} MB)")


def add_truth(path, n):
    """Truth for the elements where libgrpp's C path and the shipped matrix disagree."""
    name = os.path.basename(path)[5:-4]
    batch, z = full_system(name)
    ns = int(z["n_shells"])
    ref = assemble_lower(batch, load_ref().driver_full_batch(batch, nthreads=os.cpu_count()), ns)
    bad = np.zeros(len(ref[0]), dtype=bool)
    for c, r in zip(COMPS, ref):
        d = np.abs(r - z["shipped_" + c])
        bad |= d > strict_tol(z["shipped_" + c])
        print(f"  {name} {c}: libgrpp C path vs shipped max abs {d.max():.2e}, beyond tolerance {int(np.sum(d > strict_tol(z['shipped_' + c])))}")
    data = dict(z)
    idx = np.flatnonzero(bad)
    data["truth_idx"] = idx.astype(np.int64)
    if len(idx):
        from libgrpp_b200.system import ncart
        rows, cols = np.tril_indices(n)
        off = np.concatenate([[0], np.cumsum([ncart(int(x)) for x in batch.shell_L[:ns]])])
        sh = lambda i: int(np.searchsorted(off, i, side="right") - 1)  # noqa: E731
        pairs = sorted({(sh(rows[k]), sh(cols[k])) for k in idx})
        nc = len(batch.centre_grpp)
        ta = np.array([a for a, b in pairs for _ in range(nc)], dtype=np.int32)
        tb = np.array([b for a, b in pairs for _ in range(nc)], dtype=np.int32)
        tc = np.array([c for _ in pairs for c in range(nc)], dtype=np.int32)
        sub = batch.with_tasks(ta, tb, tc)
        truth, lev, res = truth_full_batch(sub, nthreads=os.cpu_count())
        print(f"  {name}: truth for {len(idx)} elements from {len(ta)} tasks, deepest level {lev.max()}, "
              f"worst residual {res.max():.1e}")
        tl = assemble_lower(sub, truth, ns)
        for c, r, t in zip(COMPS, ref, tl):
            data["truth_" + c] = t[idx]
            data["refdev_" + c] = np.maximum(np.abs(z["shipped_" + c][idx] - t[idx]), np.abs(r[idx] - t[idx]))
            print(f"  {name} {c}: shipped - truth max {np.abs(z['shipped_' + c][idx] - t[idx]).max():.2e}, "
                  f"C path - truth max {np.abs(r[idx] - t[idx]).max():.2e}")
    np.savez_compressed(path, **data)


if __name__ == "__main__":
    main()
