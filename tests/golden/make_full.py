"""Full-matrix fixtures of libgrpp's heavy-element tests (tests/golden/full_<name>.npz).

Run here, where the reference tree exists:

    python tests/golden/make_full.py [--ref-root <libgrpp source tree>]   (default: $LIBGRPP_REFERENCE)
    python tests/golden/make_full.py --truth-only [--only ThO UO2 KCs]   (redo the truth selection only)

For test/ThO, test/UO2 and test/KCs the molecule, basis and GRPP inputs are read with
libgrpp_b200.formats (the C driver's shell and centre order, test_libgrpp_c/main.c:196-254)
and stored flat (b_* arrays, no task list: every ordered pair of the n_shells basis
shells x every centre is a task; the outercore shells follow the basis shells), together with libgrpp's shipped matrices arep.txt, so_x.txt, so_y.txt, so_z.txt as
dense lower triangles. These are the matrices libgrpp's own ctest compares its output with
(test/compare_matrices.c:129-148, CMakeLists.txt:53-59).

libgrpp compiled here (oracle/_ref, the C driver's full-GRPP calls) reproduces the shipped
ThO and UO2 matrices to 1e-13. The shipped KCs matrices come from libgrpp's Fortran driver
(test/KCs/run_test.sh), which sums type 1, type 2 per L and outercore terms from separate
calls; one of its arep elements sits 2.1e-10 from the C path. On some elements libgrpp
keeps few digits: i-shell pairs on Th with the O potential 3.7 bohr away carry errors up
to 8e-7 against the exact value in libgrpp's own result, from cancellation in the binomial
re-centring sum. Those elements are found by running libgrpp on the inputs and on copies
moved by a few units in the last place, and the oracle under its rounding model (last-bit
changes of exp, log, pow and Bessel values); for each element where a run lands more than
an eighth of the tolerance from the shipped value, the fixture holds the binary128 value
(oracle/truth_quad.c, summed over the element's tasks) as truth_<comp>[truth_idx], and
refdev_<comp>, the largest distance from it of the shipped value and of the runs.
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
from tests.util import (assemble_lower, full_system, load_oracle, load_ref, perturbed, rounding_runs,  # noqa: E402
                        strict_tol, truth_full_batch)

COMPS = ("arep", "so_x", "so_y", "so_z")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=os.environ.get("LIBGRPP_REFERENCE", "/root/reference"))
    ap.add_argument("--truth-only", action="store_true", help="keep the shipped matrices on disk, redo the truth")
    ap.add_argument("--only", nargs="*", help="subset of ThO UO2 KCs")
    args = ap.parse_args()
    if args.truth_only:
        for name in args.only or ("ThO", "UO2", "KCs"):
            out = os.path.join(HERE, f"full_{name.lower()}.npz")
            z = np.load(out)
            data = {k: z[k] for k in z.files if not k.startswith(("truth_", "refdev_"))}
            np.savez_compressed(out, **data)
            add_truth(out, int(z["n_basis"]))
        return
    for name in args.only or ("ThO", "UO2", "KCs"):
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


FULL_INPUT_MODES = (1, 2, 3, 4)  # input perturbations of libgrpp's runs (tests.util.perturbed)
# the runs cover the shell pairs with la + lb >= FULL_MIN_LSUM, where the binomial re-centring
# about a potential centre a few bohr away amplifies last-bit differences (its factors grow as
# |CA|^la |CB|^lb); elements of the other pairs are judged by the strict tolerance alone
FULL_MIN_LSUM = 7


def add_truth(path, n):
    """Truth for the elements on which libgrpp keeps few digits: those where a run of libgrpp's
    algorithm lands more than an eighth of the tolerance from the shipped value. The runs are
    libgrpp's C path on the inputs and on copies moved by a few units in the last place
    (tests.util.perturbed, FULL_INPUT_MODES), and the oracle under its rounding model (last-bit
    changes of exp, log, pow, Bessel values and of the radial stop tests: another
    implementation's arithmetic, tests.util.rounding_runs), over the shell pairs with
    la + lb >= FULL_MIN_LSUM; a run's element is the shipped value with the pairs' part replaced."""
    name = os.path.basename(path)[5:-4]
    batch, z = full_system(name)
    ns = int(z["n_shells"])
    lib = load_ref()
    nt = os.cpu_count()
    L = batch.shell_L
    keep = np.flatnonzero(L[batch.task_a] + L[batch.task_b] >= FULL_MIN_LSUM)
    hb = batch.with_tasks(batch.task_a[keep], batch.task_b[keep], batch.task_c[keep])
    base = assemble_lower(hb, lib.driver_full_batch(hb, nthreads=nt), ns)
    runs = [base]
    for mode in FULL_INPUT_MODES:
        runs.append(assemble_lower(hb, lib.driver_full_batch(perturbed(hb, mode), nthreads=nt), ns))
    for r in rounding_runs(load_oracle(), hb, nt):
        runs.append(assemble_lower(hb, r, ns))
    # the high-l pairs' part of each element: the runs differ from libgrpp's base only there
    rest = [z["shipped_" + c] - base[m] for m, c in enumerate(COMPS)]
    runs = [[r[m] + rest[m] for m in range(4)] for r in runs]
    # and libgrpp's C path over every pair (the shipped KCs matrices come from its Fortran driver)
    runs.append(assemble_lower(batch, lib.driver_full_batch(batch, nthreads=nt), ns))
    sens = np.zeros(len(runs[0][0]), dtype=bool)
    for m, c in enumerate(COMPS):
        tol = strict_tol(z["shipped_" + c])
        d = np.abs(runs[-1][m] - z["shipped_" + c])
        print(f"  {name} {c}: libgrpp C path vs shipped max abs {d.max():.2e}, beyond tolerance {int(np.sum(d > tol))}")
        for r in runs:
            sens |= np.abs(r[m] - z["shipped_" + c]) > tol / 8
    data = dict(z)
    idx = np.flatnonzero(sens)
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
        truth, lev, res = truth_full_batch(sub, nthreads=nt)
        print(f"  {name}: truth for {len(idx)} elements of {len(pairs)} shell pairs ({len(ta)} tasks), deepest "
              f"level {lev.max()}, worst residual {res.max():.1e}")
        tl = assemble_lower(sub, truth, ns)
        for m, c in enumerate(COMPS):
            t = tl[m][idx]
            data["truth_" + c] = t
            data["refdev_" + c] = np.max([np.abs(z["shipped_" + c][idx] - t)] + [np.abs(r[m][idx] - t) for r in runs], axis=0)
            print(f"  {name} {c}: shipped - truth max {np.abs(z['shipped_' + c][idx] - t).max():.2e}, "
                  f"max refdev {data['refdev_' + c].max():.2e}")
    np.savez_compressed(path, **data)

if __name__ == "__main__":
    main()
