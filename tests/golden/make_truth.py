"""Extended-precision truth for the ill-conditioned elements of the fixtures.

Run here, after make_golden.py (needs oracle/_ref, libgrpp compiled from its sources):

    make -C oracle oracle ref
    python tests/golden/make_truth.py [--only config1 config1_moderate config2 h2o cs kcs tho uo2 config3]

On the synthetic workloads (exponents up to 5e3 on f..h shells, potential centres
up to tens of bohr away) libgrpp keeps few or no significant digits on some blocks:
its own result moves by up to the size of the values when its inputs move by a few
units in the last place. No double-precision evaluation of its formulas can be
checked against it element by element there. This script computes, for those
blocks, the value libgrpp's formulas converge to, with oracle/truth_quad.c
(binary128 arithmetic, converged radial integrals, no screening or skip
thresholds), and records how far libgrpp itself is from it.

Per fixture, written to tests/golden/truth_<name>.npz:
  tasks              fixture task indices evaluated: every task with an element
                     whose spread exceeds 1/8 of the strict tolerance
                     max(1e-10, 1e-9 |ref|), the spread being libgrpp's change under
                     last-bit input changes (env) or the oracle's under its rounding
                     model (last-bit changes of exp, log, pow and Bessel values,
                     tests/util.py rounding_runs); tasks already on disk are kept
  truth_<comp>       binary128 blocks of those tasks, rounded to double
  refdev_<comp>      max of |x - truth| over libgrpp's run, its thirty perturbed
                     re-runs (tests/util.py REFDEV_MODES) and the oracle's
                     rounding-model runs: how far implementations of libgrpp's
                     algorithm in double precision land from the exact value
  truthdev_<comp>    max over two perturbed inputs (modes 3, 4) of
                     |truth_p - truth|: the exact value's own sensitivity to the
                     same input changes (small: the loss of digits is in the
                     formulas' double-precision evaluation, not in the integral)
  level, resid       deepest radial grid level and final relative change of the
                     radial integrals per task
config3 (density-contracted gradient, all tasks): truth_grad [4, n_atoms, 3] from
the binary128 blocks of the differentiated shell pairs (L+1 with 2a N_L/N_{L+1},
L-1 with N_L/N_{L-1}, libgrpp/diff_gaussian.c:35-63) contracted with D under
libgrpp's atom and sign rule (libgrpp/grpp_integrals_gradient.c:280-393), and
refdev_grad, the oracle's own distance from it over the same runs and its rounding-model runs (the
config3 reference values are the oracle's: the compiled libgrpp gradient reads
outside its L-1 block and can return NaN).
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from libgrpp_b200.gradient import derivative_batch, gradient_terms  # noqa: E402
from libgrpp_b200.system import cartesian_list, ncart  # noqa: E402
from tests.util import (COMPS, REFDEV_MODES, fixture_subset, load_fixture, load_oracle, load_ref, perturbed,  # noqa: E402
                        rounding_runs, strict_tol, system_from_fixture, truth_full_batch)

U = 2.0 ** -53


def flagged_tasks(batch, z, rm_spread):
    """Tasks with an element on which libgrpp keeps few digits: its input-perturbation spread
    env, or the spread of the oracle's rounding-model runs, exceeds 1/8 of the strict tolerance."""
    off = batch.block_offsets()
    flag = set()
    for m, c in enumerate(COMPS):
        tol = strict_tol(z["ref_" + c]) / 8
        bad = np.where((z["env_" + c] > tol) | (rm_spread[m] > tol))[0]
        flag |= set(int(t) for t in np.searchsorted(off, bad, side="right") - 1)
    return sorted(flag)


def make_blocks(name, ref_lib, orc, nthreads, keep_tasks=False):
    """Truth of the flagged tasks of a fixture (reusing the truth of tasks already on disk) and
    libgrpp's distances from it. keep_tasks: take the task selection on disk as it is."""
    batch, z = load_fixture(name)
    out = os.path.join(HERE, f"truth_{name}.npz")
    old = np.load(out) if os.path.exists(out) else None
    have = {int(t): k for k, t in enumerate(old["tasks"])} if old is not None else {}
    if keep_tasks and old is not None:
        idx = sorted(have)
    else:
        obase = orc.driver_full_batch(batch, nthreads=nthreads)
        rm = rounding_runs(orc, batch, nthreads)
        rm_spread = [np.max([np.abs(r[m] - obase[m]) for r in rm], axis=0) for m in range(4)]
        idx = sorted(set(flagged_tasks(batch, z, rm_spread)) | set(have))
    if not idx:
        print(f"{name}: no task with an ill-conditioned element")
        if os.path.exists(out):
            os.remove(out)
        return
    sub, _, _ = fixture_subset(batch, z, idx)
    soff = sub.block_offsets()
    new = [t for t in idx if t not in have]
    truth = [np.zeros(int(soff[-1])) for _ in range(4)]
    truthdev = [np.zeros(int(soff[-1])) for _ in range(4)]
    level = np.zeros(len(idx), np.int32)
    resid = np.zeros(len(idx))
    if old is not None:
        oo = fixture_subset(batch, z, [int(x) for x in old["tasks"]])[0].block_offsets()
        for t in [t for t in idx if t in have]:
            k = idx.index(t)
            o = have[t]
            for m, c in enumerate(COMPS):
                truth[m][soff[k]:soff[k + 1]] = old["truth_" + c][oo[o]:oo[o + 1]]
                truthdev[m][soff[k]:soff[k + 1]] = old["truthdev_" + c][oo[o]:oo[o + 1]]
            level[k], resid[k] = old["level"][o], old["resid"][o]
    if new:
        nsub, _, _ = fixture_subset(batch, z, new)
        noff = nsub.block_offsets()
        t0 = time.time()
        tn, ln, rn = truth_full_batch(nsub, nthreads=nthreads)
        tds = [np.zeros_like(x) for x in tn]
        for mode in (3, 4):
            tp, _, _ = truth_full_batch(perturbed(nsub, mode), nthreads=nthreads)
            for m in range(4):
                tds[m] = np.maximum(tds[m], np.abs(tp[m] - tn[m]))
        print(f"{name}: truth of {len(new)} new tasks in {time.time() - t0:.0f} s")
        for j, t in enumerate(new):
            k = idx.index(t)
            for m in range(4):
                truth[m][soff[k]:soff[k + 1]] = tn[m][noff[j]:noff[j + 1]]
                truthdev[m][soff[k]:soff[k + 1]] = tds[m][noff[j]:noff[j + 1]]
            level[k], resid[k] = ln[j], rn[j]
    base = ref_lib.driver_full_batch(sub, nthreads=nthreads)
    refdev = [np.abs(base[m] - truth[m]) for m in range(4)]
    for mode in REFDEV_MODES:
        p = ref_lib.driver_full_batch(perturbed(sub, mode), nthreads=nthreads)
        for m in range(4):
            refdev[m] = np.maximum(refdev[m], np.abs(p[m] - truth[m]))
    for r in rounding_runs(orc, sub, nthreads):
        for m in range(4):
            refdev[m] = np.maximum(refdev[m], np.abs(r[m] - truth[m]))
    data = dict(tasks=np.array(idx, dtype=np.int32), level=level, resid=resid)
    print(f"{name}: {len(idx)} tasks with an ill-conditioned element, deepest level {level.max()}")
    for m, c in enumerate(COMPS):
        data["truth_" + c] = truth[m]
        data["refdev_" + c] = refdev[m]
        data["truthdev_" + c] = truthdev[m]
        e = np.abs(base[m] - truth[m])
        print(f"  {c}: max |ref - truth| {e.max():.2e} ({int(np.sum(e > strict_tol(truth[m])))} elements beyond "
              f"1e-10/1e-9), max refdev {refdev[m].max():.2e}, max truthdev {truthdev[m].max():.2e}")
    np.savez_compressed(out, **data)
    print(f"  -> {os.path.relpath(out, ROOT)} ({os.path.getsize(out) / 1e3:.0f} kB)")


def add_rounding(name, orc, nthreads):
    """Widen refdev of the truth on disk by the oracle's rounding-model runs on the same tasks
    (the truth and the earlier distances are kept)."""
    batch, z = load_fixture(name)
    out = os.path.join(HERE, f"truth_{name}.npz")
    old = np.load(out)
    data = {k: old[k] for k in old.files}
    if name == "config3":
        S = system_from_fixture(z)
        for r in rounding_runs(orc, batch, nthreads, grad=(S, z["D"])):
            data["refdev_grad"] = np.maximum(data["refdev_grad"], np.abs(r - data["truth_grad"]))
        print(f"config3: max refdev {data['refdev_grad'].max():.2e}")
    else:
        sub, _, _ = fixture_subset(batch, z, [int(t) for t in old["tasks"]])
        for r in rounding_runs(orc, sub, nthreads):
            for m, c in enumerate(COMPS):
                data["refdev_" + c] = np.maximum(data["refdev_" + c], np.abs(r[m] - data["truth_" + c]))
        print(f"{name}: " + ", ".join(f"{c} max refdev {data['refdev_' + c].max():.2e}" for c in COMPS))
    np.savez_compressed(out, **data)


# ---------------------------------------------------------------- gradient

def truth_gradient(system, batch, D, nthreads):
    """d tr(D V^m)/dR [4, n_atoms, 3] from binary128 blocks of the differentiated shell pairs."""
    dbatch, sub = derivative_batch(batch, system.cart_order)
    blocks, level, resid = truth_full_batch(dbatch, nthreads=nthreads)
    off = dbatch.block_offsets()
    bo = system.basis_offsets()
    g = np.zeros((4, len(system.atoms), 3))
    cl = {L: [tuple(c) for c in cartesian_list(L, system.cart_order)] for L in range(12)}
    for t in range(len(batch.task_a)):
        a, b, c = int(batch.task_a[t]), int(batch.task_b[t]), int(batch.task_c[t])
        la, lb = int(batch.shell_L[a]), int(batch.shell_L[b])
        A, B = batch.shell_origin[3 * a:3 * a + 3], batch.shell_origin[3 * b:3 * b + 3]
        C = batch.centre_origin[3 * c:3 * c + 3]
        Dab = D[bo[a]:bo[a] + ncart(la), bo[b]:bo[b] + ncart(lb)]
        side = np.zeros((2, 3, 4))  # d/dA (bra), d/dB (ket) of sum_ij D_ij V_ij
        for s, (td, tu, l_d, l_o) in enumerate(((sub[t][0], sub[t][1], la, lb), (sub[t][2], sub[t][3], lb, la))):
            for m in range(4):
                Vu = blocks[m][off[tu]:off[tu + 1]].reshape((ncart(la + 1), ncart(lb)) if s == 0 else (ncart(la), ncart(lb + 1)))
                Vd = None
                if td >= 0:
                    Vd = blocks[m][off[td]:off[td + 1]].reshape((ncart(la - 1), ncart(lb)) if s == 0 else (ncart(la), ncart(lb - 1)))
                for k in range(3):
                    acc = 0.0
                    for i, ci in enumerate(cl[l_d]):
                        up_c = list(ci)
                        up_c[k] += 1
                        iu = cl[l_d + 1].index(tuple(up_c))
                        row_u = Vu[iu, :] if s == 0 else Vu[:, iu]
                        val = row_u.copy()
                        if ci[k] > 0 and Vd is not None:
                            dn_c = list(ci)
                            dn_c[k] -= 1
                            idn = cl[l_d - 1].index(tuple(dn_c))
                            val = val - ci[k] * (Vd[idn, :] if s == 0 else Vd[:, idn])
                        acc += float(np.dot(Dab[i, :], val)) if s == 0 else float(np.dot(Dab[:, i], val))
                    side[s, k, m] = acc
        atoms = [int(system.shell_atom[a]), int(system.shell_atom[b]), int(system.centre_atom[c])]
        for q, at in enumerate(atoms):
            if at in atoms[:q]:
                continue
            for diff_bra, f in gradient_terms(A, B, C, system.atoms[at]):
                g[:, at, :] += f * side[0 if diff_bra else 1].T
    return g, level, resid


def make_gradient(nthreads, refdev_only=False):
    batch, z = load_fixture("config3")
    S = system_from_fixture(z)
    D = z["D"]
    out = os.path.join(HERE, "truth_config3.npz")
    if refdev_only:
        old = np.load(out)
        g, level, resid = old["truth_grad"], old["level"], old["resid"]
    else:
        t = time.time()
        g, level, resid = truth_gradient(S, batch, D, nthreads)
        print(f"config3: truth gradient of {len(batch.task_a)} tasks in {time.time() - t:.0f} s, deepest level "
              f"{level.max()}, worst residual {resid.max():.1e}")
    import copy
    orc = load_oracle()
    refdev = np.abs(orc.driver_grad_contract(S, batch, D, nthreads=nthreads) - g)
    for r in rounding_runs(orc, batch, nthreads, grad=(S, D)):
        refdev = np.maximum(refdev, np.abs(r - g))
    for mode in REFDEV_MODES:
        sp = copy.copy(S)
        if mode == 2:
            sp.atoms = np.asarray(S.atoms) * (1 + 4 * U)
        refdev = np.maximum(refdev, np.abs(orc.driver_grad_contract(sp, perturbed(batch, mode), D, nthreads=nthreads) - g))
    e = np.abs(z["ref_grad"] - g)
    print(f"  max |oracle - truth| {e.max():.2e} ({int(np.sum(e > strict_tol(g)))} elements beyond 1e-10/1e-9), "
          f"max refdev {refdev.max():.2e}, max |g| {np.abs(g).max():.2e}")
    np.savez_compressed(out, truth_grad=g, refdev_grad=refdev, level=level, resid=resid)
    print(f"  -> {os.path.relpath(out, ROOT)} ({os.path.getsize(out) / 1e3:.0f} kB)")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*")
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--refdev-only", action="store_true", help="config3: keep the truth on disk, recompute the distances")
    ap.add_argument("--keep-tasks", action="store_true", help="keep each fixture's task selection on disk")
    ap.add_argument("--add-rounding", action="store_true",
                    help="keep the truth files on disk and widen their refdev by the oracle's rounding-model runs")
    args = ap.parse_args()
    ref = load_ref()
    if ref is None:
        raise SystemExit("oracle/_ref/libgrpp_ref.so is not built (make -C oracle ref)")
    orc = load_oracle()
    if args.add_rounding:
        for name in args.only or ("config1", "config1_moderate", "config2", "config3"):
            add_rounding(name, orc, args.threads or os.cpu_count())
        return
    for name in ("config1", "config1_moderate", "config2", "h2o", "cs", "kcs", "tho", "uo2"):
        if not args.only or name in args.only:
            make_blocks(name, ref, orc, args.threads or os.cpu_count(), args.keep_tasks)
    if not args.only or "config3" in args.only:
        make_gradient(args.threads or os.cpu_count(), args.refdev_only)


if __name__ == "__main__":
    main()
