"""Shared helpers of the test suite (fixtures, libraries, comparisons)."""
from __future__ import annotations

import os

import numpy as np

from libgrpp_b200.system import BatchArrays

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "libgrpp_oracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libgrpp_ref.so")
TRUTH_SO = os.path.join(ROOT, "oracle", "_build", "libgrpp_truth.so")
COMPS = ("arep", "so_x", "so_y", "so_z")


def ensure_oracle():
    if not os.path.exists(ORACLE_SO):
        import subprocess
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True, capture_output=True)
    return ORACLE_SO


def truth_full_batch(batch, t0=0, t1=None, nthreads=0):
    """Extended-precision (binary128) full-GRPP blocks of tasks t0..t1-1 (oracle/truth_quad.c):
    the four output arrays, the deepest radial grid level of each task and its radial
    integrals' final change between levels relative to the sum of their absolute terms."""
    import ctypes as ct
    if not os.path.exists(TRUTH_SO):
        import subprocess
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True, capture_output=True)
    lib = ct.CDLL(TRUTH_SO)
    D = ct.POINTER(ct.c_double)
    Ip = ct.POINTER(ct.c_int)
    lib.truth_full_batch.restype = ct.c_int
    lib.truth_full_batch.argtypes = [ct.c_void_p, ct.c_int64, ct.c_int64, ct.c_int, D, D, D, D, Ip, D]
    if t1 is None:
        t1 = len(batch.task_a)
    off = batch.block_offsets()
    n = int(off[t1] - off[t0])
    outs = [np.zeros(max(n, 1)) for _ in range(4)]
    lev = np.zeros(max(t1 - t0, 1), dtype=np.int32)
    res = np.zeros(max(t1 - t0, 1))
    lib.truth_full_batch(ct.byref(batch.struct), t0, t1, nthreads, *[x.ctypes.data_as(D) for x in outs],
                         lev.ctypes.data_as(Ip), res.ctypes.data_as(D))
    return [x[:n] for x in outs], lev[:t1 - t0], res[:t1 - t0]


def load_oracle():
    from libgrpp_b200.capi import LibGRPP
    return LibGRPP(ensure_oracle())


def load_ref():
    from libgrpp_b200.capi import LibGRPP
    if not os.path.exists(REF_SO):
        return None
    return LibGRPP(REF_SO)


def load_product():
    from libgrpp_b200 import engine
    return engine.load()


def load_fixture(name: str):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    arrays = {k[2:]: np.ascontiguousarray(z[k]) for k in z.files if k.startswith("b_")}
    arrays["task_a"] = np.ascontiguousarray(z["task_a"], dtype=np.int32)
    arrays["task_b"] = np.ascontiguousarray(z["task_b"], dtype=np.int32)
    arrays["task_c"] = np.ascontiguousarray(z["task_c"], dtype=np.int32)
    return BatchArrays(**arrays), z


def fixture_subset(batch, z, idx):
    """Tasks idx of a fixture: the sub-batch and, per component, the reference blocks and envelopes."""
    idx = np.asarray(idx)
    off = batch.block_offsets()
    d = {k: v for k, v in batch.__dict__.items() if not k.startswith("_")}
    for k in ("task_a", "task_b", "task_c"):
        d[k] = np.ascontiguousarray(d[k][idx])
    sub = BatchArrays(**d)
    sel = np.concatenate([np.arange(off[t], off[t + 1]) for t in idx])
    ref = {c: z["ref_" + c][sel] for c in COMPS}
    env = {c: z["env_" + c][sel] for c in COMPS}
    return sub, ref, env


def max_abs(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) if len(a) else 0.0


def parity_report(got, want):
    """max abs error, and max relative error over elements with |want| > 1e-6"""
    got, want = np.asarray(got), np.asarray(want)
    ab = float(np.max(np.abs(got - want))) if got.size else 0.0
    big = np.abs(want) > 1e-6
    rel = float(np.max(np.abs(got[big] - want[big]) / np.abs(want[big]))) if big.any() else 0.0
    return ab, rel


def system_from_fixture(z):
    """Rebuild the System (basis shells, GRPPs, centres) stored flat in a fixture."""
    from libgrpp_b200.system import GRPP, Potential, Shell, System

    g = lambda k: z["b_" + k]  # noqa: E731
    nbasis = int(max(z["task_a"].max(), z["task_b"].max())) + 1

    def shell(i):
        o, n = int(g("shell_prim_off")[i]), int(g("shell_nprim")[i])
        return Shell(g("shell_origin")[3 * i:3 * i + 3], int(g("shell_L")[i]), g("prim_coef")[o:o + n], g("prim_alpha")[o:o + n])

    def pot(p):
        o, n = int(g("pot_prim_off")[p]), int(g("pot_nprim")[p])
        return Potential(int(g("pot_L")[p]), int(g("pot_J")[p]), g("pot_powers")[o:o + n], g("pot_coef")[o:o + n],
                         g("pot_alpha")[o:o + n])

    grpps = []
    for k in range(len(g("grpp_UL"))):
        G = GRPP()
        G.UL = pot(int(g("grpp_UL")[k])) if g("grpp_UL")[k] >= 0 else None
        lst = g("grpp_pot_list")
        G.arep = [pot(int(lst[g("grpp_arep_off")[k] + i])) for i in range(int(g("grpp_n_arep")[k]))]
        G.so = [pot(int(lst[g("grpp_so_off")[k] + i])) for i in range(int(g("grpp_n_so")[k]))]
        G.oc = [(pot(int(g("grpp_oc_pot")[g("grpp_oc_off")[k] + i])), shell(int(g("grpp_oc_shell")[g("grpp_oc_off")[k] + i])))
                for i in range(int(g("grpp_n_oc")[k]))]
        grpps.append(G)
    co = g("centre_origin").reshape(-1, 3)
    centres = [(co[i].copy(), int(g("centre_grpp")[i])) for i in range(len(g("centre_grpp")))]
    shells = [shell(i) for i in range(nbasis)]
    atoms = z["atoms"] if "atoms" in z.files else None
    sa = z["shell_atom"] if "shell_atom" in z.files else None
    ca = z["centre_atom"] if "centre_atom" in z.files else None
    return System(shells, grpps, centres, int(z["cart_order"]), sa, ca, atoms)


U = 2.0 ** -53  # unit roundoff


def perturbed(batch: BatchArrays, mode: int) -> BatchArrays:
    """The same workload with inputs moved by a few units in the last place:
    mode 1 scales every exponent by (1 + 4u); mode 2 scales contraction and
    potential coefficients by (1 - 4u), (1 + 4u) and every coordinate by (1 + 4u)
    (coincident centres stay coincident); modes 3 and above move every exponent and
    coefficient independently by a seeded random whole number of units in [-4, 4]
    (a uniform scaling can leave a cancelling sum's rounding pattern unchanged,
    independent changes do not)."""
    d = {k: v for k, v in batch.__dict__.items() if not k.startswith("_")}
    d = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    if mode == 1:
        d["prim_alpha"] = d["prim_alpha"] * (1 + 4 * U)
        d["pot_alpha"] = d["pot_alpha"] * (1 + 4 * U)
    elif mode >= 3:
        rng = np.random.default_rng(mode)
        for k in ("prim_alpha", "pot_alpha", "prim_coef", "pot_coef"):
            d[k] = d[k] * (1 + rng.integers(-4, 5, d[k].shape) * U)
    else:
        d["prim_coef"] = d["prim_coef"] * (1 - 4 * U)
        d["pot_coef"] = d["pot_coef"] * (1 + 4 * U)
        d["shell_origin"] = d["shell_origin"] * (1 + 4 * U)
        d["centre_origin"] = d["centre_origin"] * (1 + 4 * U)
    return BatchArrays(**d)


ENV_MODES = (1, 2) + tuple(range(3, 11))  # two uniform and eight independent random perturbations
# libgrpp's distance from the exact value (refdev) is the largest over its run on the inputs and thirty
# perturbed re-runs: the spread has heavy tails (a changed stop level of one radial integral moves a
# whole block), and with ten re-runs the largest distance was still growing by up to 3x
REFDEV_MODES = (1, 2) + tuple(range(3, 31))


# seeds of the oracle's rounding model (orc_set_rounding_model in oracle/orc_integrals.c): runs of
# libgrpp's algorithm whose transcendental results and Bessel values differ from libgrpp's in the
# last bit, as any other implementation's (a GPU's exp, regenerated tables) do
ROUNDING_SEEDS = tuple(range(1, 13))


def rounding_runs(oracle, batch: BatchArrays, nthreads=0, seeds=ROUNDING_SEEDS, grad=None):
    """The oracle's full-GRPP blocks (or, with grad=(system, D), its density-contracted gradient)
    under each seed of the rounding model; the model is switched off afterwards."""
    import ctypes as ct
    f = oracle.lib.orc_set_rounding_model
    f.argtypes = [ct.c_uint64]
    f.restype = None
    nthreads = nthreads or os.cpu_count()
    out = []
    try:
        for seed in seeds:
            f(seed)
            if grad is None:
                out.append(oracle.driver_full_batch(batch, nthreads=nthreads))
            else:
                out.append(oracle.driver_grad_contract(grad[0], batch, grad[1], nthreads=nthreads))
    finally:
        f(0)
    return out


def envelope(lib, batch: BatchArrays, base=None, nthreads=8, modes=ENV_MODES):
    """Per-element sensitivity of a CPU library's result to last-bit input changes:
    max over the perturbations of |result(perturbed) - result|."""
    if base is None:
        base = lib.driver_full_batch(batch, nthreads=nthreads)
    env = [np.zeros_like(x) for x in base]
    for mode in modes:
        p = lib.driver_full_batch(perturbed(batch, mode), nthreads=nthreads)
        for m in range(4):
            env[m] = np.maximum(env[m], np.abs(p[m] - base[m]))
    return base, env


def parity(got, want, env=None, abs_tol=1e-10, rel_tol=1e-9, env_factor=4.0):
    """Element-wise check of record: |got - want| <= max(abs_tol, rel_tol*|want| for |want| > 1e-6,
    env_factor * envelope). Returns (ok, max_abs, max_rel, n_elements_within_envelope_only)."""
    got, want = np.asarray(got), np.asarray(want)
    err = np.abs(got - want)
    tol = np.full(err.shape, abs_tol)
    big = np.abs(want) > 1e-6
    tol[big] = np.maximum(tol[big], rel_tol * np.abs(want[big]))
    strict_ok = err <= tol
    if env is not None:
        tol = np.maximum(tol, env_factor * np.asarray(env))
    ok = bool(np.all(err <= tol)) and bool(np.all(np.isfinite(got)))
    max_rel = float(np.max(err[big] / np.abs(want[big]))) if big.any() else 0.0
    n_env = int(np.sum(~strict_ok & (err <= tol)))
    return ok, float(err.max()) if err.size else 0.0, max_rel, n_env


def strict_tol(ref, abs_tol=1e-10, rel_tol=1e-9):
    """The tolerance of record per element: max(1e-10, 1e-9 |ref| for |ref| > 1e-6)."""
    ref = np.asarray(ref)
    tol = np.full(ref.shape, abs_tol)
    big = np.abs(ref) > 1e-6
    tol[big] = np.maximum(tol[big], rel_tol * np.abs(ref[big]))
    return tol


def load_truth(name):
    """tests/golden/truth_<name>.npz (tests/golden/make_truth.py), or None."""
    p = os.path.join(GOLDEN, f"truth_{name}.npz")
    return np.load(p) if os.path.exists(p) else None


TRUTH_FACTOR = 2.0  # an element judged against the exact value may be off by twice the reference's own distance


def truth_parity(got, ref, truth=None, tr_sel=None, comp="arep"):
    """Element-wise check of record against libgrpp with the extended-precision truth:
      - every element: |got - ref| <= max(1e-10, 1e-9 |ref| for |ref| > 1e-6) (strict), or
      - for the elements tr_sel of the tasks in the truth fixture, where libgrpp itself keeps
        few digits: |got - truth| <= max(strict tolerance of truth, 2 refdev), refdev being the
        largest distance from the truth of libgrpp's run and its thirty perturbed re-runs.
    Returns (ok, report dict)."""
    got, ref = np.asarray(got), np.asarray(ref)
    err = np.abs(got - ref)
    strict = err <= strict_tol(ref)
    ok = strict & np.isfinite(got)
    rep = {"max_abs": float(err.max()) if err.size else 0.0, "strict_fail": int(np.sum(~strict)), "truth_checked": 0,
           "truth_fail": 0, "worst_truth_ratio": 0.0, "max_ref_truth": 0.0, "max_got_truth": 0.0}
    if truth is not None and tr_sel is not None and len(tr_sel):
        tv = truth["truth_" + comp]
        bound = np.maximum(strict_tol(tv), TRUTH_FACTOR * truth["refdev_" + comp])
        e_t = np.abs(got[tr_sel] - tv)
        t_ok = e_t <= bound
        need = ~strict[tr_sel]
        rep["truth_checked"] = int(np.sum(need))
        rep["truth_fail"] = int(np.sum(need & ~t_ok))
        rep["worst_truth_ratio"] = float(np.max(e_t[need] / bound[need])) if need.any() else 0.0
        rep["max_ref_truth"] = float(np.max(np.abs(ref[tr_sel] - tv)))
        rep["max_got_truth"] = float(np.max(e_t))
        ok[tr_sel] = (strict[tr_sel] | t_ok) & np.isfinite(got[tr_sel])
    return bool(np.all(ok)), rep


def full_system(name):
    """A full-matrix fixture (tests/golden/full_<name>.npz) and its batch of every ordered pair
    of basis shells x every centre, in the C driver's order (test_libgrpp_c/eval_integrals.c)."""
    from libgrpp_b200.system import BatchArrays
    z = np.load(os.path.join(GOLDEN, f"full_{name}.npz"))
    arr = {k[2:]: np.ascontiguousarray(z[k]) for k in z.files if k.startswith("b_")}
    ns, nc = int(z["n_shells"]), len(arr["centre_grpp"])
    a, b, c = np.meshgrid(np.arange(ns), np.arange(ns), np.arange(nc), indexing="ij")
    arr["task_a"], arr["task_b"], arr["task_c"] = [np.ascontiguousarray(x.ravel(), dtype=np.int32) for x in (a, b, c)]
    return BatchArrays(**arr), z


def assemble_lower(batch, outs, n_shells):
    """Sum the task blocks of ``outs`` (one array per component, blocks row-major in task order)
    into the dense matrices over the first n_shells shells, as libgrpp's drivers accumulate them,
    and return each matrix's lower triangle (np.tril_indices order)."""
    from libgrpp_b200.system import ncart
    L = batch.shell_L[:n_shells]
    off = np.zeros(n_shells + 1, dtype=np.int64)
    off[1:] = np.cumsum([ncart(int(x)) for x in L])
    n = int(off[-1])
    sz = np.array([ncart(int(x)) for x in L], dtype=np.int64)
    ta, tb = batch.task_a.astype(np.int64), batch.task_b.astype(np.int64)
    rows, cols = [], []
    for t in range(len(ta)):  # element (i, j) of task t's block sits at row off[a] + i, column off[b] + j
        na, nb = sz[ta[t]], sz[tb[t]]
        rows.append(np.repeat(off[ta[t]] + np.arange(na), nb))
        cols.append(np.tile(off[tb[t]] + np.arange(nb), na))
    flat = np.concatenate(rows) * n + np.concatenate(cols)
    tri = np.tril_indices(n)
    return [np.bincount(flat, weights=np.asarray(o, dtype=np.float64), minlength=n * n).reshape(n, n)[tri] for o in outs]


def truth_selection(batch, truth):
    """Element indices (into a fixture's output arrays) of the tasks a truth fixture covers, in
    the truth arrays' order."""
    if truth is None:
        return None
    off = batch.block_offsets()
    return np.concatenate([np.arange(off[t], off[t + 1]) for t in truth["tasks"]]).astype(np.int64)


def grad_envelope(lib, system, batch, D, nthreads=8, modes=ENV_MODES):
    """The oracle's density-contracted gradient and its sensitivity to last-bit input
    changes (the perturbations of ``perturbed``; coordinates of atoms move with the
    shells and centres in mode 2)."""
    import copy
    base = lib.driver_grad_contract(system, batch, D, nthreads=nthreads)
    env = np.zeros_like(base)
    for mode in modes:
        sp = copy.copy(system)
        if mode == 2:
            sp.atoms = np.asarray(system.atoms) * (1 + 4 * U)
        g = lib.driver_grad_contract(sp, perturbed(batch, mode), D, nthreads=nthreads)
        env = np.maximum(env, np.abs(g - base))
    return base, env
