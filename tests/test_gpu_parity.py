"""Parity of the CUDA engine with libgrpp (golden fixtures) and with the oracle.

Criterion of record, element by element (tests.util.truth_parity):
    |gpu - ref| <= max(1e-10, 1e-9 |ref| if |ref| > 1e-6)
1e-10 absolute is libgrpp's own comparator (test/compare_matrices.c:25). On the
synthetic workloads a few blocks are ones on which libgrpp itself keeps few or
no significant digits (tight high-l primitives, far potential centres): its
result moves by up to the size of the values when its inputs move by a few
units in the last place, while the exact value does not. For the tasks of those
blocks tests/golden/truth_<name>.npz holds the exact values (binary128,
oracle/truth_quad.c) and libgrpp's own distance from them over 31 runs
(refdev); an element there that misses the strict bound must satisfy
    |gpu - truth| <= max(1e-10, 1e-9 |truth|, 2 refdev).
Each test prints how many elements were judged against the truth.
"""
import numpy as np
import pytest

from libgrpp_b200 import synthetic
from libgrpp_b200.system import ncart
from tests.util import (COMPS, assemble_lower, full_system, load_fixture, load_truth, strict_tol, system_from_fixture,
                        truth_parity, truth_selection)

pytestmark = pytest.mark.gpu

SYNTHETIC = ("config1", "config1_moderate", "config2")


@pytest.mark.parametrize("name", ["h2o", "cs", "kcs", "tho", "uo2"] + list(SYNTHETIC))
def test_fixture_blocks(gpu_lib, name):
    batch, z = load_fixture(name)
    truth = load_truth(name)
    if name in SYNTHETIC:
        assert truth is not None, f"tests/golden/truth_{name}.npz missing"
    sel = truth_selection(batch, truth)
    outs = gpu_lib.full_grpp_batch(batch)
    for m, comp in enumerate(COMPS):
        ok, rep = truth_parity(outs[m], z["ref_" + comp], truth, sel, comp)
        print(f"{name} {comp}: max abs {rep['max_abs']:.2e}, strict misses {rep['strict_fail']} "
              f"(judged against the truth: {rep['truth_checked']}, failing {rep['truth_fail']}, worst "
              f"|gpu-truth|/bound {rep['worst_truth_ratio']:.2f}; on the truth tasks max |ref-truth| "
              f"{rep['max_ref_truth']:.2e}, max |gpu-truth| {rep['max_got_truth']:.2e})")
        assert ok, (name, comp, rep)


@pytest.mark.parametrize("name", ["kcs", "tho", "uo2"])
def test_full_matrices_against_shipped(gpu_lib, name):
    """Every ordered shell pair x every centre of libgrpp's ThO, UO2 and KCs tests, summed into
    the full AREP and SO matrices and compared element by element with libgrpp's shipped
    matrices (test/<name>/arep.txt, so_*.txt), as libgrpp's own ctest does. Where libgrpp's C
    path and its shipped (Fortran-driver) matrix differ beyond the tolerance (one KCs element),
    the element is judged against its binary128 value."""
    batch, z = full_system(name)
    got = assemble_lower(batch, gpu_lib.full_grpp_batch(batch), int(z["n_shells"]))
    sel = z["truth_idx"]
    truth = {k: z[k] for k in z.files if k.startswith(("truth_", "refdev_"))} if len(sel) else None
    for comp, g in zip(COMPS, got):
        ok, rep = truth_parity(g, z["shipped_" + comp], truth, sel if len(sel) else None, comp)
        print(f"{name} {comp} ({int(z['n_basis'])}x{int(z['n_basis'])}): max abs {rep['max_abs']:.2e}, "
              f"judged against the truth {rep['truth_checked']} (worst |gpu-truth|/bound {rep['worst_truth_ratio']:.2f})")
        assert ok, (name, comp, rep)


def test_moderate_config1_is_strict_outside_two_tasks(gpu_lib):
    """Config 1 with exponents in [0.1, 50]: every element meets 1e-10 / 1e-9 against libgrpp
    except in the tasks the truth fixture lists (an f and a g shell on one atom with the centre
    3.3 bohr away, where libgrpp's spread reaches 2e-5 even so, and one g x g task at 1e-10)."""
    batch, z = load_fixture("config1_moderate")
    truth = load_truth("config1_moderate")
    assert len(truth["tasks"]) <= 2
    off = batch.block_offsets()
    keep = np.ones(int(off[-1]), dtype=bool)
    keep[truth_selection(batch, truth)] = False
    outs = gpu_lib.full_grpp_batch(batch)
    for m, comp in enumerate(COMPS):
        err = np.abs(outs[m] - z["ref_" + comp])[keep]
        assert np.all(err <= strict_tol(z["ref_" + comp])[keep]), (comp, float(err.max()))


def test_config0_full_matrix(gpu_lib, oracle_lib):
    S = synthetic.config0()
    b = S.batch()
    got = gpu_lib.full_grpp_batch(b)
    want = oracle_lib.driver_full_batch(b, nthreads=8)
    for m in range(4):
        ok, rep = truth_parity(got[m], want[m])
        print(f"config0 {COMPS[m]}: max abs {rep['max_abs']:.2e}")
        assert ok, (COMPS[m], rep)
    assert S.assemble(b, got[0]).shape == (40, 40)


def _strict(got, want, what):
    ok, rep = truth_parity(np.ravel(got), np.ravel(want))
    assert ok, (what, rep)


def test_single_task_terms(gpu_lib, oracle_lib):
    """libgrpp_type1/type2/spin_orbit/outercore_potential/full_grpp_integrals through the
    single-call C API, against the same calls on the oracle."""
    S = synthetic.moderate_heavy_system()
    for lib in (gpu_lib, oracle_lib):
        lib.set_cartesian_order(S.cart_order)
    rng = np.random.default_rng(0)
    for _ in range(8):
        i, j = (int(x) for x in rng.integers(0, len(S.shells), 2))
        C, gi = S.centres[int(rng.integers(0, 2))]
        g = S.grpps[gi]
        si, sj = S.shells[i], S.shells[j]
        nA, nB = ncart(si.L), ncart(sj.L)
        res = []
        for lib in (gpu_lib, oracle_lib):
            hA, hB = lib.new_shell(si), lib.new_shell(sj)
            pots = [lib.new_potential(p) for p, _ in g.oc]
            ocs = [lib.new_shell(sh) for _, sh in g.oc]
            o = [np.zeros(nA * nB) for _ in range(4)]
            import ctypes as ct
            D_ = ct.POINTER(ct.c_double)
            lib.lib.libgrpp_outercore_potential_integrals(
                hA, hB, np.ascontiguousarray(C).ctypes.data_as(D_), len(pots), (ct.c_void_p * len(pots))(*pots),
                (ct.c_void_p * len(ocs))(*ocs), *[x.ctypes.data_as(D_) for x in o])
            res.append([lib.type1(hA, hB, C, lib.new_potential(g.UL), nA, nB),
                        lib.type2(hA, hB, C, lib.new_potential(g.arep[2]), nA, nB),
                        *lib.spin_orbit(hA, hB, C, lib.new_potential(g.so[1]), nA, nB),
                        *o,
                        *lib.full(hA, hB, lib.new_grpp(g), C, nA, nB)])
        for k, (x, y) in enumerate(zip(*res)):
            _strict(x, y, (i, j, k))


def test_per_term_gradient_entry_points(gpu_lib, oracle_lib):
    """The five *_gradient entry points (libgrpp/grpp_integrals_gradient.c:123-272) on the GPU
    against the same calls on the oracle, for D on shell A's atom, shell B's atom and the centre."""
    S = synthetic.moderate_heavy_system(seed=9)
    for lib in (gpu_lib, oracle_lib):
        lib.set_cartesian_order(S.cart_order)
    rng = np.random.default_rng(1)
    for _ in range(4):
        i, j = (int(x) for x in rng.integers(0, len(S.shells), 2))
        C, gi = S.centres[int(rng.integers(0, 2))]
        g = S.grpps[gi]
        si, sj = S.shells[i], S.shells[j]
        nA, nB = ncart(si.L), ncart(sj.L)
        for D in (si.origin, sj.origin, C):
            res = []
            for lib in (gpu_lib, oracle_lib):
                hA, hB = lib.new_shell(si), lib.new_shell(sj)
                res.append([lib.type1_gradient(hA, hB, C, lib.new_potential(g.UL), D, nA, nB),
                            lib.type2_gradient(hA, hB, C, lib.new_potential(g.arep[1]), D, nA, nB),
                            lib.spin_orbit_gradient(hA, hB, C, lib.new_potential(g.so[2]), D, nA, nB),
                            lib.outercore_gradient(hA, hB, C, [lib.new_potential(p) for p, _ in g.oc],
                                                   [lib.new_shell(sh) for _, sh in g.oc], D, nA, nB),
                            lib.full_gradient(hA, hB, lib.new_grpp(g), C, D, nA, nB)])
            for k, (x, y) in enumerate(zip(*res)):
                _strict(x, y, (i, j, k, tuple(np.round(D, 3))))


def test_h2o_gradients(gpu_lib):
    """d V / d R_atom for all atoms against libgrpp's gradient matrices (test/H2O/*_grad_*)."""
    batch, z = load_fixture("h2o")
    S = system_from_fixture(z)
    gpu_lib.set_cartesian_order(S.cart_order)
    hs = [gpu_lib.new_shell(s) for s in S.shells]
    hg = [gpu_lib.new_grpp(g) for g in S.grpps]
    off = S.basis_offsets()
    n = int(off[-1])
    nat = len(S.atoms)
    G = np.zeros((4, nat, 3, n, n))
    for i, si in enumerate(S.shells):
        for j, sj in enumerate(S.shells):
            for at in range(nat):
                for C, gi in S.centres:
                    G[:, at, :, off[i]:off[i + 1], off[j]:off[j + 1]] += gpu_lib.full_gradient(
                        hs[i], hs[j], hg[gi], C, S.atoms[at], ncart(si.L), ncart(sj.L))
    tri = np.tril_indices(n)
    got = G[:, :, :, tri[0], tri[1]]
    _strict(got, z["ref_grad_lower"], "h2o gradients")


def test_large_batch_runs_in_chunks(gpu_lib):
    """A batch larger than one chunk (32768 tasks, and here also more than 2^27 radial
    entries) through the batched entry point, which splits it and overlaps the chunks,
    equals the same tasks run as one plan."""
    S = synthetic.config1()
    a, b, c = S.all_tasks()
    La = np.array([s.L for s in S.shells])
    gg = np.where((La[a] == 4) & (La[b] == 4))[0][:80000]  # 2295 entries per g x g task
    batch = S.batch(a[gg], b[gg], c[gg])
    chunked = gpu_lib.full_grpp_batch(batch)
    plan = gpu_lib.plan(batch, 0)
    plan.execute()
    whole = plan.outputs()
    plan.close()
    for x, y in zip(chunked, whole):
        assert np.array_equal(x, y)


def test_batched_call_into_page_locked_outputs(gpu_lib):
    """The batched call writes into caller arrays in page-locked memory (libgrpp_b200_host_alloc)
    exactly what it returns in fresh arrays; the arrays are reused across calls."""
    S = synthetic.config1()
    a, b, c = S.all_tasks()
    sel = np.random.default_rng(7).choice(len(a), 3000, replace=False)
    batch = S.batch(a[sel], b[sel], c[sel])
    n = int(batch.block_offsets()[-1])
    fresh = gpu_lib.full_grpp_batch(batch)
    outs = [gpu_lib.pinned_empty(n + 5) for _ in range(4)]
    for _ in range(2):
        got = gpu_lib.full_grpp_batch(batch, out=outs)
        for x, y in zip(got, fresh):
            assert np.array_equal(x, y)
    with pytest.raises(ValueError):
        gpu_lib.full_grpp_batch(batch, out=[np.empty(n, dtype=np.float32) for _ in range(4)])
