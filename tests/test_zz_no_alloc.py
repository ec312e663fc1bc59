"""The allocation-free entry point libgrpp_b200_type2_batch_noalloc.

It exists for callers that must not trigger device allocations (processes whose
device memory belongs to a pool or a framework allocator, services with a fixed
device footprint): all its device data sit in static device arrays, with a
32 MiB scratch array shared by all calls. Its output must equal the arep blocks
of the regular batched entry point (libgrpp_b200_full_grpp_batch) for GRPPs
made of averaged (AREP) potentials only, call after call, even though the
scratch array keeps the previous call's contents, and the oracle's on the same
tasks.

This file is collected last, so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process.
"""
import numpy as np
import pytest

from libgrpp_b200 import synthetic
from tests.util import parity

pytestmark = pytest.mark.gpu


def _arep_only(S):
    for g in S.grpps:
        g.UL = None
        g.so = []
        g.oc = []
    return S


LMAX = 2  # s, p, d shells


def _moderate_system():
    """Three atoms with AREP projectors l = 0..4 and s, p, d shells of 6 primitives with
    exponents in [0.1, 20]: blocks libgrpp evaluates to many significant digits (its own
    sensitivity to last-bit input changes stays below 1.2e-10 on values up to 630), so
    two correct implementations agree to the tolerance of record. On f and g shells, or
    with exponents up to 5000, libgrpp's results can move by as much as the values under
    last-bit input changes, and no fixed tolerance between two implementations holds."""
    from libgrpp_b200.system import System
    rng = np.random.default_rng(8)
    xyz = np.array([[0.0, 0.0, 0.0], [1.9, 0.4, -0.7], [-0.8, 2.2, 1.1]])
    grpps = [synthetic._scalar_grpp(rng, 4, 4) for _ in range(3)]
    shells = [synthetic._shell(rng, xyz[i], L, 6, amin=0.1, amax=20.0) for i in range(3) for L in range(LMAX + 1)]
    return System(shells, grpps, [(xyz[i].copy(), i) for i in range(3)], synthetic.CART_ORDER_TURBOMOLE)


def test_noalloc_matches_batched_entry_point(gpu_lib):
    S0 = _arep_only(synthetic.config0())
    S2 = _arep_only(_moderate_system())
    for batch in (S0.batch(), S2.batch()):
        want = gpu_lib.full_grpp_batch(batch)[0]
        first = gpu_lib.type2_batch_noalloc(batch)
        second = gpu_lib.type2_batch_noalloc(batch)
        for got in (first, second):
            ok, ab, rel, _ = parity(got, want)
            assert ok, (ab, rel)
        assert np.array_equal(first, second)


def test_noalloc_mixed_batch_against_oracle(gpu_lib, oracle_lib):
    """One-centre tasks (both shells on the potential's atom) and a centre whose GRPP has no
    AREP potential (its blocks are zero) in one batch, against the batched entry point element
    by element and against the oracle at the tolerance of record."""
    from libgrpp_b200.system import GRPP
    S = _arep_only(_moderate_system())
    S.grpps.append(GRPP())
    S.centres.append((np.array([0.6, -1.3, 2.0]), len(S.grpps) - 1))
    batch = S.batch()
    want = gpu_lib.full_grpp_batch(batch)[0]
    got = gpu_lib.type2_batch_noalloc(batch)
    ok, ab, rel, _ = parity(got, want)
    assert ok, (ab, rel)
    ref = oracle_lib.driver_full_batch(batch, nthreads=8)[0]
    ok, ab, rel, _ = parity(got, ref)
    assert ok, (ab, rel)
    off = batch.block_offsets()
    empty = [t for t in range(len(batch.task_c)) if batch.task_c[t] == len(S.centres) - 1]
    assert empty and all(np.all(got[off[t]:off[t + 1]] == 0.0) for t in empty)


def test_noalloc_rejects_oversized_batch(gpu_lib):
    S = synthetic.config1()
    a, b, c = S.all_tasks()
    batch = S.batch(a[:200000], b[:200000], c[:200000])
    with pytest.raises(RuntimeError, match="bytes of device memory"):
        gpu_lib.type2_batch_noalloc(batch)
    assert gpu_lib.last_error() == 1  # LIBGRPP_B200_ERR_INVALID
