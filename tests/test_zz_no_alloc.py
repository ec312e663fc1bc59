"""The allocation-free entry point libgrpp_b200_type2_batch_noalloc.

It exists for callers that must not trigger device allocations (code inside
CUDA graph capture, processes whose device memory belongs to a pool or a
framework allocator, services with a fixed device footprint): all its device
data sit in static device arrays, with a 32 MiB scratch array shared by all
calls. Its output must equal the arep blocks of the regular batched entry
point (libgrpp_b200_full_grpp_batch) for GRPPs made of averaged (AREP)
potentials only, call after call, even though the scratch array keeps the
previous call's contents.

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


def test_noalloc_matches_batched_entry_point(gpu_lib):
    S0 = _arep_only(synthetic.config0())
    S2 = _arep_only(synthetic.config2(seed=5, n_heavy=3, n_h=3, lmax=4, box=9.0))
    a, b, c = S2.all_tasks()
    sel = np.random.default_rng(3).choice(len(a), 400, replace=False)
    for batch in (S0.batch(), S2.batch(a[sel], b[sel], c[sel])):
        want = gpu_lib.full_grpp_batch(batch)[0]
        first = gpu_lib.type2_batch_noalloc(batch)
        second = gpu_lib.type2_batch_noalloc(batch)
        for got in (first, second):
            ok, ab, rel, _ = parity(got, want)
            assert ok, (ab, rel)
        assert np.array_equal(first, second)


def test_noalloc_rejects_oversized_batch(gpu_lib):
    S = synthetic.config1()
    a, b, c = S.all_tasks()
    batch = S.batch(a[:200000], b[:200000], c[:200000])
    with pytest.raises(RuntimeError, match="bytes of device memory"):
        gpu_lib.type2_batch_noalloc(batch)
    assert gpu_lib.last_error() == 1  # LIBGRPP_B200_ERR_INVALID
