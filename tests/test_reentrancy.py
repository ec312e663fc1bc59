"""Re-entrancy of the single-call C API.

libgrpp's outercore term writes the caller's outercore shells' origins during a call
(libgrpp/outercore_integrals.c:107-111), so one GRPP object used from several threads for
different centres races there. This library writes no caller object: several host threads
calling libgrpp_full_grpp_integrals on one shared libgrpp_grpp_t (with outercore shells),
for different shell pairs and different centres at the same time, get exactly the serial
results, and the outercore shells' origins keep the values the caller gave them.
"""
import ctypes as ct
import threading

import numpy as np
import pytest

from libgrpp_b200 import synthetic
from libgrpp_b200.system import ncart

pytestmark = pytest.mark.gpu


class Shell(ct.Structure):
    _fields_ = [("L", ct.c_int), ("cart_size", ct.c_int), ("cart_list", ct.POINTER(ct.c_int)),
                ("num_primitives", ct.c_int), ("coeffs", ct.POINTER(ct.c_double)), ("alpha", ct.POINTER(ct.c_double)),
                ("origin", ct.c_double * 3)]


class Grpp(ct.Structure):
    _fields_ = [("n_arep", ct.c_int), ("n_esop", ct.c_int), ("n_oc_shells", ct.c_int), ("U_L", ct.c_void_p),
                ("U_arep", ct.c_void_p), ("U_esop", ct.c_void_p), ("U_oc", ct.c_void_p),
                ("oc_shells", ct.POINTER(ct.POINTER(Shell)))]


def _oc_origins(handle):
    g = ct.cast(ct.c_void_p(handle), ct.POINTER(Grpp)).contents
    return np.array([[g.oc_shells[i].contents.origin[d] for d in range(3)] for i in range(g.n_oc_shells)])


def test_concurrent_calls_on_one_grpp_object(gpu_lib):
    S = synthetic.moderate_heavy_system(seed=13)
    gpu_lib.set_cartesian_order(S.cart_order)
    hs = [gpu_lib.new_shell(s) for s in S.shells]
    shared = gpu_lib.new_grpp(S.grpps[0])  # one GRPP object serves every centre and thread
    before = _oc_origins(shared)
    assert len(before) > 0
    # two centres, far from the outercore shells' stored origins
    centres = [np.array([0.0, 0.0, 0.0]), np.array([1.1, -0.6, 2.3]), np.array([-3.0, 1.0, 0.5])]
    rng = np.random.default_rng(2)
    jobs = [(int(i), int(j), int(c)) for i, j, c in zip(rng.integers(0, len(hs), 48), rng.integers(0, len(hs), 48),
                                                          rng.integers(0, len(centres), 48))]

    def call(job):
        i, j, c = job
        return gpu_lib.full(hs[i], hs[j], shared, centres[c], ncart(S.shells[i].L), ncart(S.shells[j].L))

    serial = [call(job) for job in jobs]
    results = [None] * len(jobs)
    errors = []

    def worker(k):
        try:
            for q in range(k, len(jobs), 4):
                results[q] = call(jobs[q])
        except Exception as e:  # reported below
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for q in range(len(jobs)):
        for x, y in zip(results[q], serial[q]):
            assert np.array_equal(x, y), jobs[q]
    assert np.array_equal(_oc_origins(shared), before)
