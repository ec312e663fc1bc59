"""C-ABI of the engine library and host-side logic (no GPU needed)."""
import ctypes as ct
import os
import re

import numpy as np
import pytest

from libgrpp_b200 import formats, synthetic
from libgrpp_b200.capi import PRODUCT_LIB
from libgrpp_b200.system import CART_ORDER_DIRAC, CART_ORDER_TURBOMOLE, cartesian_list

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in ("libgrpp.h", "libgrpp_b200.h", "libgrpp_f90.h"):
        txt = open(os.path.join(ROOT, "include", h)).read()
        names |= set(re.findall(r"\b(libgrpp_\w+|evaluate_overlap_integral_contracted_|radial_gto_norm_factor_)\s*\(", txt))
    return sorted(names)


@pytest.fixture(scope="module")
def product_handle():
    if not os.path.exists(PRODUCT_LIB):
        from libgrpp_b200.build import build
        build()
    return ct.CDLL(PRODUCT_LIB)


def test_library_exports_every_declared_symbol(product_handle):
    missing = [n for n in declared_symbols() if not hasattr(product_handle, n)]
    assert not missing, missing
    assert hasattr(product_handle, "libgrpp_params")


def test_containers_without_gpu(product_handle):
    """Constructors and parameter setters are host code: they work on a machine without a GPU."""
    L = product_handle
    L.libgrpp_new_shell.restype = ct.c_void_p
    L.libgrpp_get_shell_size.argtypes = [ct.c_void_p]
    L.libgrpp_delete_shell.argtypes = [ct.c_void_p]
    L.libgrpp_new_potential.restype = ct.c_void_p
    L.libgrpp_potential_value.restype = ct.c_double
    L.libgrpp_potential_value.argtypes = [ct.c_void_p, ct.c_double]
    o = (ct.c_double * 3)(0, 0, 0)
    c = (ct.c_double * 2)(0.5, 0.0)
    a = (ct.c_double * 2)(1.0, 2.0)
    s = L.libgrpp_new_shell(o, 3, 2, c, a)
    assert L.libgrpp_get_shell_size(s) == 10
    L.libgrpp_delete_shell(s)
    pw = (ct.c_int * 3)(2, 1, 0)
    pc = (ct.c_double * 3)(1.5, 1e-15, -2.0)  # middle term dropped (|c| < 1e-14)
    pa = (ct.c_double * 3)(0.7, 1.0, 0.3)
    p = L.libgrpp_new_potential(1, 0, 3, pw, pc, pa)
    r = 1.3
    want = 1.5 * np.exp(-0.7 * r * r) - 2.0 * r ** -2 * np.exp(-0.3 * r * r)
    assert abs(L.libgrpp_potential_value(p, r) - want) < 1e-14


def test_uninitialised_call_reports_error(product_handle):
    """Integrators before libgrpp_init() zero their outputs and set the error code
    (libgrpp asserts, type1_integrals.c:51)."""
    L = product_handle
    L.libgrpp_finalize()
    L.libgrpp_new_shell.restype = ct.c_void_p
    L.libgrpp_new_potential.restype = ct.c_void_p
    L.libgrpp_type1_integrals.argtypes = [ct.c_void_p, ct.c_void_p, ct.POINTER(ct.c_double), ct.c_void_p,
                                          ct.POINTER(ct.c_double)]
    o = (ct.c_double * 3)(0, 0, 0)
    c = (ct.c_double * 1)(1.0)
    a = (ct.c_double * 1)(1.0)
    s = L.libgrpp_new_shell(o, 0, 1, c, a)
    pw = (ct.c_int * 1)(2)
    p = L.libgrpp_new_potential(0, 0, 1, pw, c, a)
    out = (ct.c_double * 1)(123.0)
    L.libgrpp_type1_integrals(s, s, o, p, out)
    assert out[0] == 0.0
    assert L.libgrpp_b200_last_error() == 4  # LIBGRPP_B200_ERR_NOT_INIT
    L.libgrpp_init()


def test_cartesian_orders():
    assert cartesian_list(2, CART_ORDER_DIRAC).tolist() == [[2, 0, 0], [1, 1, 0], [1, 0, 1], [0, 2, 0], [0, 1, 1], [0, 0, 2]]
    assert cartesian_list(2, CART_ORDER_TURBOMOLE).tolist() == [[2, 0, 0], [1, 1, 0], [1, 0, 1], [0, 2, 0], [0, 1, 1], [0, 0, 2]]
    d3, t3 = cartesian_list(3, CART_ORDER_DIRAC).tolist(), cartesian_list(3, CART_ORDER_TURBOMOLE).tolist()
    assert sorted(d3) == sorted(t3) and len(d3) == 10


def test_synthetic_workloads_are_seeded():
    a, b = synthetic.config1(), synthetic.config1()
    assert len(a.shells) == 320 and len(a.centres) == 64
    assert np.array_equal(a.shells[17].alpha, b.shells[17].alpha)
    d = np.linalg.norm(a.atoms[:, None] - a.atoms[None], axis=-1) + np.eye(64) * 100
    assert d.min() >= 3.0 and a.atoms.max() <= 40.0
    c0 = synthetic.config0()
    assert c0.n_basis() == 40 and len(c0.all_tasks()[0]) == 64
    c2 = synthetic.config2()
    assert len(c2.atoms) == 48 and len(c2.centres) == 16


def test_lower_triangle_roundtrip(tmp_path):
    M = np.tril(np.random.default_rng(1).normal(size=(7, 7)))
    M[2, 1] = 1e-15
    p = tmp_path / "m.txt"
    formats.write_lower_triangle(p, M)
    R = formats.read_lower_triangle(p)
    M[2, 1] = 0.0
    assert np.allclose(R, M, rtol=1e-15, atol=0)


def test_batch_arrays_block_offsets():
    S = synthetic.config0()
    b = S.batch()
    off = b.block_offsets()
    assert off[-1] == 40 * 40
    assert b.struct.n_tasks == 64


def test_noalloc_rejects_malformed_batch_on_the_host():
    """The allocation-free entry point checks the batch on the host before any CUDA call:
    a potential power of 3, a GRPP potential index past n_pots or a centre GRPP index past
    n_grpps returns LIBGRPP_B200_ERR_INVALID with no device present."""
    from libgrpp_b200.capi import LibGRPP
    from libgrpp_b200.system import BatchArrays
    lib = LibGRPP(PRODUCT_LIB)
    base = synthetic.config0().batch()
    d0 = {k: v for k, v in base.__dict__.items() if not k.startswith("_")}

    def bad(**changes):
        d = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d0.items()}
        for k, f in changes.items():
            f(d[k])
        return BatchArrays(**d)

    def set0(v):
        v[0] = 3

    def set_idx(n):
        def f(v):
            v[0] = n
        return f

    for batch, what in ((bad(pot_powers=set0), "power"),
                        (bad(grpp_pot_list=set_idx(len(base.pot_L))), "GRPP potential index"),
                        (bad(centre_grpp=set_idx(len(base.grpp_UL))), "centre GRPP index")):
        with pytest.raises(RuntimeError, match=what):
            lib.type2_batch_noalloc(batch)
        assert lib.last_error() == 1  # LIBGRPP_B200_ERR_INVALID
