"""The Fortran ABI (include/libgrpp_f90.h): libgrpp's Fortran-callable symbols
(libgrpp/fortran.c:29-1083), every argument by address, 32-bit integers. Each entry
point is called through ctypes exactly as gfortran would call it, on this library and
on libgrpp compiled from its sources (whose fortran.c is part of the build), with the
same arguments, and the results are compared at the tolerance of record."""
import ctypes as ct

import numpy as np
import pytest

from libgrpp_b200 import synthetic
from libgrpp_b200.capi import PRODUCT_LIB
from libgrpp_b200.system import ncart
from tests.util import truth_parity

D = ct.POINTER(ct.c_double)
I32 = ct.POINTER(ct.c_int32)


def _d(x):
    a = np.ascontiguousarray(np.atleast_1d(x), dtype=np.float64)
    return a, a.ctypes.data_as(D)


def _i(x):
    a = np.ascontiguousarray(np.atleast_1d(x), dtype=np.int32)
    return a, a.ctypes.data_as(I32)


class Args:
    """Keeps the argument arrays alive for the call."""

    def __init__(self):
        self.keep = []

    def d(self, x):
        a, p = _d(x)
        self.keep.append(a)
        return p

    def i(self, x):
        a, p = _i(x)
        self.keep.append(a)
        return p

    def shell(self, s):
        return [self.d(s.origin), self.i(s.L), self.i(len(s.alpha)), self.d(s.coeffs), self.d(s.alpha)]

    def pot(self, p, with_L=True, with_J=False):
        out = [self.i(p.L)] if with_L else []
        if with_J:
            out.append(self.i(p.J))
        return out + [self.i(len(p.alpha)), self.i(p.powers), self.d(p.coeffs), self.d(p.alpha)]


def _call(lib, name, args):
    f = getattr(lib, name)
    f.restype = None
    f(*args)


def test_nuclear_model_functions_f90(ref_lib):
    """The host-code entry points (rms radii, densities, potentials) against libgrpp's."""
    P, R = ct.CDLL(PRODUCT_LIB), ref_lib.lib
    for name, vals in (("libgrpp_coulomb_potential_fermi_", (3e-5, 19.0, 6.5e-5, 1.1e-5)),
                       ("libgrpp_coulomb_potential_fermi_bubble_", (3e-5, 19.0, 6.5e-5, 1.1e-5, 0.3)),
                       ("libgrpp_charge_density_gaussian_", (2e-5, 19.0, 7e-5)),
                       ("libgrpp_coulomb_potential_ball_", (2e-5, 19.0, 7e-5))):
        out = []
        for L in (P, R):
            a = Args()
            res = np.zeros(1)
            _call(L, name, [a.d(v) for v in vals] + [res.ctypes.data_as(D)])
            out.append(res[0])
        assert abs(out[0] - out[1]) <= 1e-12 * abs(out[1]), (name, out)
    for L_ in (P, R):
        a = Args()
        c, aa, err = np.zeros(1), np.zeros(1), np.zeros(1, np.int32)
        _call(L_, "libgrpp_estimate_fermi_model_parameters_", [a.d(4.1), c.ctypes.data_as(D), aa.ctypes.data_as(D),
                                                               err.ctypes.data_as(I32)])
        assert err[0] == 1 and c[0] > 0


@pytest.mark.gpu
def test_f90_entry_points_match_reference(gpu_lib, ref_lib):
    S = synthetic.moderate_heavy_system(seed=5)
    P, R = gpu_lib.lib, ref_lib.lib
    g = S.grpps[0]
    C = S.centres[0][0]
    rng = np.random.default_rng(3)
    order = np.array([1], np.int32)
    for L_ in (P, R):
        _call(L_, "libgrpp_set_cartesian_order_", [order.ctypes.data_as(I32)])
        _call(L_, "libgrpp_init_", [])
    for _ in range(4):
        i, j = (int(x) for x in rng.integers(0, len(S.shells), 2))
        si, sj = S.shells[i], S.shells[j]
        n = ncart(si.L) * ncart(sj.L)
        cases = [("libgrpp_type1_integrals_", lambda a: a.shell(si) + a.shell(sj) + [a.d(C)] + a.pot(g.UL, with_L=False), 1),
                 ("libgrpp_type2_integrals_", lambda a: a.shell(si) + a.shell(sj) + [a.d(C)] + a.pot(g.arep[2]), 1),
                 ("libgrpp_spin_orbit_integrals_", lambda a: a.shell(si) + a.shell(sj) + [a.d(C)] + a.pot(g.so[1]), 3),
                 ("libgrpp_overlap_integrals_", lambda a: a.shell(si) + a.shell(sj), 1),
                 ("libgrpp_kinetic_energy_integrals_", lambda a: a.shell(si) + a.shell(sj), 1),
                 ("libgrpp_momentum_integrals_", lambda a: a.shell(si) + a.shell(sj), 3),
                 ("libgrpp_nuclear_attraction_integrals_point_charge_",
                  lambda a: a.shell(si) + a.shell(sj) + [a.d(C), a.i(55)], 1),
                 ("libgrpp_nuclear_attraction_integrals_charged_ball_",
                  lambda a: a.shell(si) + a.shell(sj) + [a.d(C), a.i(55), a.d(1.3e-4)], 1),
                 ("libgrpp_nuclear_attraction_integrals_",
                  lambda a: a.shell(si) + a.shell(sj) + [a.d(C), a.i(55), a.i(3), a.d([1.1e-4, 1.0e-5, 0.0])], 1),
                 ("libgrpp_nuclear_attraction_integrals_gaussian_model_",
                  lambda a: a.shell(si) + a.shell(sj) + [a.d(C), a.i(55), a.d(1.3e-4)], 1),
                 ("libgrpp_nuclear_attraction_integrals_fermi_model_",
                  lambda a: a.shell(si) + a.shell(sj) + [a.d(C), a.i(55), a.d(1.1e-4), a.d(1.0e-5)], 1),
                 ("libgrpp_type1_integrals_gradient_",
                  lambda a: a.shell(si) + a.shell(sj) + [a.d(C)] + a.pot(g.UL, with_L=False) + [a.d(si.origin)], 3),
                 ("libgrpp_type2_integrals_gradient_",
                  lambda a: a.shell(si) + a.shell(sj) + [a.d(C)] + a.pot(g.arep[1]) + [a.d(C)], 3),
                 ("libgrpp_spin_orbit_integrals_gradient_",
                  lambda a: a.shell(si) + a.shell(sj) + [a.d(C)] + a.pot(g.so[0]) + [a.d(sj.origin)], 9)]
        for p, sh in g.oc[:3]:
            cases.append(("libgrpp_outercore_potential_integrals_part_1_",
                          lambda a, p=p, sh=sh: a.shell(si) + a.shell(sj) + [a.d(C)] + a.pot(p, with_J=True) +
                          [a.i(len(sh.alpha)), a.d(sh.coeffs), a.d(sh.alpha)], 4))
        for (p1, s1), (p2, s2) in ((g.oc[1], g.oc[1]), (g.oc[1], g.oc[3]), (g.oc[2], g.oc[4])):
            cases.append(("libgrpp_outercore_potential_integrals_part_2_",
                          lambda a, p1=p1, s1=s1, p2=p2, s2=s2: a.shell(si) + a.shell(sj) + [a.d(C)] +
                          a.pot(p1, with_J=True) + [a.i(len(s1.alpha)), a.d(s1.coeffs), a.d(s1.alpha)] +
                          a.pot(p2, with_J=True) + [a.i(len(s2.alpha)), a.d(s2.coeffs), a.d(s2.alpha)], 4))
        for name, build, nout in cases:
            res = []
            for L_ in (P, R):
                a = Args()
                outs = [np.full(n, 0.25) if "part_" in name else np.zeros(n) for _ in range(nout)]  # parts accumulate
                _call(L_, name, build(a) + [o.ctypes.data_as(D) for o in outs])
                res.append(np.concatenate(outs))
            ok, rep = truth_parity(res[0], res[1])
            assert ok, (name, i, j, rep)
    # the auxiliary overlap of single components and the radial norm factor
    s = S.shells[4]
    vals = []
    for L_ in (P, R):
        a = Args()
        v = np.zeros(1)
        _call(L_, "radial_gto_norm_factor_", [a.i(s.L), a.i(len(s.alpha)), a.d(s.coeffs), a.d(s.alpha), v.ctypes.data_as(D)])
        vals.append(v[0])
    assert abs(vals[0] - vals[1]) <= 1e-12 * abs(vals[1])
