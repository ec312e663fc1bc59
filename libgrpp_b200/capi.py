"""ctypes binding of the libgrpp C API.

One binding serves every library that exports libgrpp's C interface
(libgrpp/libgrpp.h:33-231): the CUDA engine ``libgrpp_b200/libgrpp_b200.so``,
and, for tests only, the CPU oracle and the compiled reference. Objects are
built through the library's own constructors, exactly as a C caller would.
"""
from __future__ import annotations

import ctypes as ct
import os
import weakref

import numpy as np

from .system import GRPP, Potential, Shell, ncart

_D = ct.POINTER(ct.c_double)
_I = ct.POINTER(ct.c_int)
_V = ct.c_void_p

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PRODUCT_LIB = os.path.join(ROOT, "libgrpp_b200", "libgrpp_b200.so")


def _dp(a):
    return a.ctypes.data_as(_D)


def _ip(a):
    return a.ctypes.data_as(_I)


class LibGRPP:
    """A loaded library exporting the libgrpp C API."""

    def __init__(self, path: str):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built")
        self.path = path
        self.lib = ct.CDLL(path, mode=getattr(os, "RTLD_LOCAL", 0) | getattr(os, "RTLD_NOW", 2))
        L = self.lib
        proto = {
            "libgrpp_init": (None, []),
            "libgrpp_finalize": (None, []),
            "libgrpp_is_initialized": (ct.c_int, []),
            "libgrpp_set_cartesian_order": (None, [ct.c_int]),
            "libgrpp_new_shell": (_V, [_D, ct.c_int, ct.c_int, _D, _D]),
            "libgrpp_delete_shell": (None, [_V]),
            "libgrpp_get_shell_size": (ct.c_int, [_V]),
            "libgrpp_new_potential": (_V, [ct.c_int, ct.c_int, ct.c_int, _I, _D, _D]),
            "libgrpp_delete_potential": (None, [_V]),
            "libgrpp_potential_value": (ct.c_double, [_V, ct.c_double]),
            "libgrpp_new_grpp": (_V, []),
            "libgrpp_grpp_set_local_potential": (None, [_V, _V]),
            "libgrpp_grpp_add_averaged_potential": (None, [_V, _V]),
            "libgrpp_grpp_add_spin_orbit_potential": (None, [_V, _V]),
            "libgrpp_grpp_add_outercore_potential": (None, [_V, _V, _V]),
            "libgrpp_delete_grpp": (None, [_V]),
            "libgrpp_type1_integrals": (None, [_V, _V, _D, _V, _D]),
            "libgrpp_type2_integrals": (None, [_V, _V, _D, _V, _D]),
            "libgrpp_spin_orbit_integrals": (None, [_V, _V, _D, _V, _D, _D, _D]),
            "libgrpp_outercore_potential_integrals": (None, [_V, _V, _D, ct.c_int, ct.POINTER(_V), ct.POINTER(_V), _D, _D, _D, _D]),
            "libgrpp_full_grpp_integrals": (None, [_V, _V, _V, _D, _D, _D, _D, _D]),
            "libgrpp_full_grpp_integrals_gradient": (None, [_V, _V, _V, _D, _D, ct.POINTER(_D), ct.POINTER(_D), ct.POINTER(_D), ct.POINTER(_D)]),
            "libgrpp_type1_integrals_gradient": (None, [_V, _V, _D, _V, _D, ct.POINTER(_D)]),
            "libgrpp_type2_integrals_gradient": (None, [_V, _V, _D, _V, _D, ct.POINTER(_D)]),
            "libgrpp_spin_orbit_integrals_gradient": (None, [_V, _V, _D, _V, _D, ct.POINTER(_D), ct.POINTER(_D), ct.POINTER(_D)]),
            "libgrpp_outercore_potential_integrals_gradient": (None, [_V, _V, _D, ct.c_int, ct.POINTER(_V), ct.POINTER(_V), _D,
                                                                      ct.POINTER(_D), ct.POINTER(_D), ct.POINTER(_D),
                                                                      ct.POINTER(_D)]),
        }
        for name, (res, args) in proto.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        self._opt("grpp_driver_full_batch", ct.c_int, [_V, ct.c_int64, ct.c_int64, ct.c_int, _D, _D, _D, _D])
        self._opt("grpp_driver_term", ct.c_int, [_V, ct.c_int64, ct.c_int, ct.c_int, _D, _D, _D])
        self._opt("grpp_driver_grad_contract", ct.c_int, [_V, ct.c_int64, ct.c_int64, ct.c_int, _I, _I, _D, ct.c_int, _I, ct.c_int, _D, _D])
        self._opt("grpp_driver_num_threads", ct.c_int, [])
        self._opt("libgrpp_b200_last_error", ct.c_int, [])
        self._opt("libgrpp_b200_last_error_message", ct.c_char_p, [])
        self._opt("libgrpp_b200_full_grpp_batch", ct.c_int, [_V, ct.c_int, _D, _D, _D, _D])
        self._opt("libgrpp_b200_set_device", ct.c_int, [ct.c_int])
        self._opt("libgrpp_b200_host_alloc", _V, [ct.c_size_t])
        self._opt("libgrpp_b200_host_free", None, [_V])
        self._opt("libgrpp_b200_fp64_peak", ct.c_int, [_D])
        self._opt("libgrpp_b200_type2_batch_noalloc", ct.c_int, [_V, _D])
        self._opt("libgrpp_b200_plan_create", _V, [_V, ct.c_int])
        self._opt("libgrpp_b200_plan_create_ex", _V, [_V, ct.c_int, ct.c_int])
        self._opt("libgrpp_b200_autotune_assembly", ct.c_int, [_V, ct.c_int, ct.POINTER(ct.c_double), ct.c_int])
        self._opt("libgrpp_b200_autotune_reset", None, [])
        self._opt("libgrpp_b200_plan_execute", ct.c_int, [_V])
        self._opt("libgrpp_b200_plan_outputs", ct.c_int, [_V, _D, _D, _D, _D])
        self._opt("libgrpp_b200_plan_stats", ct.c_int, [_V, _D, ct.POINTER(ct.c_int64)])
        self._opt("libgrpp_b200_plan_destroy", None, [_V])
        self._opt("libgrpp_b200_plan_counters", ct.c_int, [_V, ct.POINTER(ct.c_uint64), ct.c_int])
        self._opt("libgrpp_b200_plan_set_counting", ct.c_int, [_V, ct.c_int])
        _F = ct.POINTER(ct.c_float)
        _B = ct.POINTER(ct.c_int8)
        self._opt("libgrpp_b200_plan_learned_stats", ct.c_int, [_V, _D, ct.POINTER(ct.c_int64)])
        self._opt("libgrpp_b200_grpp_gradient_contract", ct.c_int,
                  [_V, ct.c_int, _I, _I, _D, ct.c_int, _I, ct.c_int, _D, _D])
        self._opt("libgrpp_b200_grpp_gradient_contract_symmetric", ct.c_int,
                  [_V, ct.c_int, _I, _I, _D, ct.c_int, _I, ct.c_int, _D, _D])
        self._opt("libgrpp_b200_set_level_model", ct.c_int, [_F])
        self._opt("libgrpp_b200_level_samples", ct.c_int, [_V, _F, _B, ct.POINTER(ct.c_int64)])
        self._opt("libgrpp_overlap_integrals", None, [_V, _V, _D])
        self._opt("libgrpp_kinetic_energy_integrals", None, [_V, _V, _D])
        self._opt("libgrpp_momentum_integrals", None, [_V, _V, _D, _D, _D])
        self._opt("libgrpp_overlap_integrals_gradient", None, [_V, _V, _D, ct.POINTER(_D)])
        self._opt("libgrpp_nuclear_attraction_integrals", None, [_V, _V, _D, ct.c_int, ct.c_int, _D, _D])
        self._opt("libgrpp_estimate_nuclear_rms_radius_johnson_1985", ct.c_double, [ct.c_int])
        self._opt("libgrpp_estimate_fermi_model_parameters", ct.c_int, [ct.c_double, _D, _D])
        self._opt("libgrpp_b200_onee_batch", ct.c_int, [_V, ct.c_int, _D, _D, _D])
        self._opt("libgrpp_b200_nuclear_attraction_batch", ct.c_int, [_V, ct.c_int, _D, _D, _D])
        self._opt("libgrpp_b200_type1_numeric_batch", ct.c_int, [_V, _D])
        self._opt("libgrpp_b200_mlp_grad", ct.c_int, [_F, _F, _B, ct.c_int, _F, _F])
        self._opt("libgrpp_b200_mlp_train", ct.c_int, [_F, _B, ct.c_int64, ct.c_int, ct.c_int, ct.c_float, ct.c_uint32, _F, _F])
        self._opt("libgrpp_b200_mlp_predict", ct.c_int, [_F, _F, ct.c_int64, _B])
        self.lib.libgrpp_init()

    def _opt(self, name, res, args):
        f = getattr(self.lib, name, None)
        if f is not None:
            f.restype = res
            f.argtypes = args

    def has(self, name: str) -> bool:
        return getattr(self.lib, name, None) is not None

    # ------------------------------------------------------------ objects
    def set_cartesian_order(self, order: int):
        self.lib.libgrpp_set_cartesian_order(order)

    def new_shell(self, s: Shell) -> int:
        o = np.ascontiguousarray(s.origin, dtype=np.float64)
        c = np.ascontiguousarray(s.coeffs, dtype=np.float64)
        a = np.ascontiguousarray(s.alpha, dtype=np.float64)
        return self.lib.libgrpp_new_shell(_dp(o), int(s.L), len(a), _dp(c), _dp(a))

    def new_potential(self, p: Potential) -> int:
        pw = np.ascontiguousarray(p.powers, dtype=np.int32)
        c = np.ascontiguousarray(p.coeffs, dtype=np.float64)
        a = np.ascontiguousarray(p.alpha, dtype=np.float64)
        return self.lib.libgrpp_new_potential(int(p.L), int(p.J), len(a), _ip(pw), _dp(c), _dp(a))

    def new_grpp(self, g: GRPP) -> int:
        h = self.lib.libgrpp_new_grpp()
        if g.UL is not None:
            self.lib.libgrpp_grpp_set_local_potential(h, self.new_potential(g.UL))
        for p in g.arep:
            self.lib.libgrpp_grpp_add_averaged_potential(h, self.new_potential(p))
        for p in g.so:
            self.lib.libgrpp_grpp_add_spin_orbit_potential(h, self.new_potential(p))
        for p, s in g.oc:
            self.lib.libgrpp_grpp_add_outercore_potential(h, self.new_potential(p), self.new_shell(s))
        return h

    # ------------------------------------------------------------ integrators
    def type1(self, hA, hB, C, hpot, nA, nB):
        out = np.zeros(nA * nB)
        self.lib.libgrpp_type1_integrals(hA, hB, _dp(np.ascontiguousarray(C, dtype=np.float64)), hpot, _dp(out))
        return out.reshape(nA, nB)

    def type2(self, hA, hB, C, hpot, nA, nB):
        out = np.zeros(nA * nB)
        self.lib.libgrpp_type2_integrals(hA, hB, _dp(np.ascontiguousarray(C, dtype=np.float64)), hpot, _dp(out))
        return out.reshape(nA, nB)

    def spin_orbit(self, hA, hB, C, hpot, nA, nB):
        o = [np.zeros(nA * nB) for _ in range(3)]
        self.lib.libgrpp_spin_orbit_integrals(hA, hB, _dp(np.ascontiguousarray(C, dtype=np.float64)), hpot,
                                              _dp(o[0]), _dp(o[1]), _dp(o[2]))
        return [x.reshape(nA, nB) for x in o]

    def full(self, hA, hB, hg, C, nA, nB):
        o = [np.zeros(nA * nB) for _ in range(4)]
        self.lib.libgrpp_full_grpp_integrals(hA, hB, hg, _dp(np.ascontiguousarray(C, dtype=np.float64)),
                                             *[_dp(x) for x in o])
        return [x.reshape(nA, nB) for x in o]

    def full_gradient(self, hA, hB, hg, C, D, nA, nB):
        g = np.zeros((4, 3, nA * nB))
        ptrs = [(_D * 3)(*[g[m, k].ctypes.data_as(_D) for k in range(3)]) for m in range(4)]
        self.lib.libgrpp_full_grpp_integrals_gradient(
            hA, hB, hg, _dp(np.ascontiguousarray(C, dtype=np.float64)), _dp(np.ascontiguousarray(D, dtype=np.float64)),
            *ptrs)
        return g.reshape(4, 3, nA, nB)

    def _grad_ptrs(self, g):
        return [(_D * 3)(*[g[m, k].ctypes.data_as(_D) for k in range(3)]) for m in range(g.shape[0])]

    def type1_gradient(self, hA, hB, C, hpot, D, nA, nB):
        """libgrpp_type1_integrals_gradient: d<A|U|B>/dD, [3, nA, nB]."""
        g = np.zeros((1, 3, nA * nB))
        self.lib.libgrpp_type1_integrals_gradient(hA, hB, _dp(np.ascontiguousarray(C, dtype=np.float64)), hpot,
                                                  _dp(np.ascontiguousarray(D, dtype=np.float64)), self._grad_ptrs(g)[0])
        return g.reshape(3, nA, nB)

    def type2_gradient(self, hA, hB, C, hpot, D, nA, nB):
        """libgrpp_type2_integrals_gradient: [3, nA, nB]."""
        g = np.zeros((1, 3, nA * nB))
        self.lib.libgrpp_type2_integrals_gradient(hA, hB, _dp(np.ascontiguousarray(C, dtype=np.float64)), hpot,
                                                  _dp(np.ascontiguousarray(D, dtype=np.float64)), self._grad_ptrs(g)[0])
        return g.reshape(3, nA, nB)

    def spin_orbit_gradient(self, hA, hB, C, hpot, D, nA, nB):
        """libgrpp_spin_orbit_integrals_gradient: [3 (so_x, so_y, so_z), 3, nA, nB]."""
        g = np.zeros((3, 3, nA * nB))
        p = self._grad_ptrs(g)
        self.lib.libgrpp_spin_orbit_integrals_gradient(hA, hB, _dp(np.ascontiguousarray(C, dtype=np.float64)), hpot,
                                                       _dp(np.ascontiguousarray(D, dtype=np.float64)), p[0], p[1], p[2])
        return g.reshape(3, 3, nA, nB)

    def outercore_gradient(self, hA, hB, C, hpots, hocs, D, nA, nB):
        """libgrpp_outercore_potential_integrals_gradient: [4 (arep, so_x, so_y, so_z), 3, nA, nB]."""
        g = np.zeros((4, 3, nA * nB))
        p = self._grad_ptrs(g)
        n = len(hpots)
        pots = (_V * max(n, 1))(*hpots)
        ocs = (_V * max(n, 1))(*hocs)
        self.lib.libgrpp_outercore_potential_integrals_gradient(
            hA, hB, _dp(np.ascontiguousarray(C, dtype=np.float64)), n, pots, ocs,
            _dp(np.ascontiguousarray(D, dtype=np.float64)), *p)
        return g.reshape(4, 3, nA, nB)

    # ------------------------------------------------------------ one-electron integrals
    def overlap(self, hA, hB, nA, nB):
        out = np.zeros(nA * nB)
        self.lib.libgrpp_overlap_integrals(hA, hB, _dp(out))
        return out.reshape(nA, nB)

    def kinetic(self, hA, hB, nA, nB):
        out = np.zeros(nA * nB)
        self.lib.libgrpp_kinetic_energy_integrals(hA, hB, _dp(out))
        return out.reshape(nA, nB)

    def momentum(self, hA, hB, nA, nB):
        o = [np.zeros(nA * nB) for _ in range(3)]
        self.lib.libgrpp_momentum_integrals(hA, hB, *[_dp(x) for x in o])
        return [x.reshape(nA, nB) for x in o]

    def overlap_gradient(self, hA, hB, D, nA, nB):
        g = np.zeros((1, 3, nA * nB))
        self.lib.libgrpp_overlap_integrals_gradient(hA, hB, _dp(np.ascontiguousarray(D, dtype=np.float64)),
                                                    self._grad_ptrs(g)[0])
        return g.reshape(3, nA, nB)

    def nuclear_attraction(self, hA, hB, C, Z, model, params, nA, nB):
        out = np.zeros(nA * nB)
        p = np.zeros(4) if params is None else np.ascontiguousarray(params, dtype=np.float64)
        self.lib.libgrpp_nuclear_attraction_integrals(hA, hB, _dp(np.ascontiguousarray(C, dtype=np.float64)), int(Z),
                                                      int(model), _dp(p), _dp(out))
        return out.reshape(nA, nB)

    def onee_batch(self, batch, kind):
        """Overlap (kind 0), kinetic (1) or momentum (2: three arrays) blocks of every task's shell pair."""
        n = int(batch.block_offsets()[-1])
        o = [np.zeros(max(n, 1)) for _ in range(3)]
        self._check(self.lib.libgrpp_b200_onee_batch(ct.byref(batch.struct), kind, *[_dp(x) for x in o]),
                    "libgrpp_b200_onee_batch")
        return [x[:n] for x in o[:3 if kind == 2 else 1]]

    def nuclear_attraction_batch(self, batch, model, charges, params=None):
        """Nuclear attraction blocks of every task (nucleus at the task's centre)."""
        n = int(batch.block_offsets()[-1])
        out = np.zeros(max(n, 1))
        q = np.ascontiguousarray(charges, dtype=np.float64)
        p = np.zeros(3 * len(q)) if params is None else np.ascontiguousarray(params, dtype=np.float64).ravel()
        self._check(self.lib.libgrpp_b200_nuclear_attraction_batch(ct.byref(batch.struct), int(model), _dp(q), _dp(p),
                                                                   _dp(out)), "libgrpp_b200_nuclear_attraction_batch")
        return out[:n]

    def type1_numeric_batch(self, batch):
        """<A|U_L|B> of every task by numeric radial quadrature."""
        n = int(batch.block_offsets()[-1])
        out = np.zeros(max(n, 1))
        self._check(self.lib.libgrpp_b200_type1_numeric_batch(ct.byref(batch.struct), _dp(out)),
                    "libgrpp_b200_type1_numeric_batch")
        return out[:n]

    # ------------------------------------------------------------ batched (CPU drivers)
    def driver_full_batch(self, batch, t0=0, t1=None, nthreads=1):
        if t1 is None:
            t1 = len(batch.task_a)
        off = batch.block_offsets()
        n = int(off[t1] - off[t0])
        outs = [np.zeros(max(n, 1)) for _ in range(4)]
        self.lib.grpp_driver_full_batch(ct.byref(batch.struct), t0, t1, nthreads, *[_dp(x) for x in outs])
        return [x[:n] for x in outs]

    def driver_grad_contract(self, system, batch, D, t0=0, t1=None, nthreads=1):
        if t1 is None:
            t1 = len(batch.task_a)
        nat = len(system.atoms)
        g = np.zeros((4, nat, 3))
        sa = np.ascontiguousarray(system.shell_atom, dtype=np.int32)
        ca = np.ascontiguousarray(system.centre_atom, dtype=np.int32)
        xyz = np.ascontiguousarray(system.atoms, dtype=np.float64)
        bo = np.ascontiguousarray(system.basis_offsets()[:-1], dtype=np.int32)
        Dm = np.ascontiguousarray(D, dtype=np.float64)
        self.lib.grpp_driver_grad_contract(ct.byref(batch.struct), t0, t1, nthreads, _ip(sa), _ip(ca), _dp(xyz), nat,
                                           _ip(bo), int(Dm.shape[0]), _dp(Dm), _dp(g))
        return g

    def num_threads(self) -> int:
        return int(self.lib.grpp_driver_num_threads())

    # ------------------------------------------------------------ batched (GPU engine)
    def full_grpp_batch(self, batch, radial_mode=0, out=None):
        """AREP, SO_x, SO_y, SO_z blocks of every task. out: optional four float64 arrays of at
        least the batch's output size (e.g. from pinned_empty), written in place and returned."""
        if radial_mode == 1:
            self.ensure_level_model()
        n = int(batch.block_offsets()[-1])
        if out is None:
            outs = [np.empty(max(n, 1)) for _ in range(4)]  # the call writes every element
        else:
            outs = list(out)
            if len(outs) != 4 or any(x.dtype != np.float64 or not x.flags.c_contiguous or x.size < n for x in outs):
                raise ValueError("out must be four C-contiguous float64 arrays of at least the batch's output size")
        rc = self.lib.libgrpp_b200_full_grpp_batch(ct.byref(batch.struct), radial_mode, *[_dp(x) for x in outs])
        if rc != 0:
            raise RuntimeError(f"libgrpp_b200_full_grpp_batch failed ({rc}): {self.last_error_message()}")
        return [x[:n] for x in outs]

    def pinned_empty(self, n: int) -> np.ndarray:
        """A float64 array of n elements in page-locked host memory (freed with the array)."""
        nbytes = max(int(n), 1) * 8
        p = self.lib.libgrpp_b200_host_alloc(nbytes)
        if not p:
            raise MemoryError(f"libgrpp_b200_host_alloc({nbytes}) failed: {self.last_error_message()}")
        buf = (ct.c_double * max(int(n), 1)).from_address(p)
        arr = np.frombuffer(buf, dtype=np.float64, count=max(int(n), 1))
        weakref.finalize(arr, self.lib.libgrpp_b200_host_free, ct.c_void_p(p))
        return arr[:int(n)] if n > 0 else arr

    def type2_batch_noalloc(self, batch):
        """AREP type 2 blocks of every task through the allocation-free entry point."""
        n = int(batch.block_offsets()[-1])
        out = np.zeros(max(n, 1))
        rc = self.lib.libgrpp_b200_type2_batch_noalloc(ct.byref(batch.struct), _dp(out))
        if rc != 0:
            raise RuntimeError(f"libgrpp_b200_type2_batch_noalloc failed ({rc}): {self.last_error_message()}")
        return out[:n]

    def set_device(self, device: int):
        rc = self.lib.libgrpp_b200_set_device(int(device))
        if rc != 0:
            raise RuntimeError(f"libgrpp_b200_set_device({device}) failed: {self.last_error_message()}")

    def fp64_peak(self) -> float:
        v = ct.c_double(0.0)
        rc = self.lib.libgrpp_b200_fp64_peak(ct.byref(v))
        if rc != 0:
            raise RuntimeError(self.last_error_message())
        return v.value

    def grad_contract(self, system, batch, D, radial_mode=0, symmetric=False):
        """d tr(D V^m) / d R for the four matrices m over the batch's tasks: [4, n_atoms, 3]
        (libgrpp_b200_grpp_gradient_contract; same quantity as the oracle's driver_grad_contract).
        symmetric: libgrpp_b200_grpp_gradient_contract_symmetric (D symmetric: shell pairs folded,
        spin-orbit parts zero)."""
        if radial_mode == 1:
            self.ensure_level_model()
        nat = len(system.atoms)
        g = np.zeros((4, nat, 3))
        sa = np.ascontiguousarray(system.shell_atom, dtype=np.int32)
        ca = np.ascontiguousarray(system.centre_atom, dtype=np.int32)
        xyz = np.ascontiguousarray(system.atoms, dtype=np.float64)
        bo = np.ascontiguousarray(system.basis_offsets()[:-1], dtype=np.int32)
        Dm = np.ascontiguousarray(D, dtype=np.float64)
        f = self.lib.libgrpp_b200_grpp_gradient_contract_symmetric if symmetric else self.lib.libgrpp_b200_grpp_gradient_contract
        rc = f(ct.byref(batch.struct), radial_mode, _ip(sa), _ip(ca), _dp(xyz), nat, _ip(bo), int(Dm.shape[0]), _dp(Dm),
               _dp(g))
        self._check(rc, "libgrpp_b200_grpp_gradient_contract")
        return g

    # ------------------------------------------------------------ learned grid-level model
    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed ({rc}): {self.last_error_message()}")

    def set_level_model(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32)
        self._check(self.lib.libgrpp_b200_set_level_model(p.ctypes.data_as(ct.POINTER(ct.c_float))),
                    "libgrpp_b200_set_level_model")
        self._lm_set = True

    def level_samples(self, batch):
        """(features [n, 12] float32, stop level [n] int8, -1 if not walked) of every radial task."""
        nt = max(len(batch.task_a), 1)
        X = np.zeros((nt, 12), dtype=np.float32)
        y = np.zeros(nt, dtype=np.int8)
        n = ct.c_int64(0)
        self._check(self.lib.libgrpp_b200_level_samples(ct.byref(batch.struct), X.ctypes.data_as(ct.POINTER(ct.c_float)),
                                                        y.ctypes.data_as(ct.POINTER(ct.c_int8)), ct.byref(n)),
                    "libgrpp_b200_level_samples")
        return X[: n.value], y[: n.value]

    def mlp_grad(self, params, X, y):
        p = np.ascontiguousarray(params, dtype=np.float32)
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.int8)
        g = np.zeros_like(p)
        loss = ct.c_float(0.0)
        F = ct.POINTER(ct.c_float)
        self._check(self.lib.libgrpp_b200_mlp_grad(p.ctypes.data_as(F), X.ctypes.data_as(F),
                                                   y.ctypes.data_as(ct.POINTER(ct.c_int8)), len(y), g.ctypes.data_as(F),
                                                   ct.byref(loss)), "libgrpp_b200_mlp_grad")
        return g, float(loss.value)

    def mlp_train(self, params, X, y, epochs=4, batch=2048, lr=2e-3, seed=0):
        p = np.array(params, dtype=np.float32, copy=True)
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.int8)
        losses = np.zeros(epochs, dtype=np.float32)
        F = ct.POINTER(ct.c_float)
        self._check(self.lib.libgrpp_b200_mlp_train(X.ctypes.data_as(F), y.ctypes.data_as(ct.POINTER(ct.c_int8)), len(y),
                                                    epochs, batch, lr, seed, p.ctypes.data_as(F), losses.ctypes.data_as(F)),
                    "libgrpp_b200_mlp_train")
        return p, losses

    def mlp_predict(self, params, X):
        p = np.ascontiguousarray(params, dtype=np.float32)
        X = np.ascontiguousarray(X, dtype=np.float32)
        out = np.zeros(len(X), dtype=np.int8)
        F = ct.POINTER(ct.c_float)
        self._check(self.lib.libgrpp_b200_mlp_predict(p.ctypes.data_as(F), X.ctypes.data_as(F), len(X),
                                                      out.ctypes.data_as(ct.POINTER(ct.c_int8))),
                    "libgrpp_b200_mlp_predict")
        return out

    def ensure_level_model(self):
        """Install the committed level model (libgrpp_b200/level_model.bin) once, for the
        learned radial mode; callers that set their own model first are left alone."""
        if getattr(self, "_lm_set", False) or not self.has("libgrpp_b200_set_level_model"):
            return
        from . import level_model
        if os.path.exists(level_model.MODEL_FILE):
            self.set_level_model(level_model.load()[0])

    def plan(self, batch, radial_mode=0, assembly_threads=0) -> "Plan":
        """A prepared batch; assembly_threads fixes the assembly kernel's block size for every
        task (128, 256, 512), 0 takes the autotuner's per-class table or the default rule."""
        if radial_mode == 1:
            self.ensure_level_model()
        return Plan(self, batch, radial_mode, assembly_threads)

    def autotune_assembly(self, batch, radial_mode=0):
        """Time every assembly class of the batch with 128, 256 and 512 threads per block and keep
        the fastest per class for this device; returns {class key: (tasks, ms128, ms256, ms512, choice)}."""
        if radial_mode == 1:
            self.ensure_level_model()
        cap = 4096
        rows = np.zeros(6 * cap)
        n = self.lib.libgrpp_b200_autotune_assembly(ct.byref(batch.struct), radial_mode, _dp(rows), cap)
        self._check(min(n, 0), "libgrpp_b200_autotune_assembly")
        r = rows[: 6 * min(n, cap)].reshape(-1, 6)
        return {int(x[0]): (int(x[1]), float(x[2]), float(x[3]), float(x[4]), int(x[5])) for x in r}

    def autotune_reset(self):
        self.lib.libgrpp_b200_autotune_reset()

    def last_error(self) -> int:
        return int(self.lib.libgrpp_b200_last_error())

    def last_error_message(self) -> str:
        m = self.lib.libgrpp_b200_last_error_message()
        return m.decode() if m else ""


def shells_handles(lib: LibGRPP, system):
    return [lib.new_shell(s) for s in system.shells]


def dense_full(lib: LibGRPP, system, threads=None):
    """Dense (arep, so_x, so_y, so_z) matrices of a system through the single-task
    API, serially in the C driver's order (test_libgrpp_c/eval_integrals.c:78-123)."""
    lib.set_cartesian_order(system.cart_order)
    hs = shells_handles(lib, system)
    hg = [lib.new_grpp(g) for g in system.grpps]
    off = system.basis_offsets()
    n = int(off[-1])
    M = np.zeros((4, n, n))
    for i, si in enumerate(system.shells):
        for j, sj in enumerate(system.shells):
            for C, gi in system.centres:
                blocks = lib.full(hs[i], hs[j], hg[gi], C, ncart(si.L), ncart(sj.L))
                for m in range(4):
                    M[m, off[i]:off[i + 1], off[j]:off[j + 1]] += blocks[m]
    return M


class Plan:
    """A batch prepared on the device (libgrpp_b200_plan_*): execute() runs the kernels only."""

    def __init__(self, lib: LibGRPP, batch, radial_mode=0, assembly_threads=0):
        self.lib = lib
        self.batch = batch
        self.n_out = int(batch.block_offsets()[-1])
        self.h = lib.lib.libgrpp_b200_plan_create_ex(ct.byref(batch.struct), radial_mode, assembly_threads)
        if not self.h:
            raise RuntimeError(f"libgrpp_b200_plan_create failed: {lib.last_error_message()}")

    def execute(self):
        rc = self.lib.lib.libgrpp_b200_plan_execute(self.h)
        if rc != 0:
            raise RuntimeError(f"libgrpp_b200_plan_execute failed ({rc}): {self.lib.last_error_message()}")

    def outputs(self):
        outs = [np.zeros(max(self.n_out, 1)) for _ in range(4)]
        rc = self.lib.lib.libgrpp_b200_plan_outputs(self.h, *[_dp(x) for x in outs])
        if rc != 0:
            raise RuntimeError(self.lib.last_error_message())
        return [x[: self.n_out] for x in outs]

    def stats(self):
        ms = np.zeros(5)
        cnt = np.zeros(5, dtype=np.int64)
        self.lib.lib.libgrpp_b200_plan_stats(self.h, _dp(ms), cnt.ctypes.data_as(ct.POINTER(ct.c_int64)))
        return {"ms_total": ms[0], "ms_type1": ms[1], "ms_radial": ms[2], "ms_assembly": ms[3], "ms_screen": ms[4],
                "n_tasks": int(cnt[0]), "n_radial": int(cnt[1]), "n_type1_items": int(cnt[2]),
                "n_entries": int(cnt[3]), "h2d_bytes": int(cnt[4])}

    def set_counting(self, on: bool):
        self.lib.lib.libgrpp_b200_plan_set_counting(self.h, 1 if on else 0)

    def learned_stats(self):
        ms = ct.c_double(0.0)
        fb = ct.c_int64(0)
        self.lib.lib.libgrpp_b200_plan_learned_stats(self.h, ct.byref(ms), ct.byref(fb))
        return {"ms_predict": ms.value, "fallbacks": int(fb.value)}

    COUNTERS = ("screen_cycles", "quad_cycles", "items", "points", "bessel", "prim_pts", "term_pts", "pow_pts",
                "accum", "scr_combos", "scr_iters", "scr_final", "levels", "mmd_triples", "mmd_flops")

    def counters(self):
        c = np.zeros(len(self.COUNTERS), dtype=np.uint64)
        self.lib.lib.libgrpp_b200_plan_counters(self.h, c.ctypes.data_as(ct.POINTER(ct.c_uint64)), len(c))
        return {k: int(v) for k, v in zip(self.COUNTERS, c)}

    def close(self):
        if self.h:
            self.lib.lib.libgrpp_b200_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
