"""Host-side description of a GRPP integral workload.

The objects mirror libgrpp's containers (libgrpp/libgrpp.h:42-103): a shell is
an atom-centred contracted Cartesian Gaussian shell, a potential is a sum of
c_k r^(n_k-2) exp(-zeta_k r^2) terms, a GRPP is the local part U_L plus
semilocal averaged (AREP), spin-orbit (SO) and outercore (OC) parts.

A :class:`System` holds basis shells, GRPP operators, potential centres and a
task list of (shell A, shell B, centre C). :meth:`System.batch` flattens it into
the ``libgrpp_b200_batch_t`` arrays of ``include/libgrpp_b200.h``.
"""
from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass, field

import numpy as np

CART_ORDER_DIRAC = 0
CART_ORDER_TURBOMOLE = 1


def ncart(L: int) -> int:
    return (L + 1) * (L + 2) // 2


def cartesian_list(L: int, order: int) -> np.ndarray:
    """Cartesian components (x, y, z powers) of angular momentum L in libgrpp's
    DIRAC or TURBOMOLE order (libgrpp/parameters.c:94-134)."""
    out = []
    if order == CART_ORDER_DIRAC:
        for r in range(L, -1, -1):
            for s in range(L, -1, -1):
                for t in range(L, -1, -1):
                    if r + s + t == L:
                        out.append((r, s, t))
    elif order == CART_ORDER_TURBOMOLE:
        for r in range(L, -1, -1):
            for s in range(L - r, -1, -1):
                out.append((r, s, L - r - s))
    else:
        raise ValueError(f"unknown Cartesian order {order}")
    return np.asarray(out, dtype=np.int32).reshape(-1, 3)


@dataclass
class Shell:
    origin: np.ndarray
    L: int
    coeffs: np.ndarray
    alpha: np.ndarray

    def __post_init__(self):
        self.origin = np.asarray(self.origin, dtype=np.float64).reshape(3)
        self.coeffs = np.asarray(self.coeffs, dtype=np.float64).ravel()
        self.alpha = np.asarray(self.alpha, dtype=np.float64).ravel()
        if self.coeffs.shape != self.alpha.shape:
            raise ValueError("coeffs and alpha differ in length")


@dataclass
class Potential:
    L: int
    J: int
    powers: np.ndarray
    coeffs: np.ndarray
    alpha: np.ndarray

    def __post_init__(self):
        self.powers = np.asarray(self.powers, dtype=np.int32).ravel()
        self.coeffs = np.asarray(self.coeffs, dtype=np.float64).ravel()
        self.alpha = np.asarray(self.alpha, dtype=np.float64).ravel()


@dataclass
class GRPP:
    UL: Potential | None = None
    arep: list = field(default_factory=list)       # list[Potential]
    so: list = field(default_factory=list)         # list[Potential]
    oc: list = field(default_factory=list)         # list[tuple[Potential, Shell]]


class BatchArrays:
    """Flat numpy arrays + the ctypes ``libgrpp_b200_batch_t`` that points at them."""

    def __init__(self, **arrays):
        self.__dict__.update(arrays)
        self._struct = None

    @property
    def struct(self) -> "BatchStruct":
        if self._struct is None:
            s = BatchStruct()

            def ip(a):
                return a.ctypes.data_as(ct.POINTER(ct.c_int))

            def dp(a):
                return a.ctypes.data_as(ct.POINTER(ct.c_double))

            s.n_shells = len(self.shell_L)
            s.shell_L, s.shell_nprim, s.shell_prim_off = ip(self.shell_L), ip(self.shell_nprim), ip(self.shell_prim_off)
            s.prim_coef, s.prim_alpha, s.shell_origin = dp(self.prim_coef), dp(self.prim_alpha), dp(self.shell_origin)
            s.shell_cart_off, s.cart_list = ip(self.shell_cart_off), ip(self.cart_list)
            s.n_pots = len(self.pot_L)
            s.pot_L, s.pot_J, s.pot_nprim, s.pot_prim_off = ip(self.pot_L), ip(self.pot_J), ip(self.pot_nprim), ip(self.pot_prim_off)
            s.pot_powers, s.pot_coef, s.pot_alpha = ip(self.pot_powers), dp(self.pot_coef), dp(self.pot_alpha)
            s.n_grpps = len(self.grpp_UL)
            s.grpp_UL = ip(self.grpp_UL)
            s.grpp_arep_off, s.grpp_n_arep = ip(self.grpp_arep_off), ip(self.grpp_n_arep)
            s.grpp_so_off, s.grpp_n_so = ip(self.grpp_so_off), ip(self.grpp_n_so)
            s.grpp_oc_off, s.grpp_n_oc = ip(self.grpp_oc_off), ip(self.grpp_n_oc)
            s.grpp_pot_list, s.grpp_oc_pot, s.grpp_oc_shell = ip(self.grpp_pot_list), ip(self.grpp_oc_pot), ip(self.grpp_oc_shell)
            s.n_centres = len(self.centre_grpp)
            s.centre_origin, s.centre_grpp = dp(self.centre_origin), ip(self.centre_grpp)
            s.n_tasks = len(self.task_a)
            s.task_a, s.task_b, s.task_c = ip(self.task_a), ip(self.task_b), ip(self.task_c)
            self._struct = s
        return self._struct

    def block_sizes(self) -> np.ndarray:
        nc = (self.shell_L + 1) * (self.shell_L + 2) // 2
        return nc[self.task_a].astype(np.int64) * nc[self.task_b].astype(np.int64)

    def block_offsets(self) -> np.ndarray:
        sz = self.block_sizes()
        off = np.zeros(len(sz) + 1, dtype=np.int64)
        np.cumsum(sz, out=off[1:])
        return off

    def with_tasks(self, a, b, c) -> "BatchArrays":
        d = {k: v for k, v in self.__dict__.items() if not k.startswith("_")}
        d["task_a"] = np.ascontiguousarray(a, dtype=np.int32)
        d["task_b"] = np.ascontiguousarray(b, dtype=np.int32)
        d["task_c"] = np.ascontiguousarray(c, dtype=np.int32)
        return BatchArrays(**d)


class BatchStruct(ct.Structure):
    _fields_ = [
        ("n_shells", ct.c_int),
        ("shell_L", ct.POINTER(ct.c_int)), ("shell_nprim", ct.POINTER(ct.c_int)),
        ("shell_prim_off", ct.POINTER(ct.c_int)),
        ("prim_coef", ct.POINTER(ct.c_double)), ("prim_alpha", ct.POINTER(ct.c_double)),
        ("shell_origin", ct.POINTER(ct.c_double)),
        ("shell_cart_off", ct.POINTER(ct.c_int)), ("cart_list", ct.POINTER(ct.c_int)),
        ("n_pots", ct.c_int),
        ("pot_L", ct.POINTER(ct.c_int)), ("pot_J", ct.POINTER(ct.c_int)),
        ("pot_nprim", ct.POINTER(ct.c_int)), ("pot_prim_off", ct.POINTER(ct.c_int)),
        ("pot_powers", ct.POINTER(ct.c_int)),
        ("pot_coef", ct.POINTER(ct.c_double)), ("pot_alpha", ct.POINTER(ct.c_double)),
        ("n_grpps", ct.c_int),
        ("grpp_UL", ct.POINTER(ct.c_int)),
        ("grpp_arep_off", ct.POINTER(ct.c_int)), ("grpp_n_arep", ct.POINTER(ct.c_int)),
        ("grpp_so_off", ct.POINTER(ct.c_int)), ("grpp_n_so", ct.POINTER(ct.c_int)),
        ("grpp_oc_off", ct.POINTER(ct.c_int)), ("grpp_n_oc", ct.POINTER(ct.c_int)),
        ("grpp_pot_list", ct.POINTER(ct.c_int)), ("grpp_oc_pot", ct.POINTER(ct.c_int)),
        ("grpp_oc_shell", ct.POINTER(ct.c_int)),
        ("n_centres", ct.c_int),
        ("centre_origin", ct.POINTER(ct.c_double)), ("centre_grpp", ct.POINTER(ct.c_int)),
        ("n_tasks", ct.c_int64),
        ("task_a", ct.POINTER(ct.c_int)), ("task_b", ct.POINTER(ct.c_int)), ("task_c", ct.POINTER(ct.c_int)),
    ]


@dataclass
class System:
    """Basis shells, GRPPs, potential centres and the (A, B, C) task list."""

    shells: list                   # list[Shell]
    grpps: list                    # list[GRPP]
    centres: list                  # list[tuple[origin(3,), grpp index]]
    cart_order: int = CART_ORDER_TURBOMOLE
    shell_atom: np.ndarray | None = None   # atom index of every basis shell
    centre_atom: np.ndarray | None = None  # atom index of every centre
    atoms: np.ndarray | None = None        # (n_atoms, 3) coordinates

    def basis_offsets(self) -> np.ndarray:
        off = np.zeros(len(self.shells) + 1, dtype=np.int64)
        np.cumsum([ncart(s.L) for s in self.shells], out=off[1:])
        return off

    def n_basis(self) -> int:
        return int(self.basis_offsets()[-1])

    def all_tasks(self):
        """All ordered shell pairs x all centres, in the reference driver's order
        (test_libgrpp_c/eval_integrals.c:64-83, 102-123)."""
        ns, nc = len(self.shells), len(self.centres)
        a, b, c = np.meshgrid(np.arange(ns), np.arange(ns), np.arange(nc), indexing="ij")
        return a.ravel().astype(np.int32), b.ravel().astype(np.int32), c.ravel().astype(np.int32)

    def batch(self, task_a=None, task_b=None, task_c=None) -> BatchArrays:
        if task_a is None:
            task_a, task_b, task_c = self.all_tasks()
        shells = list(self.shells)
        pots: list[Potential] = []
        grpp_UL, arep_off, n_arep, so_off, n_so, oc_off, n_oc = [], [], [], [], [], [], []
        pot_list, oc_pot, oc_shell = [], [], []

        def add_pot(p):
            pots.append(p)
            return len(pots) - 1

        for g in self.grpps:
            grpp_UL.append(add_pot(g.UL) if g.UL is not None else -1)
            arep_off.append(len(pot_list))
            n_arep.append(len(g.arep))
            for p in g.arep:
                pot_list.append(add_pot(p))
            so_off.append(len(pot_list))
            n_so.append(len(g.so))
            for p in g.so:
                pot_list.append(add_pot(p))
            oc_off.append(len(oc_pot))
            n_oc.append(len(g.oc))
            for p, s in g.oc:
                oc_pot.append(add_pot(p))
                shells.append(s)
                oc_shell.append(len(shells) - 1)

        shell_L = np.array([s.L for s in shells], dtype=np.int32)
        nprim = np.array([len(s.alpha) for s in shells], dtype=np.int32)
        poff = np.zeros(len(shells), dtype=np.int32)
        if len(shells) > 1:
            poff[1:] = np.cumsum(nprim)[:-1]
        cart_tabs = {}
        cart_off = np.zeros(len(shells), dtype=np.int32)
        cart_rows = []
        for L in sorted(set(shell_L.tolist())):
            cart_tabs[L] = sum(len(r) for r in cart_rows)
            cart_rows.append(cartesian_list(L, self.cart_order))
        for i, L in enumerate(shell_L):
            cart_off[i] = cart_tabs[int(L)]
        pnp = np.array([len(p.alpha) for p in pots], dtype=np.int32)
        ppoff = np.zeros(len(pots), dtype=np.int32)
        if len(pots) > 1:
            ppoff[1:] = np.cumsum(pnp)[:-1]

        def cat(xs, dt):
            return np.ascontiguousarray(np.concatenate(xs) if xs else np.zeros(1), dtype=dt)

        def arr(x, dt=np.int32):
            return np.ascontiguousarray(np.array(x if len(x) else [0], dtype=dt))

        return BatchArrays(
            shell_L=shell_L, shell_nprim=nprim, shell_prim_off=poff,
            prim_coef=cat([s.coeffs for s in shells], np.float64),
            prim_alpha=cat([s.alpha for s in shells], np.float64),
            shell_origin=np.ascontiguousarray(np.stack([s.origin for s in shells]).ravel()),
            shell_cart_off=cart_off, cart_list=np.ascontiguousarray(np.concatenate(cart_rows).ravel(), dtype=np.int32),
            pot_L=arr([p.L for p in pots]), pot_J=arr([p.J for p in pots]),
            pot_nprim=arr(pnp.tolist()), pot_prim_off=arr(ppoff.tolist()),
            pot_powers=cat([p.powers for p in pots], np.int32),
            pot_coef=cat([p.coeffs for p in pots], np.float64),
            pot_alpha=cat([p.alpha for p in pots], np.float64),
            grpp_UL=arr(grpp_UL), grpp_arep_off=arr(arep_off), grpp_n_arep=arr(n_arep),
            grpp_so_off=arr(so_off), grpp_n_so=arr(n_so), grpp_oc_off=arr(oc_off), grpp_n_oc=arr(n_oc),
            grpp_pot_list=arr(pot_list), grpp_oc_pot=arr(oc_pot), grpp_oc_shell=arr(oc_shell),
            centre_origin=np.ascontiguousarray(np.array([c[0] for c in self.centres], dtype=np.float64).ravel()),
            centre_grpp=arr([c[1] for c in self.centres]),
            task_a=np.ascontiguousarray(task_a, dtype=np.int32),
            task_b=np.ascontiguousarray(task_b, dtype=np.int32),
            task_c=np.ascontiguousarray(task_c, dtype=np.int32),
        )

    def assemble(self, batch: BatchArrays, blocks: np.ndarray) -> np.ndarray:
        """Sum per-task blocks into the dense n_basis x n_basis matrix, in task order."""
        off = self.basis_offsets()
        n = int(off[-1])
        M = np.zeros((n, n))
        boff = batch.block_offsets()
        nc = (batch.shell_L + 1) * (batch.shell_L + 2) // 2
        for t in range(len(batch.task_a)):
            a, b = int(batch.task_a[t]), int(batch.task_b[t])
            na, nb = int(nc[a]), int(nc[b])
            M[off[a]:off[a] + na, off[b]:off[b] + nb] += blocks[boff[t]:boff[t + 1]].reshape(na, nb)
        return M
