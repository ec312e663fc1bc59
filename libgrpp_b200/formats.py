"""Readers for the plain-text inputs libgrpp's C test driver uses, and its
lower-triangle matrix format.

* ``molecule.xyz``: atom count, then ``symbol x y z`` lines (coordinates used
  as given, bohr) — test_libgrpp_c/molecule.c:47-99.
* ``basis.inp``: ``* Z n_blocks`` entries; block ``l`` is ``n_prim n_contr``
  followed by rows ``exponent c_1 .. c_n_contr``; each contracted function is
  normalised to unit self-overlap of its x^l component times (2l-1)!!
  — test_libgrpp_c/basis.c:88-160, libgrpp/fortran.c:689-702.
* ``ecp.inp``: ``* Z n_oc_blocks n_arep`` entries with outercore shells then
  ``n_arep`` potential blocks of rows ``n zeta c_arep c_so c_oc...``; the last
  block is the local part U_L, spin-orbit terms exist for l >= 1, outercore
  potential ``ioc`` has J = |2l -+ 1| — test_libgrpp_c/rpp.c:17-148.
* matrices: first line the dimension, then ``i j value`` (1-based) for the lower
  triangle entries with |value| > 1e-14 — test_libgrpp_c/print_matrix.c:31-48.
"""
from __future__ import annotations

import math
import re

import numpy as np

from .system import GRPP, Potential, Shell, System, CART_ORDER_TURBOMOLE

_SYMBOLS = (
    "H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co Ni Cu Zn Ga Ge As Se Br Kr "
    "Rb Sr Y Zr Nb Mo Tc Ru Rh Pd Ag Cd In Sn Sb Te I Xe Cs Ba La Ce Pr Nd Pm Sm Eu Gd Tb Dy Ho Er Tm Yb "
    "Lu Hf Ta W Re Os Ir Pt Au Hg Tl Pb Bi Po At Rn Fr Ra Ac Th Pa U Np Pu Am Cm Bk Cf Es Fm Md No Lr Rf "
    "Db Sg Bh Hs Mt Ds Rg Cn Nh Fl Mc Lv Ts Og"
).split()
ELEMENT_Z = {s.lower(): i + 1 for i, s in enumerate(_SYMBOLS)}


def _tokens(text: str):
    return text.split()


def read_molecule(path):
    with open(path) as f:
        tok = _tokens(f.read())
    n = int(tok[0])
    Z, xyz = [], []
    for i in range(n):
        sym, x, y, z = tok[1 + 4 * i: 5 + 4 * i]
        Z.append(ELEMENT_Z[sym.lower()])
        xyz.append((float(x), float(y), float(z)))
    return np.array(Z, dtype=np.int32), np.array(xyz, dtype=np.float64)


def _dfact(n: int) -> float:
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return float(r)


def _os_same_centre(L: int, p: float) -> float:
    """1D Obara-Saika overlap S[L][L] of two primitives on one centre, with the
    operation order of libgrpp/overlap.c:92-120 (X_PA = X_PB = 0)."""
    pf = 1.0 / (2.0 * p)
    S = [[0.0] * (L + 1) for _ in range(L + 1)]
    for i in range(L + 1):
        for j in range(L + 1):
            if i + j == 0:
                S[0][0] = math.sqrt(math.pi / p) * math.exp(-0.0)
                continue
            s = 0.0
            if i == 0:
                s += 0.0 * S[i][j - 1]
                if j - 1 > 0:
                    s += float(j - 1) * pf * S[i][j - 2]
            else:
                s += 0.0 * S[i - 1][j]
                if i - 1 > 0:
                    s += float(i - 1) * pf * S[i - 2][j]
                if j > 0:
                    s += float(j) * pf * S[i - 1][j - 1]
            S[i][j] = s
    return S[L][L]


def contracted_norm(L: int, coeffs: np.ndarray, alpha: np.ndarray) -> float:
    """sqrt((2L-1)!!) / sqrt(<x^L g | x^L g>) for the contracted radial function
    with libgrpp's primitive normalisation (2a/pi)^(3/4) (4a)^(L/2).

    The self-overlap is accumulated in the same floating-point order as the C
    driver's normalisation (libgrpp/fortran.c:641-702 through
    libgrpp_overlap_integrals, libgrpp/overlap.c:39-139): the reference's
    adaptive quadrature is sensitive to last-bit changes of the coefficients.
    """
    S = 0.0
    for ci, ai in zip(coeffs.tolist(), alpha.tolist()):
        for cj, aj in zip(coeffs.tolist(), alpha.tolist()):
            p = ai + aj
            NA = math.pow(2 * ai / math.pi, 0.75) * math.pow(4 * ai, 0.5 * L)
            NB = math.pow(2 * aj / math.pi, 0.75) * math.pow(4 * aj, 0.5 * L)
            s0 = math.sqrt(math.pi / p) * math.exp(-0.0)
            buf = NA * NB * _os_same_centre(L, p) * s0 * s0
            S += (ci * cj) * buf
    return math.sqrt(_dfact(2 * L - 1)) / math.sqrt(S)


class _Lines:
    def __init__(self, path):
        with open(path) as f:
            self.text = f.read()

    def entry(self, header_len: int, z: int):
        """Token stream positioned after the '* Z ...' header for element z (None if absent)."""
        for m in re.finditer(r"^\s*\*", self.text, flags=re.M):
            rest = self.text[m.end():]
            head = rest.split(None, header_len)
            if int(head[0]) == z:
                return rest
        return None


def read_basis(path, z: int):
    """List of (L, coeffs, alpha) contracted functions for element z."""
    text = _Lines(path).entry(2, z)
    if text is None:
        raise KeyError(f"no basis for Z={z} in {path}")
    lines = text.splitlines()
    head = lines[0].split()
    n_blocks = int(head[1])
    pos = 1
    out = []
    for L in range(n_blocks):
        while not lines[pos].split():
            pos += 1
        nprim, ncontr = map(int, lines[pos].split()[:2])
        pos += 1
        rows = []
        while len(rows) < nprim:
            t = lines[pos].split()
            pos += 1
            if t:
                rows.append([float(v.replace("D", "E")) for v in t[: 1 + ncontr]])
        rows = np.array(rows)
        for k in range(ncontr):
            c = rows[:, 1 + k].copy()
            a = rows[:, 0].copy()
            c = c * contracted_norm(L, c, a)
            out.append((L, c, a))
    return out


def read_grpp(path, z: int):
    """GRPP operator of element z, or None (test_libgrpp_c/rpp.c:17-148)."""
    text = _Lines(path).entry(3, z)
    if text is None:
        return None
    lines = text.splitlines()
    head = lines[0].split()
    n_blocks, n_arep = int(head[1]), int(head[2])
    pos = 1
    oc_shells = []
    for L in range(n_blocks):
        while not lines[pos].split():
            pos += 1
        n_alpha, n_contr = map(int, lines[pos].split()[:2])
        pos += 1
        vals = []
        while len(vals) < n_alpha * (1 + n_contr):
            vals.extend(float(v.replace("D", "E")) for v in lines[pos].split())
            pos += 1
        rows = np.array(vals[: n_alpha * (1 + n_contr)]).reshape(n_alpha, 1 + n_contr)
        for k in range(n_contr):
            oc_shells.append(Shell(np.zeros(3), L, rows[:, 1 + k].copy(), rows[:, 0].copy()))
    g = GRPP()
    oc_pots = []
    for L in range(n_arep):
        while not lines[pos].split():
            pos += 1
        n_prim, n_oc = map(int, lines[pos].split()[:2])
        pos += 1
        rows = []
        while len(rows) < n_prim:
            t = lines[pos].split()
            pos += 1
            if t:
                rows.append([float(v.replace("D", "E")) for v in t[: 4 + n_oc]])
        rows = np.array(rows)
        pw = rows[:, 0].astype(np.int32)
        ex = rows[:, 1]
        arep = _potential(L, 0, pw, rows[:, 2], ex)
        if L == n_arep - 1:
            g.UL = arep
        else:
            g.arep.append(arep)
        if L > 0:
            g.so.append(_potential(L, 0, pw, rows[:, 3], ex))
        for ioc in range(n_oc):
            J = abs(2 * L + (-1 if ioc % 2 == 0 else 1))
            oc_pots.append(_potential(L, J, pw, rows[:, 4 + ioc], ex))
    g.oc = list(zip(oc_pots, oc_shells))
    return g


def _potential(L, J, powers, coeffs, alpha):
    """libgrpp_new_potential drops terms with |c| < 1e-14 (libgrpp/potential.c:31-42)."""
    keep = np.abs(coeffs) >= 1e-14
    return Potential(L, J, powers[keep], coeffs[keep], alpha[keep])


def read_system(directory, cart_order=CART_ORDER_TURBOMOLE) -> System:
    """The molecule, basis and GRPPs of one of libgrpp's test directories, with
    shells and centres in the C driver's order (test_libgrpp_c/main.c:196-254)."""
    import os

    Z, xyz = read_molecule(os.path.join(directory, "molecule.xyz"))
    basis_cache, grpp_cache = {}, {}
    shells, shell_atom = [], []
    for i, z in enumerate(Z):
        if z not in basis_cache:
            basis_cache[z] = read_basis(os.path.join(directory, "basis.inp"), int(z))
        for L, c, a in basis_cache[z]:
            shells.append(Shell(xyz[i], L, c, a))
            shell_atom.append(i)
    grpps, centres, centre_atom, gidx = [], [], [], {}
    for i, z in enumerate(Z):
        if z not in grpp_cache:
            grpp_cache[z] = read_grpp(os.path.join(directory, "ecp.inp"), int(z))
        if grpp_cache[z] is None:
            continue
        if z not in gidx:
            gidx[z] = len(grpps)
            grpps.append(grpp_cache[z])
        centres.append((xyz[i].copy(), gidx[z]))
        centre_atom.append(i)
    return System(shells, grpps, centres, cart_order, np.array(shell_atom, dtype=np.int32),
                  np.array(centre_atom, dtype=np.int32), xyz)


def read_lower_triangle(path) -> np.ndarray:
    with open(path) as f:
        tok = f.read().split()
    n = int(tok[0])
    M = np.zeros((n, n))
    vals = np.array(tok[1:], dtype=object).reshape(-1, 3)
    i = vals[:, 0].astype(int) - 1
    j = vals[:, 1].astype(int) - 1
    M[i, j] = vals[:, 2].astype(float)
    return M


def write_lower_triangle(path, M: np.ndarray):
    n = M.shape[0]
    with open(path, "w") as f:
        f.write(f"{n:6d}\n")
        for i in range(n):
            for j in range(i + 1):
                if abs(M[i, j]) > 1e-14:
                    f.write(f"{i + 1:6d}{j + 1:6d}{M[i, j]:30.16E}\n")
