"""Seeded synthetic GRPP workloads.

libgrpp publishes no benchmark suite; these generators produce the five
workloads the engine is measured on, with numpy's PCG64 (``default_rng``).
Every draw happens in the order written below, so a seed fixes the workload.

Potential terms c r^(n-2) exp(-zeta r^2): n uniform in {0,1,2}, zeta
log-uniform in [0.05, 50], c uniform in [-20, 20] (spin-orbit terms: c in
[-5, 5]). Contraction coefficients are uniform in [-1, 1] and are passed to
the shell constructor unchanged.
"""
from __future__ import annotations

import numpy as np

from .system import GRPP, Potential, Shell, System, CART_ORDER_TURBOMOLE


def _terms(rng, L, J, n, cmax=20.0):
    powers = rng.integers(0, 3, n).astype(np.int32)
    zeta = np.exp(rng.uniform(np.log(0.05), np.log(50.0), n))
    c = rng.uniform(-cmax, cmax, n)
    return Potential(L, J, powers, c, zeta)


def _scalar_grpp(rng, n_local, l_proj):
    g = GRPP()
    g.UL = _terms(rng, l_proj + 1, 0, n_local)
    for l in range(l_proj + 1):
        g.arep.append(_terms(rng, l, 0, 3))
    return g


def _place(rng, n, box, dmin, max_tries=100000):
    pts = []
    tries = 0
    while len(pts) < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place atoms")
        p = rng.uniform(0.0, box, 3)
        if all(np.linalg.norm(p - q) >= dmin for q in pts):
            pts.append(p)
    return np.array(pts)


def _shell(rng, origin, L, nprim, alpha=None, amin=0.02, amax=5e3):
    if alpha is None:
        alpha = np.exp(rng.uniform(np.log(amin), np.log(amax), nprim))
    c = rng.uniform(-1.0, 1.0, nprim)
    return Shell(origin, L, c, alpha)


def config0(seed: int = 0) -> System:
    """Two atoms, A=(0,0,0) with U_L (4 terms) + projectors l=0..3 (3 terms),
    B=(0,0,2); both carry s,p,d,f shells of 6 even-tempered primitives
    0.03*3^k. One centre (A); 8x8 ordered shell pairs = 64 tasks, 40x40 matrix."""
    rng = np.random.default_rng(seed)
    g = _scalar_grpp(rng, 4, 3)
    A, B = np.zeros(3), np.array([0.0, 0.0, 2.0])
    alpha = 0.03 * 3.0 ** np.arange(6)
    shells, shell_atom = [], []
    for ia, o in enumerate((A, B)):
        for L in range(4):
            shells.append(_shell(rng, o, L, 6, alpha=alpha))
            shell_atom.append(ia)
    return System(shells, [g], [(A.copy(), 0)], CART_ORDER_TURBOMOLE, np.array(shell_atom, np.int32),
                  np.array([0], np.int32), np.stack([A, B]))


def config1(seed: int = 1, n_atoms: int = 64, amin: float = 0.02, amax: float = 5e3) -> System:
    """64 atoms uniform in a 40-bohr cube (min separation 3 bohr); every atom has
    U_L (4 terms) + projectors l=0..4 (3 terms each) and s..g shells of 8
    primitives, exponents log-uniform [amin, amax] ([0.02, 5e3] for the workload;
    config1_moderate() narrows them)."""
    rng = np.random.default_rng(seed)
    xyz = _place(rng, n_atoms, 40.0, 3.0)
    grpps, shells, shell_atom, centres = [], [], [], []
    for i in range(n_atoms):
        grpps.append(_scalar_grpp(rng, 4, 4))
        centres.append((xyz[i].copy(), i))
        for L in range(5):
            shells.append(_shell(rng, xyz[i], L, 8, amin=amin, amax=amax))
            shell_atom.append(i)
    return System(shells, grpps, centres, CART_ORDER_TURBOMOLE, np.array(shell_atom, np.int32),
                  np.arange(n_atoms, dtype=np.int32), xyz)


def config1_moderate(seed: int = 1) -> System:
    """Config 1 with exponents log-uniform [0.1, 50]: the same atoms, potentials and
    shell shapes, on which libgrpp keeps its digits (its results move by less than
    the 1e-10 / 1e-9 tolerance under last-bit input changes)."""
    return config1(seed, amin=0.1, amax=50.0)


def _heavy_grpp(rng, l_proj=4, l_so=4, l_oc=3):
    """U_L + AREP projectors l=0..l_proj + SO l=1..l_so (c in [-5,5]) + outercore:
    for l=0..l_oc one (l=0) or two (l>0, J=2l-1 then 2l+1) 6-primitive
    subvalence shells (zeta log-uniform [0.1,30]) each paired with its own
    3-term potential, in the pairing order of test_libgrpp_c/rpp.c:118-139."""
    g = _scalar_grpp(rng, 4, l_proj)
    for l in range(1, l_so + 1):
        g.so.append(_terms(rng, l, 0, 3, cmax=5.0))
    for l in range(l_oc + 1):
        for ioc in range(1 if l == 0 else 2):
            J = abs(2 * l + (-1 if ioc % 2 == 0 else 1))
            sh = _shell(rng, np.zeros(3), l, 6, amin=0.1, amax=30.0)
            g.oc.append((_terms(rng, l, J, 3), sh))
    return g


def config2(seed: int = 2, n_heavy: int = 16, n_h: int = 32, lmax: int = 5, box: float = 30.0,
            l_proj: int = 4) -> System:
    """16 heavy atoms (full GRPP, shells l=0..lmax) + 32 H (s,p shells, no GRPP)
    in a 30-bohr box, min separation 1.5 bohr; basis shells have 8 primitives."""
    rng = np.random.default_rng(seed)
    xyz = _place(rng, n_heavy + n_h, box, 1.5)
    shells, shell_atom, grpps, centres, centre_atom = [], [], [], [], []
    for i in range(n_heavy + n_h):
        heavy = i < n_heavy
        if heavy:
            grpps.append(_heavy_grpp(rng, l_proj=l_proj))
            centres.append((xyz[i].copy(), len(grpps) - 1))
            centre_atom.append(i)
        for L in range(lmax + 1 if heavy else 2):
            shells.append(_shell(rng, xyz[i], L, 8))
            shell_atom.append(i)
    return System(shells, grpps, centres, CART_ORDER_TURBOMOLE, np.array(shell_atom, np.int32),
                  np.array(centre_atom, np.int32), xyz)


def moderate_heavy_system(seed: int = 7) -> System:
    """Two heavy atoms (U_L, projectors l <= 4, SO l <= 4, outercore s..d shells) and one H;
    basis shells s..f (H: s, p) of 6 primitives with exponents log-uniform [0.1, 30]. On
    such blocks libgrpp keeps its digits, so two implementations can be held to the strict
    1e-10 / 1e-9 tolerance element by element."""
    rng = np.random.default_rng(seed)
    xyz = np.array([[0.0, 0.0, 0.0], [1.1, -0.6, 2.3], [-1.4, 1.2, 0.7]])
    grpps = [_heavy_grpp(rng, l_proj=4, l_so=4, l_oc=2) for _ in range(2)]
    shells, shell_atom = [], []
    for i in range(3):
        for L in range(4 if i < 2 else 2):
            shells.append(_shell(rng, xyz[i], L, 6, amin=0.1, amax=30.0))
            shell_atom.append(i)
    return System(shells, grpps, [(xyz[0].copy(), 0), (xyz[1].copy(), 1)], CART_ORDER_TURBOMOLE,
                  np.array(shell_atom, np.int32), np.array([0, 1], np.int32), xyz)


def config3_density(system: System, seed: int = 3) -> np.ndarray:
    """Random symmetric density, entries uniform in [-1, 1]."""
    rng = np.random.default_rng(seed)
    n = system.n_basis()
    D = rng.uniform(-1.0, 1.0, (n, n))
    return np.triu(D) + np.triu(D, 1).T


def config4(seed: int = 4, n_mol: int = 512):
    """512 independent molecules of 2..24 atoms (uniform), drawn as config 2 with
    basis l <= 6 and projectors l <= 5; returns a list of Systems."""
    rng = np.random.default_rng(seed)
    mols = []
    for m in range(n_mol):
        n = int(rng.integers(2, 25))
        n_heavy = max(1, n // 3)
        sub_seed = int(rng.integers(0, 2**31 - 1))
        mols.append(config2(sub_seed, n_heavy=n_heavy, n_h=n - n_heavy, lmax=6, box=6.0 + 1.5 * n, l_proj=5))
    return mols


def sort_tasks(system: System, a, b, c):
    """Order tasks by class (la, lb, lmax of the centre's projectors)."""
    La = np.array([s.L for s in system.shells])
    lpot = np.array([max([p.L for p in g.arep + g.so] + [0]) for g in system.grpps])
    cg = np.array([cc[1] for cc in system.centres])
    key = (La[a] * 16 + La[b]) * 16 + lpot[cg[c]]
    o = np.lexsort((c, b, a, key))
    return a[o], b[o], c[o]


def merge_systems(systems):
    """One System holding independent molecules side by side (shells, GRPPs, centres and
    atoms concatenated; all must share one Cartesian order), and its task list: every
    ordered shell pair x centre within each molecule, sorted by class (la, lb, lpot)."""
    shells, grpps, centres, shell_atom, centre_atom, atoms = [], [], [], [], [], []
    ta, tb, tc = [], [], []
    for S in systems:
        s0, g0, c0, a0 = len(shells), len(grpps), len(centres), len(atoms)
        shells += list(S.shells)
        grpps += list(S.grpps)
        centres += [(o, gi + g0) for o, gi in S.centres]
        shell_atom.append(np.asarray(S.shell_atom) + a0)
        centre_atom.append(np.asarray(S.centre_atom) + a0)
        atoms += list(np.asarray(S.atoms))
        a, b, c = S.all_tasks()
        ta.append(a + s0)
        tb.append(b + s0)
        tc.append(c + c0)
    M = System(shells, grpps, centres, systems[0].cart_order, np.concatenate(shell_atom).astype(np.int32),
               np.concatenate(centre_atom).astype(np.int32), np.array(atoms))
    a, b, c = sort_tasks(M, np.concatenate(ta), np.concatenate(tb), np.concatenate(tc))
    return M, (a.astype(np.int32), b.astype(np.int32), c.astype(np.int32))
