"""Host side of the density-contracted gradient: the differentiated shells and the task list of
the derivative blocks, and libgrpp's rule for which atoms a block's derivative reaches.

libgrpp differentiates a Cartesian Gaussian as d/dA_k |a> = |a + 1_k>' - a_k |a - 1_k>', with
the L+1 shell's coefficients multiplied by 2 alpha N_L / N_{L+1} and the L-1 shell's by
N_L / N_{L-1} (libgrpp/diff_gaussian.c:35-63); which atom receives the bra or ket derivative,
with which sign, follows libgrpp/grpp_integrals_gradient.c:280-393. The engine applies the same
construction in C (libgrpp_b200_grpp_gradient_contract); this module exposes it to Python for
the benchmark's kernel timing and for the test fixtures.
"""
from __future__ import annotations

import numpy as np

from .system import BatchArrays, cartesian_list


def points_equal(a, b):
    return bool(np.all(np.abs(np.asarray(a) - np.asarray(b)) < 1e-12))


def gradient_terms(A, B, C, D):
    """(differentiate bra?, sign) pairs of libgrpp_full_grpp_integrals_gradient for point D
    (libgrpp/grpp_integrals_gradient.c:280-393)."""
    pe = points_equal
    out = []
    if pe(A, C) and pe(B, C):
        return out
    if not pe(A, D) and not pe(B, D) and not pe(C, D):
        return out
    if not pe(A, C) and not pe(C, B) and not pe(A, B):
        if pe(A, D):
            out.append((True, 1.0))
        if pe(B, D):
            out.append((False, 1.0))
        if pe(C, D):
            out += [(True, -1.0), (False, -1.0)]
    if pe(A, B) and not pe(A, C):
        f = 1.0 if pe(A, D) else -1.0
        out += [(True, f), (False, f)]
    if not pe(A, C) and pe(C, B):
        out.append((True, 1.0 if pe(A, D) else -1.0))
    if pe(A, C) and not pe(C, B):
        out.append((False, 1.0 if pe(B, D) else -1.0))
    return out


def _gnorm(L, a):
    return (2 * a / np.pi) ** 0.75 * (4 * a) ** (0.5 * L)


def derivative_batch(batch, cart_order):
    """The batch's shells plus, for each shell, its L+1 and L-1 differentiated shells, and the
    task list (A-1,B) (A+1,B) (A,B-1) (A,B+1) per task (-1 where L = 0)."""
    d = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in batch.__dict__.items() if not k.startswith("_")}
    sL, snp, spo, sco = (list(d[k]) for k in ("shell_L", "shell_nprim", "shell_prim_off", "shell_cart_off"))
    pc, pa, so, cart = list(d["prim_coef"]), list(d["prim_alpha"]), list(d["shell_origin"]), list(d["cart_list"])
    ns = len(sL)

    def add(s, L, raise_):
        idx = len(sL)
        sL.append(L)
        snp.append(snp[s])
        spo.append(len(pc))
        sco.append(len(cart) // 3)
        cart.extend(cartesian_list(L, cart_order).ravel().tolist())
        for i in range(snp[s]):
            al = pa[spo[s] + i]
            f = 2.0 * al * _gnorm(sL[s], al) / _gnorm(L, al) if raise_ else _gnorm(sL[s], al) / _gnorm(L, al)
            pc.append(pc[spo[s] + i] * f)
            pa.append(al)
        so.extend(so[3 * s:3 * s + 3])
        return idx

    up = [add(s, sL[s] + 1, True) for s in range(ns)]
    dn = [add(s, sL[s] - 1, False) if sL[s] > 0 else -1 for s in range(ns)]
    ta, tb, tc, sub = [], [], [], []
    for t in range(len(d["task_a"])):
        a, b, c = int(d["task_a"][t]), int(d["task_b"][t]), int(d["task_c"][t])
        ids = []
        for x, y in ((dn[a], b), (up[a], b), (a, dn[b]), (a, up[b])):
            if x < 0 or y < 0:
                ids.append(-1)
                continue
            ta.append(x)
            tb.append(y)
            tc.append(c)
            ids.append(len(ta) - 1)
        sub.append(ids)
    d.update(shell_L=np.array(sL, np.int32), shell_nprim=np.array(snp, np.int32), shell_prim_off=np.array(spo, np.int32),
             shell_cart_off=np.array(sco, np.int32), prim_coef=np.array(pc), prim_alpha=np.array(pa),
             shell_origin=np.array(so), cart_list=np.array(cart, np.int32), task_a=np.array(ta, np.int32),
             task_b=np.array(tb, np.int32), task_c=np.array(tc, np.int32))
    return BatchArrays(**d), sub


