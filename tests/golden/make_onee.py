"""Golden fixture of the one-electron integrals (tests/golden/onee.npz) from libgrpp itself.

Run here, where the reference tree and its compiled library exist:

    make -C oracle ref
    python tests/golden/make_onee.py [--ref-root <libgrpp source tree>]   (default: $LIBGRPP_REFERENCE)

For libgrpp's test directories H2O, Cs and K the molecule and basis are read with
libgrpp_b200.formats; the reference library (oracle/_ref/libgrpp_ref.so, libgrpp
compiled from its own sources) evaluates, shell pair by shell pair (and nucleus by
nucleus), the integrals libgrpp's C test driver writes
(test_libgrpp_c/main.c:396-489, eval_integrals.c:251-410, eval_integrals_grad.c):
  H2O  overlap, kinetic energy, momentum x/y/z, point-charge nuclear attraction and
       the overlap gradients d S / d R_atom;
  Cs   overlap, point-charge nuclear attraction;
  K    nuclear attraction for the point (analytic and numerical), charged-ball,
       Gaussian and Fermi nuclear models, the parameters from the K-39 rms radius
       of Johnson's estimate as the driver derives them (eval_integrals.c:372-390),
       and the Fermi-bubble model (k = 0.3), for which libgrpp ships no matrix;
  numeric type 1 <A|U_L|B> of config 0 (all tasks) and of 240 seeded H2O GRPP tasks by
       libgrpp's numeric radial quadrature (type1_integrals.c:109-270, called per
       primitive pair and contracted c_i c_j, primitive pairs in order), beside its
       McMurchie-Davidson value (libgrpp_type1_integrals).
Every matrix is checked against libgrpp's shipped one (absolute 1e-10 as
test/compare_matrices.c:25) before anything is written. The fixture holds, per
system, the flattened shells (b_* arrays), the shell-pair task list, the nuclei,
and the reference's per-task blocks.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from libgrpp_b200.capi import LibGRPP  # noqa: E402
from libgrpp_b200.formats import read_basis, read_lower_triangle, read_molecule  # noqa: E402
from libgrpp_b200.system import CART_ORDER_TURBOMOLE, GRPP, Shell, System, ncart  # noqa: E402

MASS_NUMBER = {1: 1, 8: 16, 19: 39, 55: 133}  # most abundant isotopes (test_libgrpp_c/elements.c)
FERMI_UNITS_TO_ATOMIC = 1.0 / 52917.7210903
MODELS = {"point": 0, "ball": 1, "gauss": 2, "fermi": 3, "fermi_bubble": 4, "point_numerical": 5}
SHIPPED = {"point": "nucattr_point.txt", "point_numerical": "nucattr_point_numerical.txt",
           "ball": "nucattr_charged_ball.txt", "gauss": "nucattr_gaussian.txt", "fermi": "nucattr_fermi.txt"}


def read_shells(d):
    Z, xyz = read_molecule(os.path.join(d, "molecule.xyz"))
    shells, cache = [], {}
    for i, z in enumerate(Z):
        if z not in cache:
            cache[z] = read_basis(os.path.join(d, "basis.inp"), int(z))
        shells += [Shell(xyz[i], L, c, a) for L, c, a in cache[z]]
    return Z, xyz, shells


def model_params(lib, z, model):
    """(Z-independent) parameters of a nuclear model as the C driver derives them."""
    R = lib.lib.libgrpp_estimate_nuclear_rms_radius_johnson_1985(MASS_NUMBER[int(z)])
    if model in ("ball", "gauss"):
        return np.array([R * FERMI_UNITS_TO_ATOMIC, 0.0, 0.0])
    if model in ("fermi", "fermi_bubble"):
        import ctypes as ct
        c, a = ct.c_double(), ct.c_double()
        lib.lib.libgrpp_estimate_fermi_model_parameters(R, ct.byref(c), ct.byref(a))
        k = 0.3 if model == "fermi_bubble" else 0.0
        return np.array([c.value * FERMI_UNITS_TO_ATOMIC, a.value * FERMI_UNITS_TO_ATOMIC, k])
    return np.zeros(3)


def dense(blocks, shells, pairs, nbf, off):
    M = np.zeros((nbf, nbf))
    o = 0
    for (i, j) in pairs:
        nA, nB = ncart(shells[i].L), ncart(shells[j].L)
        M[off[i]:off[i + 1], off[j]:off[j + 1]] += blocks[o:o + nA * nB].reshape(nA, nB)
        o += nA * nB
    return M


def check(d, fname, M, tol=1e-10):
    S = read_lower_triangle(os.path.join(d, fname))
    tri = np.tril_indices(M.shape[0])
    worst = float(np.max(np.abs(M[tri] - S[tri])))
    assert worst <= tol, f"{d}/{fname}: reference differs from shipped matrix by {worst}"
    return worst


def numeric_type1(lib, data):
    """Numeric type 1 blocks of U_L through libgrpp's own quadrature (an internal function of the
    reference library: evaluate_type1_integral_primitive_gaussians) and the MMD blocks."""
    import ctypes as ct
    from libgrpp_b200 import synthetic
    from libgrpp_b200.system import BatchArrays, cartesian_list
    from tests.util import fixture_subset, load_fixture, system_from_fixture
    D, I = ct.POINTER(ct.c_double), ct.POINTER(ct.c_int)
    f = lib.lib.evaluate_type1_integral_primitive_gaussians
    f.restype = None
    f.argtypes = [D, ct.c_int, I, ct.c_double, D, ct.c_int, I, ct.c_double, D, ct.c_void_p, D]
    h2o, z = load_fixture("h2o")
    sel = np.sort(np.random.default_rng(17).choice(len(h2o.task_a), 240, replace=False))
    h2o_sub, _, _ = fixture_subset(h2o, z, sel)
    for key, system, batch in (("config0", synthetic.config0(), synthetic.config0().batch()),
                               ("h2o", system_from_fixture(z), h2o_sub)):
        lib.set_cartesian_order(system.cart_order)
        d = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in batch.__dict__.items() if not k.startswith("_")}
        for k in ("grpp_n_arep", "grpp_n_so", "grpp_n_oc"):
            d[k] = np.zeros_like(d[k])
        ul = BatchArrays(**d)
        num, mmd = [], []
        for t in range(len(ul.task_a)):
            si, sj = system.shells[int(ul.task_a[t])], system.shells[int(ul.task_b[t])]
            C, g = system.centres[int(ul.task_c[t])]
            nA, nB = ncart(si.L), ncart(sj.L)
            hp = lib.new_potential(system.grpps[g].UL)
            ca = np.ascontiguousarray(cartesian_list(si.L, system.cart_order).ravel())
            cb = np.ascontiguousarray(cartesian_list(sj.L, system.cart_order).ravel())
            C = np.ascontiguousarray(C, dtype=np.float64)
            oa, ob = np.ascontiguousarray(si.origin), np.ascontiguousarray(sj.origin)
            blk = np.zeros(nA * nB)
            for p in range(len(si.alpha)):
                for q in range(len(sj.alpha)):
                    buf = np.zeros(nA * nB)
                    f(oa.ctypes.data_as(D), nA, ca.ctypes.data_as(I), si.alpha[p], ob.ctypes.data_as(D), nB,
                      cb.ctypes.data_as(I), sj.alpha[q], C.ctypes.data_as(D), hp, buf.ctypes.data_as(D))
                    blk += (si.coeffs[p] * sj.coeffs[q]) * buf
            num.append(blk)
            mmd.append(lib.type1(lib.new_shell(si), lib.new_shell(sj), C, hp, nA, nB).ravel())
        for k, v in ul.__dict__.items():
            if not k.startswith("_"):
                data[f"num_{key}_b_{k}"] = v
        data[f"num_{key}_numeric"] = np.concatenate(num)
        data[f"num_{key}_mmd"] = np.concatenate(mmd)
        gap = np.abs(data[f"num_{key}_numeric"] - data[f"num_{key}_mmd"])
        print(f"numeric type 1 ({key}): {len(num)} tasks; libgrpp's numeric vs its MMD max abs {gap.max():.2e}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=os.environ.get("LIBGRPP_REFERENCE", "/root/reference"))
    args = ap.parse_args()
    lib = LibGRPP(os.path.join(ROOT, "oracle", "_ref", "libgrpp_ref.so"))
    lib.set_cartesian_order(CART_ORDER_TURBOMOLE)
    data = {}
    for name, kinds, models in (("H2O", ("overlap", "kinetic", "momentum"), ("point",)),
                                ("Cs", ("overlap",), ("point",)),
                                ("K", (), ("point", "point_numerical", "ball", "gauss", "fermi", "fermi_bubble"))):
        d = os.path.join(args.ref_root, "test", name)
        Z, xyz, shells = read_shells(d)
        S = System(shells, [GRPP()], [(xyz[i].copy(), 0) for i in range(len(Z))], CART_ORDER_TURBOMOLE)
        ns = len(shells)
        pairs = [(i, j) for i in range(ns) for j in range(ns)]
        a = np.array([p[0] for p in pairs], np.int32)
        b = np.array([p[1] for p in pairs], np.int32)
        # nuclear attraction tasks: every pair x every nucleus (centre c = atom c)
        na = np.repeat(a, len(Z))
        nb = np.repeat(b, len(Z))
        nc = np.tile(np.arange(len(Z), dtype=np.int32), len(pairs))
        batch = S.batch(na, nb, nc)
        key = name.lower()
        for k, v in batch.__dict__.items():
            if not k.startswith("_"):
                data[f"{key}_b_{k}"] = v
        data[f"{key}_Z"] = Z
        off = S.basis_offsets()
        nbf = int(off[-1])
        hs = [lib.new_shell(s) for s in shells]
        msg = []
        for kind in kinds:
            outs = []
            for (i, j) in pairs:
                nA, nB = ncart(shells[i].L), ncart(shells[j].L)
                if kind == "overlap":
                    outs.append([lib.overlap(hs[i], hs[j], nA, nB).ravel()])
                elif kind == "kinetic":
                    outs.append([lib.kinetic(hs[i], hs[j], nA, nB).ravel()])
                else:
                    outs.append([x.ravel() for x in lib.momentum(hs[i], hs[j], nA, nB)])
            comps = [np.concatenate([o[m] for o in outs]) for m in range(len(outs[0]))]
            files = {"overlap": ["overlap.txt"], "kinetic": ["kinetic_energy.txt"],
                     "momentum": ["momentum_x.txt", "momentum_y.txt", "momentum_z.txt"]}[kind]
            for m, (f, c) in enumerate(zip(files, comps)):
                w = check(d, f, dense(c, shells, pairs, nbf, off))
                data[f"{key}_{f[:-4]}"] = c
                msg.append(f"{f[:-4]} {w:.1e}")
        for model in models:
            prm = np.stack([model_params(lib, z, model) for z in Z])
            blocks = []
            for t in range(len(na)):
                i, j, c = int(na[t]), int(nb[t]), int(nc[t])
                blocks.append(lib.nuclear_attraction(hs[i], hs[j], xyz[c], int(Z[c]), MODELS[model], prm[c],
                                                     ncart(shells[i].L), ncart(shells[j].L)).ravel())
            blocks = np.concatenate(blocks)
            data[f"{key}_nuc_{model}"] = blocks
            data[f"{key}_nuc_{model}_params"] = prm
            fname = "coulomb.txt" if name != "K" else SHIPPED.get(model)
            if fname:
                M = np.zeros((nbf, nbf))
                o = 0
                for t in range(len(na)):
                    i, j = int(na[t]), int(nb[t])
                    nA, nB = ncart(shells[i].L), ncart(shells[j].L)
                    M[off[i]:off[i + 1], off[j]:off[j + 1]] += blocks[o:o + nA * nB].reshape(nA, nB)
                    o += nA * nB
                msg.append(f"nuc_{model} {check(d, fname, M):.1e}")
        if name == "H2O":
            # overlap gradients: libgrpp's shipped matrices d S / d R_atom (lower triangles)
            tri = np.tril_indices(nbf)
            g = np.zeros((len(Z), 3, len(tri[0])))
            for at in range(len(Z)):
                for k, ax in enumerate("xyz"):
                    g[at, k] = read_lower_triangle(os.path.join(d, f"overlap_grad_{at}{ax}.txt"))[tri]
            data["h2o_overlap_grad_lower"] = g
        print(f"{name}: {ns} shells, {nbf} basis functions; shipped-matrix check: " + ", ".join(msg))
    numeric_type1(lib, data)
    out = os.path.join(HERE, "onee.npz")
    np.savez_compressed(out, **data)
    print(f"-> {os.path.relpath(out, ROOT)} ({os.path.getsize(out) / 1e3:.0f} kB)")


if __name__ == "__main__":
    main()
