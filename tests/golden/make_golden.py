"""Generate the golden fixtures under tests/golden/ from libgrpp itself.

Run here, where the reference tree and its compiled library exist:

    make -C oracle ref
    python tests/golden/make_golden.py [--ref-root <libgrpp source tree>]   (default: $LIBGRPP_REFERENCE)

For each of libgrpp's GRPP test directories (test/H2O, Cs, ThO, UO2, KCs) the
molecule, basis and GRPP inputs are read with libgrpp_b200.formats, the
reference library (oracle/_ref/libgrpp_ref.so, libgrpp compiled from its own
sources) evaluates libgrpp_full_grpp_integrals task by task, and the result is
checked against the reference's own shipped matrices (arep.txt, so_*.txt;
absolute 1e-10 as test/compare_matrices.c:25) before anything is written.

Fixtures (npz): the flattened task description (``b_*`` arrays), the task list,
the reference's per-task blocks (``ref_arep`` ... ``ref_so_z``) and their
sensitivity to last-bit input changes (``env_*``: the largest change of each
element when the reference is re-run with exponents, coefficients and
coordinates moved by up to 4 units of roundoff: uniformly scaled, and
independently per primitive in eight seeded random draws, tests/util.py
``perturbed``). H2O and Cs
hold every task; ThO, UO2 and KCs hold a seeded sample of shell pairs x all
centres (the full matrices are tens of MB). H2O also holds libgrpp's
shipped GRPP gradient matrices d V / d R_atom (36 lower triangles from
test/H2O/{arep,so_x,so_y,so_z}_grad_{0,1,2}{x,y,z}.txt).

Two more fixtures pin the engine on the seeded synthetic workloads it is
benchmarked on (libgrpp_b200.synthetic): config1.npz, 512 seeded tasks of the
config-1 task list (64 atoms, s..g shells, U_L + projectors l = 0..4), and
config2.npz, 384 seeded tasks of config 2 (full GRPP: U_L, projectors,
spin-orbit and outercore terms, basis up to h). Their reference values and
envelopes come from the same compiled libgrpp. config3.npz pins the
density-contracted gradient d tr(D V)/dR on a seeded task sample of a small
config-2-type system (3 heavy atoms + 3 H, basis up to f) with a random
symmetric D; its reference is the oracle's driver over the restated
libgrpp_full_grpp_integrals_gradient (pinned against libgrpp's 36 shipped H2O
gradient matrices), because the compiled libgrpp gradient reads past its L-1
block and can return NaN (grpp_integrals_gradient.c:452-466).
"""
from __future__ import annotations

import argparse
import os
import sys
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from libgrpp_b200 import synthetic  # noqa: E402
from libgrpp_b200.capi import LibGRPP  # noqa: E402
from libgrpp_b200.formats import read_lower_triangle, read_system  # noqa: E402
from tests.util import envelope  # noqa: E402

COMPS = ("arep", "so_x", "so_y", "so_z")
# fixture -> (all tasks?, tolerance against the shipped matrices)
FIXTURES = {"H2O": (True, 1e-10), "Cs": (True, 1e-10), "ThO": (False, 1e-10), "UO2": (False, 1e-10),
            "KCs": (False, 3e-10)}


def batch_arrays(b):
    return {"b_" + k: v for k, v in b.__dict__.items() if not k.startswith("_") and not k.startswith("task_")}


def dense_from_blocks(system, batch, blocks):
    return system.assemble(batch, blocks)


def check_against_shipped(d, system, batch, outs, tol):
    worst = 0.0
    for m, name in enumerate(COMPS):
        M = dense_from_blocks(system, batch, outs[m])
        G = read_lower_triangle(os.path.join(d, name + ".txt"))
        L = np.tril(M)
        L[np.abs(L) <= 1e-14] = 0.0
        d_ = np.abs(L - G)
        assert np.all(np.isfinite(d_)), "non-finite reference value"
        worst = max(worst, float(d_.max()))
    return worst


def sample_tasks(system, n_pairs, seed):
    rng = np.random.default_rng(seed)
    ns, nc = len(system.shells), len(system.centres)
    pairs = rng.choice(ns * ns, size=min(n_pairs, ns * ns), replace=False)
    a = np.repeat(pairs // ns, nc).astype(np.int32)
    b = np.repeat(pairs % ns, nc).astype(np.int32)
    c = np.tile(np.arange(nc), len(pairs)).astype(np.int32)
    return a, b, c


# synthetic fixture -> (generator, number of seeded tasks, sampling seed)
SYNTHETIC = {"config1": (synthetic.config1, 512, 11), "config2": (synthetic.config2, 384, 12),
             "config1_moderate": (synthetic.config1_moderate, 512, 11)}


def write_fixture(name, system, a, b, c, outs, env, extra=None):
    batch = system.batch(a, b, c)
    data = dict(batch_arrays(batch))
    data.update(task_a=a, task_b=b, task_c=c, n_basis=system.n_basis(),
                basis_offsets=system.basis_offsets(), cart_order=system.cart_order)
    for m, comp in enumerate(COMPS):
        data["ref_" + comp] = outs[m]
        data["env_" + comp] = env[m]
    if extra:
        data.update(extra)
    out = os.path.join(HERE, f"{name.lower()}.npz")
    np.savez_compressed(out, **data)
    return out


def make_synthetic(lib, name):
    gen, n, seed = SYNTHETIC[name]
    system = gen()
    a, b, c = system.all_tasks()
    sel = np.sort(np.random.default_rng(seed).choice(len(a), n, replace=False))
    a, b, c = a[sel], b[sel], c[sel]
    outs, env = envelope(lib, system.batch(a, b, c))
    n_ill = sum(int(np.sum(e > 1e-10)) for e in env)
    out = write_fixture(name, system, a, b, c, outs, env)
    print(f"{name}: {len(a)} tasks -> {os.path.relpath(out, ROOT)} ({os.path.getsize(out) / 1e3:.0f} kB); "
          f"{n_ill} elements move by more than 1e-10 under 4-ulp input changes")


def make_gradient_fixture(n_tasks=160, seed=13):
    from tests.util import grad_envelope, load_oracle
    orc = load_oracle()
    system = synthetic.config2(seed=3, n_heavy=3, n_h=3, lmax=3, box=8.0)
    D = synthetic.config3_density(system, seed=3)
    a, b, c = system.all_tasks()
    sel = np.sort(np.random.default_rng(seed).choice(len(a), n_tasks, replace=False))
    a, b, c = a[sel], b[sel], c[sel]
    batch = system.batch(a, b, c)
    g, env = grad_envelope(orc, system, batch, D)
    assert np.all(np.isfinite(g))
    out = os.path.join(HERE, "config3.npz")
    data = dict(batch_arrays(batch))
    data.update(task_a=a, task_b=b, task_c=c, n_basis=system.n_basis(), basis_offsets=system.basis_offsets(),
                cart_order=system.cart_order, atoms=system.atoms, shell_atom=system.shell_atom,
                centre_atom=system.centre_atom, D=D, ref_grad=g, env_grad=env)
    for comp in COMPS:  # no per-task blocks in this fixture
        data["ref_" + comp] = np.zeros(0)
        data["env_" + comp] = np.zeros(0)
    np.savez_compressed(out, **data)
    print(f"config3: {len(a)} tasks, gradient [4, {len(system.atoms)}, 3] -> {os.path.relpath(out, ROOT)} "
          f"({os.path.getsize(out) / 1e3:.0f} kB); max |g| {np.abs(g).max():.3e}, max env {env.max():.3e}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=os.environ.get("LIBGRPP_REFERENCE", "/root/reference"))
    ap.add_argument("--only", nargs="*")
    ap.add_argument("--pairs", type=int, default=48)
    args = ap.parse_args()
    lib = LibGRPP(os.path.join(ROOT, "oracle", "_ref", "libgrpp_ref.so"))
    for name in SYNTHETIC:
        if args.only and name not in args.only:
            continue
        make_synthetic(lib, name)
    if not args.only or "config3" in args.only:
        make_gradient_fixture()
    for name, (full, tol) in FIXTURES.items():
        if args.only and name not in args.only:
            continue
        d = os.path.join(args.ref_root, "test", name)
        system = read_system(d)
        if full:
            a, b, c = system.all_tasks()
        else:
            a, b, c = sample_tasks(system, args.pairs, seed=zlib.crc32(name.encode()) % 1000)
        batch = system.batch(a, b, c)
        outs, env = envelope(lib, batch)
        data = dict(batch_arrays(batch))
        data.update(task_a=a, task_b=b, task_c=c, n_basis=system.n_basis(),
                    basis_offsets=system.basis_offsets(), cart_order=system.cart_order)
        for m, comp in enumerate(COMPS):
            data["ref_" + comp] = outs[m]
            data["env_" + comp] = env[m]
        msg = ""
        if full:
            worst = check_against_shipped(d, system, batch, outs, tol)
            assert worst <= tol, f"{name}: reference through this reader differs from shipped matrices by {worst}"
            msg = f"shipped-matrix check {worst:.2e}"
        if name == "H2O":
            # gradient goldens: libgrpp's shipped matrices themselves. (Recomputing them
            # through the compiled library is not used: libgrpp_full_grpp_integrals_gradient
            # reads outside its L-1 block when a Cartesian exponent is 0 and multiplies the
            # value by 0, which yields NaN whenever that memory holds one.)
            tri = np.tril_indices(system.n_basis())
            gl = np.zeros((4, len(system.atoms), 3, len(tri[0])))
            for m, comp in enumerate(COMPS):
                for at in range(len(system.atoms)):
                    for k, ax in enumerate("xyz"):
                        Gs = read_lower_triangle(os.path.join(d, f"{comp}_grad_{at}{ax}.txt"))
                        gl[m, at, k] = Gs[tri]
            assert np.all(np.isfinite(gl))
            data["ref_grad_lower"] = gl
            data["atoms"] = system.atoms
            data["shell_atom"] = system.shell_atom
            data["centre_atom"] = system.centre_atom
            msg += "; gradients from the shipped matrices"
        out = os.path.join(HERE, f"{name.lower()}.npz")
        np.savez_compressed(out, **data)
        print(f"{name}: {len(a)} tasks -> {os.path.relpath(out, ROOT)} ({os.path.getsize(out) / 1e3:.0f} kB) {msg}")


if __name__ == "__main__":
    main()
