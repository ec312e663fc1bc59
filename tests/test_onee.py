"""One-electron integrals: overlap, kinetic energy, momentum, nuclear attraction for the
point, charged-ball, Gaussian, Fermi and Fermi-bubble nuclear models, overlap gradients,
and the numeric radial type 1 quadrature.

GPU results are compared with tests/golden/onee.npz (libgrpp compiled from its sources,
checked against libgrpp's shipped H2O, Cs and K matrices by tests/golden/make_onee.py) at
the tolerance of record, max(1e-10, 1e-9 |ref|). The numeric type 1 quadrature is checked
against the McMurchie-Davidson evaluation of the same U_L blocks. The nuclear-model
functions are host code and are compared with libgrpp's own on the CPU.
"""
import ctypes as ct
import os

import numpy as np
import pytest

from libgrpp_b200.capi import PRODUCT_LIB
from libgrpp_b200.system import BatchArrays, ncart
from tests.util import GOLDEN, load_fixture, truth_parity

MODELS = {"point": 0, "ball": 1, "gauss": 2, "fermi": 3, "fermi_bubble": 4, "point_numerical": 5}


def _onee(system):
    z = np.load(os.path.join(GOLDEN, "onee.npz"))
    key = system + "_b_"
    batch = BatchArrays(**{k[len(key):]: np.ascontiguousarray(z[k]) for k in z.files if k.startswith(key)})
    return batch, z


def _shells(batch):
    from libgrpp_b200.system import Shell
    out = []
    for i in range(len(batch.shell_L)):
        o, n = int(batch.shell_prim_off[i]), int(batch.shell_nprim[i])
        out.append(Shell(batch.shell_origin[3 * i:3 * i + 3], int(batch.shell_L[i]), batch.prim_coef[o:o + n],
                         batch.prim_alpha[o:o + n]))
    return out


def _pairs(batch, n_nuclei):
    """The shell-pair tasks (one per pair) of a nuclear-attraction task list (pairs x nuclei)."""
    d = {k: v for k, v in batch.__dict__.items() if not k.startswith("_")}
    for k in ("task_a", "task_b", "task_c"):
        d[k] = np.ascontiguousarray(d[k][::n_nuclei])
    return BatchArrays(**d)


def test_nuclear_models_match_reference(ref_lib):
    """libgrpp_coulomb_potential_*, charge densities and rms radii (host code; the Fermi forms
    through the regenerated S_k table) against libgrpp's own functions."""
    P, R = ct.CDLL(PRODUCT_LIB), ref_lib.lib
    d = ct.c_double
    sig = {"libgrpp_coulomb_potential_fermi": [d] * 4, "libgrpp_coulomb_potential_fermi_bubble": [d] * 5,
           "libgrpp_coulomb_potential_ball": [d] * 3, "libgrpp_coulomb_potential_gaussian": [d] * 3,
           "libgrpp_coulomb_potential_point": [d] * 2, "libgrpp_charge_density_fermi": [d] * 4,
           "libgrpp_charge_density_fermi_bubble": [d] * 5, "libgrpp_charge_density_ball": [d] * 3,
           "libgrpp_charge_density_gaussian": [d] * 3, "libgrpp_rms_radius_fermi": [ct.c_int, d, d],
           "libgrpp_rms_radius_fermi_bubble": [ct.c_int, d, d, d],
           "libgrpp_estimate_nuclear_rms_radius_johnson_1985": [ct.c_int],
           "libgrpp_estimate_nuclear_rms_radius_golovko_2008": [ct.c_int]}
    for L in (P, R):
        for n, args in sig.items():
            getattr(L, n).restype = d
            getattr(L, n).argtypes = args
    worst = 0.0
    for c, a in ((6.5e-5, 1.1e-5), (1.3e-4, 1.0e-5)):
        for r in np.concatenate([np.geomspace(1e-7, 1e-3, 300), np.linspace(1e-5, 3e-4, 300)]):
            for fn, extra in (("libgrpp_coulomb_potential_fermi", (19.0, c, a)),
                              ("libgrpp_coulomb_potential_fermi_bubble", (19.0, c, a, 0.3)),
                              ("libgrpp_coulomb_potential_ball", (19.0, c)), ("libgrpp_coulomb_potential_gaussian", (19.0, c)),
                              ("libgrpp_coulomb_potential_point", (19.0,)), ("libgrpp_charge_density_fermi", (19.0, c, a)),
                              ("libgrpp_charge_density_fermi_bubble", (19.0, c, a, 0.3)),
                              ("libgrpp_charge_density_ball", (19.0, c)), ("libgrpp_charge_density_gaussian", (19.0, c))):
                x, y = getattr(P, fn)(r, *extra), getattr(R, fn)(r, *extra)
                worst = max(worst, abs(x - y) / max(abs(y), 1e-300))
        for Z in (19, 55, 92):
            assert abs(P.libgrpp_rms_radius_fermi(Z, c, a) / R.libgrpp_rms_radius_fermi(Z, c, a) - 1) < 1e-13
            assert abs(P.libgrpp_rms_radius_fermi_bubble(Z, c, a, 0.3) / R.libgrpp_rms_radius_fermi_bubble(Z, c, a, 0.3) - 1) < 1e-13
    for A in (1, 39, 238):
        assert P.libgrpp_estimate_nuclear_rms_radius_johnson_1985(A) == R.libgrpp_estimate_nuclear_rms_radius_johnson_1985(A)
        assert P.libgrpp_estimate_nuclear_rms_radius_golovko_2008(A) == R.libgrpp_estimate_nuclear_rms_radius_golovko_2008(A)
    print(f"nuclear models: max relative difference {worst:.2e}")
    assert worst < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("system", ["h2o", "cs"])
def test_onee_batch_blocks(gpu_lib, system):
    """Overlap, kinetic energy and momentum blocks of every shell pair (libgrpp_b200_onee_batch)."""
    batch, z = _onee(system)
    pairs = _pairs(batch, len(z[f"{system}_Z"]))
    kinds = [("overlap", 0, ["overlap"])]
    if system == "h2o":
        kinds += [("kinetic", 1, ["kinetic_energy"]), ("momentum", 2, ["momentum_x", "momentum_y", "momentum_z"])]
    for name, kind, keys in kinds:
        got = gpu_lib.onee_batch(pairs, kind)
        for g, k in zip(got, keys):
            ok, rep = truth_parity(g, z[f"{system}_{k}"])
            print(f"{system} {k}: max abs {rep['max_abs']:.2e}")
            assert ok, (system, k, rep)


@pytest.mark.gpu
@pytest.mark.parametrize("system,model", [("h2o", "point"), ("cs", "point")] +
                         [("k", m) for m in ("point", "point_numerical", "ball", "gauss", "fermi", "fermi_bubble")])
def test_nuclear_attraction_batch(gpu_lib, system, model):
    """libgrpp_b200_nuclear_attraction_batch for every (pair, nucleus) task: point charges through the
    type 1 McMurchie-Davidson kernel, the finite models through the numeric type 1 kernel."""
    batch, z = _onee(system)
    Z = z[f"{system}_Z"].astype(np.float64)
    charges = Z  # centre c is nucleus c
    params = z[f"{system}_nuc_{model}_params"] if f"{system}_nuc_{model}_params" in z.files else None
    got = gpu_lib.nuclear_attraction_batch(batch, MODELS[model], charges, params)
    ok, rep = truth_parity(got, z[f"{system}_nuc_{model}"])
    print(f"{system} nuclear attraction ({model}): max abs {rep['max_abs']:.2e}")
    assert ok, (system, model, rep)


@pytest.mark.gpu
def test_single_call_one_electron_api(gpu_lib):
    """libgrpp_overlap/kinetic_energy/momentum/nuclear_attraction_integrals for single shell pairs
    through the C API against the fixture's blocks."""
    batch, z = _onee("k")
    gpu_lib.set_cartesian_order(1)
    shells = _shells(batch)
    off = batch.block_offsets()
    Z = int(z["k_Z"][0])
    for t in (0, 13, 47, len(batch.task_a) - 1):
        i, j = int(batch.task_a[t]), int(batch.task_b[t])
        si, sj = shells[i], shells[j]
        nA, nB = ncart(si.L), ncart(sj.L)
        hA, hB = gpu_lib.new_shell(si), gpu_lib.new_shell(sj)
        C = batch.centre_origin[:3]
        for model in ("point", "ball", "fermi"):
            got = gpu_lib.nuclear_attraction(hA, hB, C, Z, MODELS[model], z[f"k_nuc_{model}_params"][0], nA, nB)
            ok, rep = truth_parity(got.ravel(), z[f"k_nuc_{model}"][off[t]:off[t + 1]])
            assert ok, (t, model, rep)


@pytest.mark.gpu
def test_overlap_gradients_h2o(gpu_lib):
    """d S / d R_atom for all atoms through libgrpp_overlap_integrals_gradient against libgrpp's
    shipped matrices (test/H2O/overlap_grad_*)."""
    batch, z = _onee("h2o")
    gpu_lib.set_cartesian_order(1)
    nuc = len(z["h2o_Z"])
    pairs = _pairs(batch, nuc)
    shells = _shells(pairs)
    off = np.concatenate([[0], np.cumsum([ncart(s.L) for s in shells])])
    n = int(off[-1])
    atoms = batch.centre_origin.reshape(-1, 3)
    hs = [gpu_lib.new_shell(s) for s in shells]
    G = np.zeros((nuc, 3, n, n))
    for i, si in enumerate(shells):
        for j, sj in enumerate(shells):
            for at in range(nuc):
                G[at, :, off[i]:off[i + 1], off[j]:off[j + 1]] = gpu_lib.overlap_gradient(hs[i], hs[j], atoms[at],
                                                                                          ncart(si.L), ncart(sj.L))
    tri = np.tril_indices(n)
    ok, rep = truth_parity(G[:, :, tri[0], tri[1]].ravel(), z["h2o_overlap_grad_lower"].ravel())
    assert ok, rep


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["h2o", "config0"])
def test_numeric_type1(gpu_lib, name):
    """<A|U_L|B> by the numeric radial quadrature (libgrpp_b200_type1_numeric_batch) against libgrpp's
    own numeric quadrature of the same blocks (strict), and against the McMurchie-Davidson values:
    the two methods agree to ~1e-15 on H2O; on config 0 (f x f blocks, potential exponents up to 50)
    libgrpp's numeric scheme, capped at 8191 points, stays 3.6e-7 from its MMD on one element, and
    the GPU's numeric path reproduces exactly that gap."""
    batch, z = _onee("num_" + name)
    num = gpu_lib.type1_numeric_batch(batch)
    ok, rep = truth_parity(num, z[f"num_{name}_numeric"])
    gap_ref = np.abs(z[f"num_{name}_numeric"] - z[f"num_{name}_mmd"])
    gap_gpu = np.abs(num - gpu_lib.full_grpp_batch(batch)[0])
    print(f"{name}: numeric type 1 vs libgrpp's numeric max abs {rep['max_abs']:.2e}; numeric vs MMD: libgrpp "
          f"{gap_ref.max():.2e}, GPU {gap_gpu.max():.2e}")
    assert ok, rep
    assert np.all(gap_gpu <= gap_ref + np.maximum(1e-10, 1e-9 * np.abs(z[f"num_{name}_mmd"])))
