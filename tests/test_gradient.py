"""Density-contracted GRPP gradient (libgrpp_b200_grpp_gradient_contract):
g[m][atom][k] = d tr(D V^m) / d R_atom,k for the four matrices m = arep, so_x, so_y, so_z.

Checked against the oracle's driver over the restated
libgrpp_full_grpp_integrals_gradient contracted with D (golden fixture config3)
at 1e-10 / 1e-9; where the oracle keeps fewer digits than that, against the
binary128 gradient of tests/golden/truth_config3.npz within twice the oracle's
own distance from it. Also against central finite differences (h = 1e-4 bohr)
of tr(D V^m) computed with the engine's integrals.
"""
import numpy as np
import pytest

from libgrpp_b200 import synthetic
from libgrpp_b200.system import GRPP, System
from tests.util import load_fixture, load_truth, system_from_fixture, truth_parity

pytestmark = pytest.mark.gpu
COMPS = ("arep", "so_x", "so_y", "so_z")


@pytest.mark.parametrize("mode", [0, 1])
def test_gradient_contract_matches_oracle(gpu_lib, mode):
    batch, z = load_fixture("config3")
    S = system_from_fixture(z)
    truth = load_truth("config3")
    g = gpu_lib.grad_contract(S, batch, z["D"], radial_mode=mode)
    tr = {"truth_grad": truth["truth_grad"].ravel(), "refdev_grad": truth["refdev_grad"].ravel()}
    ok, rep = truth_parity(g.ravel(), z["ref_grad"].ravel(), tr, np.arange(g.size), "grad")
    print(f"config3 gradient (mode {mode}): max abs {rep['max_abs']:.2e}, strict misses {rep['strict_fail']} "
          f"(judged against the truth {rep['truth_checked']}, failing {rep['truth_fail']}; max |oracle-truth| "
          f"{rep['max_ref_truth']:.2e}, max |gpu-truth| {rep['max_got_truth']:.2e})")
    assert ok, rep


def test_symmetric_density_folding(gpu_lib):
    """libgrpp_b200_grpp_gradient_contract_symmetric: shell pairs folded onto A <= B and no
    spin-orbit work. On the config3 fixture (a partial task list) the arep gradient equals the
    oracle's (and the truth where the oracle keeps few digits) and the spin-orbit gradient
    receives nothing. On a system with every ordered shell pair listed, the unfolded spin-orbit
    contractions, whose exact value is zero for a symmetric density (the SO matrices are
    antisymmetric), are rounding noise, and the folded arep gradient equals the unfolded one."""
    batch, z = load_fixture("config3")
    S = system_from_fixture(z)
    truth = load_truth("config3")
    sym = gpu_lib.grad_contract(S, batch, z["D"], symmetric=True)
    tr = {"truth_grad": truth["truth_grad"][0].ravel(), "refdev_grad": truth["refdev_grad"][0].ravel()}
    ok, rep = truth_parity(sym[0].ravel(), z["ref_grad"][0].ravel(), tr, np.arange(sym[0].size), "grad")
    assert ok, rep
    assert np.all(sym[1:] == 0.0)
    S2 = _small_system()
    b2 = S2.batch()  # every ordered shell pair x every centre
    n = int(S2.basis_offsets()[-1])
    D = np.random.default_rng(5).uniform(-1, 1, (n, n))
    D = 0.5 * (D + D.T)
    full = gpu_lib.grad_contract(S2, b2, D)
    sym2 = gpu_lib.grad_contract(S2, b2, D, symmetric=True)
    scale = np.abs(full[0]).max()
    print(f"complete pair list: folded vs unfolded arep gradient max abs {np.abs(sym2[0] - full[0]).max():.2e} "
          f"(max |g| {scale:.2e}); unfolded SO max {np.abs(full[1:]).max():.2e}")
    assert np.all(np.abs(full[1:]) <= 1e-10 * scale)
    assert np.all(sym2[1:] == 0.0)
    assert np.all(np.abs(sym2[0] - full[0]) <= 1e-10 * scale)


def _small_system(shift=None):
    """Two heavy atoms with the full GRPP (U_L, projectors l <= 2, SO l <= 2, outercore
    s,p) and one H; shells s..d of 4 primitives with exponents in [0.3, 8]."""
    rng = np.random.default_rng(21)
    xyz = np.array([[0.0, 0.0, 0.0], [0.3, -0.2, 2.4], [1.7, 0.9, 1.1]])
    if shift is not None:
        xyz = xyz.copy()
        xyz[shift[0], shift[1]] += shift[2]
    grpps = [synthetic._heavy_grpp(rng, l_proj=2, l_so=2, l_oc=1) for _ in range(2)]
    shells, shell_atom = [], []
    for i in range(3):
        for L in range(3 if i < 2 else 2):
            shells.append(synthetic._shell(rng, xyz[i], L, 4, amin=0.3, amax=8.0))
            shell_atom.append(i)
    centres = [(xyz[0].copy(), 0), (xyz[1].copy(), 1)]
    return System(shells, grpps, centres, synthetic.CART_ORDER_TURBOMOLE, np.array(shell_atom, np.int32),
                  np.array([0, 1], np.int32), xyz)


def _energy(lib, S, D):
    b = S.batch()
    outs = lib.full_grpp_batch(b)
    return np.array([np.sum(D * S.assemble(b, outs[m])) for m in range(4)])


def test_gradient_contract_finite_differences(gpu_lib):
    S = _small_system()
    D = synthetic.config3_density(S, seed=5)
    g = gpu_lib.grad_contract(S, S.batch(), D)
    h = 1e-4
    fd = np.zeros_like(g)
    for at in range(3):
        for k in range(3):
            ep = _energy(gpu_lib, _small_system((at, k, h)), D)
            em = _energy(gpu_lib, _small_system((at, k, -h)), D)
            fd[:, at, k] = (ep - em) / (2 * h)
    err = np.abs(fd - g)
    scale = np.abs(g).max(axis=(1, 2), keepdims=True)
    print("finite differences: max |fd - g| per matrix", err.max(axis=(1, 2)), "max |g|", scale.ravel())
    assert np.all(err <= 1e-6 * scale + 1e-8)
    # translational invariance: the atom gradients sum to zero
    assert np.all(np.abs(g.sum(axis=1)) <= 1e-9 * scale[:, 0] + 1e-12)
