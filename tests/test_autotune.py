"""Assembly launch groups and the per-class autotuner of the assembly kernel's block size.

The block size (128, 256 or 512 threads) only changes which thread computes which V entry
and Cartesian pair; every value is formed by the same operations in the same order. So the
outputs of every block size, of the default rule and of the autotuned table are
bit-identical, and the autotuner's choice per class is the fastest of its timings.
"""
import numpy as np
import pytest

from tests.util import COMPS, load_fixture

pytestmark = pytest.mark.gpu


def _outputs(lib, batch, threads, mode=0):
    p = lib.plan(batch, mode, assembly_threads=threads)
    p.execute()
    out = p.outputs()
    p.close()
    return out


@pytest.mark.parametrize("name", ["config2", "tho", "config1"])
def test_block_sizes_give_identical_outputs(gpu_lib, name):
    batch, z = load_fixture(name)
    base = _outputs(gpu_lib, batch, 128)
    for threads in (256, 512, 0):
        out = _outputs(gpu_lib, batch, threads)
        for m, comp in enumerate(COMPS):
            assert np.array_equal(out[m], base[m]), (name, threads, comp)


def test_autotuner_table(gpu_lib):
    batch, z = load_fixture("config2")
    gpu_lib.autotune_reset()
    base = _outputs(gpu_lib, batch, 128)
    table = gpu_lib.autotune_assembly(batch, 0)
    la = batch.shell_L[batch.task_a]
    lb = batch.shell_L[batch.task_b]
    # every (la, lb) of the batch appears among the class keys ((la*16+lb)*16+L)*2+so
    keys = {(k // 2 // 16 // 16, (k // 2 // 16) % 16) for k in table}
    assert keys == set(zip(la.tolist(), lb.tolist()))
    assert sum(v[0] for v in table.values()) == len(batch.task_a)
    for key, (n, t128, t256, t512, choice) in table.items():
        assert n > 0 and min(t128, t256, t512) > 0
        assert choice == (128, 256, 512)[int(np.argmin([t128, t256, t512]))]
    out = _outputs(gpu_lib, batch, 0)
    for m in range(4):
        assert np.array_equal(out[m], base[m])
    gpu_lib.autotune_reset()


def test_invalid_block_size_is_rejected(gpu_lib):
    batch, z = load_fixture("h2o")
    with pytest.raises(RuntimeError):
        gpu_lib.plan(batch, 0, assembly_threads=96)
