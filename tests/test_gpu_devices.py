"""Device-level behaviour of the library: FP64 solvers on two GPUs in one process (the shared-
memory opt-in of the tiled stage kernel is a per-device attribute), and device memory that stays
flat when the roughness fields are set again and again."""
import numpy as np
import pytest
import torch

from mfcm_b200 import SaintVenantSolver
from tests.scenarios import setup, wet_dry_state

pytestmark = pytest.mark.gpu


def _run(device, variant, nx=96, ny=70, dx=2.0, steps=12):
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=5)
    s = SaintVenantSolver(nx, ny, dx, cn_target=0.5, device=device)
    setup(s, z, h, u, v)
    s.set_kernel_variant(variant)
    s.run_timesteps(steps, begin=True)
    out = [s.get_field(f) for f in ("H", "U", "V")]
    s.close()
    return out


@pytest.mark.skipif(torch.cuda.device_count() < 2, reason="needs two GPUs")
@pytest.mark.parametrize("variant", [0, 1, 8, 11])
def test_fp64_solvers_on_two_devices_in_one_process(variant):
    """The tiled 32x8 FP64 kernel needs more than 48 KB of shared memory, an opt-in set per
    device: a solver on the second GPU after one on the first must launch and agree bit for
    bit, and so must the first GPU again afterwards."""
    a = _run(0, variant)
    b = _run(1, variant)
    c = _run(0, variant)
    for x, y, w in zip(a, b, c):
        assert np.array_equal(x, y, equal_nan=True) and np.array_equal(x, w, equal_nan=True)


def test_roughness_fields_set_repeatedly_keep_device_memory_flat():
    """n_deep shares n_shallow's array while the two are equal and moves to an array of its own
    when they part; alternating the two must reuse that one array, not allocate a new one each
    time (8 MB per allocation at 1024 x 1024 in FP64)."""
    nx = ny = 1024
    s = SaintVenantSolver(nx, ny, 2.0, device=0)
    rng = np.random.default_rng(1)
    a = rng.uniform(0.02, 0.05, (ny, nx))
    b = rng.uniform(0.03, 0.08, (ny, nx))

    def cycle():
        s.set_field("N_SHALLOW", a)
        s.set_field("N_DEEP", a)   # equal: shares n_shallow's array
        s.set_field("N_SHALLOW", b)  # parts: n_deep keeps a in its own array
        s.set_field("N_DEEP", b)   # equal again
        s.set_field("N_DEEP", a)   # parts again
        torch.cuda.synchronize(0)

    cycle()
    free0 = torch.cuda.mem_get_info(0)[0]
    for _ in range(16):
        cycle()
    free1 = torch.cuda.mem_get_info(0)[0]
    np.testing.assert_array_equal(s.get_field("N_DEEP"), a)
    np.testing.assert_array_equal(s.get_field("N_SHALLOW"), b)
    s.close()
    assert free0 - free1 < 32 << 20, f"device memory fell by {(free0 - free1) / 2**20:.1f} MiB over 16 cycles"
