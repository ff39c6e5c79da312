"""Checkpoint and restart of the CUDA solver: a solve resumed from a checkpoint continues bit
for bit, in FP64 and in FP32 with FP64 tile datums, with the infiltration capacity carried."""
import numpy as np
import pytest

from mfcm_b200 import SaintVenantSolver, outputs, synth, solve, EDGE_XMAX
from tests.scenarios import same, rain_series

pytestmark = pytest.mark.gpu


def _solver(precision, nx, ny, dx, z, infil):
    s = SaintVenantSolver(nx, ny, dx, precision=precision, cn_target=0.5, step_duration=20.0, rain_mode="physical")
    s.set_field("Z", z)
    s.set_manning(0.03, 0.03, 0.1, 0.3)
    if infil:
        s.set_field("INFIL_RATE", np.full((ny, nx), 5e-6))
        s.set_field("INFIL_CAP", np.full((ny, nx), 4e-4))
    return s


@pytest.mark.parametrize("precision", ["f64", "f32_datum64"])
def test_checkpoint_resumes_bit_for_bit(tmp_path, precision):
    nx, ny, dx = 70, 41, 2.0
    z = 120.0 + synth.plane_with_gaussians(nx, ny, dx, seed=6)
    rain = rain_series(60 * synth.MM_PER_H, stop=1e4)
    a = _solver(precision, nx, ny, dx, z, True)
    a.set_field("H", np.full((ny, nx), 2e-3))
    solve(a, 0.0, 40.0, rain=rain, head=0.0, head_edges=EDGE_XMAX)
    ck = str(tmp_path / "ck.bin")
    outputs.save_checkpoint(a, ck, t=40.0, infiltration=True)
    solve(a, 40.0, 100.0, rain=rain, head=0.0, head_edges=EDGE_XMAX)
    b = _solver(precision, nx, ny, dx, z, True)
    outputs.load_checkpoint(b, ck)
    solve(b, 40.0, 100.0, rain=rain, head=0.0, head_edges=EDGE_XMAX)
    for f in ("H", "U", "V", "INFIL_CAP"):
        assert same(a.get_field(f), b.get_field(f)), f
    assert a.stats() == b.stats()
    a.close()
    b.close()


def test_measures_and_timed_outputs_follow_the_solve(tmp_path):
    nx, ny, dx = 48, 32, 5.0
    z = synth.plane_with_gaussians(nx, ny, dx, seed=1)
    s = _solver("f64", nx, ny, dx, z, False)
    s.set_field("H", np.zeros((ny, nx)))
    vol = outputs.VolumeMeasure()
    pt = outputs.DepthPointMeasure((100.0, 60.0), nx, ny, dx, dx)
    out = outputs.MultiFieldOutput(str(tmp_path / "h"), ["h", "stage"], every=40.0)

    def on_step(t, solver):
        out.timed_output(t, solver)
        vol.update(t, solver)
        pt.update(t, solver)

    solve(s, 0.0, 100.0, rain=rain_series(50 * synth.MM_PER_H), head=0.0, head_edges=EDGE_XMAX, on_step=on_step)
    assert len(out.written) == 3                         # t = 0, 40, 80 (steps start at 0, 20, ..., 80)
    assert [p[0] for p in vol.points] == [0.0, 20.0, 40.0, 60.0, 80.0, 100.0]   # step starts and the end
    assert vol.points[-1][1] > vol.points[1][1] > 0.0    # rain accumulates
    vol.write(str(tmp_path / "volume.csv"))
    lines = open(tmp_path / "volume.csv").read().splitlines()
    assert lines[0] == '"ID", "volume", ' and len(lines) == 7
    s.close()
