"""Serving: requests arriving while others run are admitted into the same batch as memory
frees up, and each request's result is bit-identical to solving it alone."""
import numpy as np
import pytest

from mfcm_b200 import SaintVenantSolver, start_new_step_forcing, RAIN_UNIFORM
from mfcm_b200.serving import FloodServer, make_requests
from tests.scenarios import same

pytestmark = pytest.mark.gpu


def _alone(req, variant, L=60.0, precision="f32"):
    """The request solved on its own, with the kernel variant batches use (FP32 arithmetic is
    contracted per kernel, so FP32 bits are reproducible per variant)."""
    s = SaintVenantSolver(req.nx, req.ny, req.dx, precision=precision, cn_target=0.5, step_duration=L,
                          rain_mode="physical")
    s.set_kernel_variant(variant)
    s.set_field("Z", req.z)
    z0 = np.zeros((req.ny, req.nx))
    for f in ("H", "U", "V"):
        s.set_field(f, z0)
    s.set_manning(req.n, req.n, 0.1, 0.3)
    t = 0.0
    while t < req.horizon - 1e-9:
        s.set_forcing(start_new_step_forcing(t, L, rain=req.rain, rain_kind=RAIN_UNIFORM, head=0.0,
                                             head_edges=req.head_edges))
        s.advance()
        t += L
    h = s.get_field("H")
    s.close()
    return h


def test_requests_overlap_and_match_their_solo_runs():
    reqs = make_requests(rate=50.0, count=12, seed=5, side=(32, 96), horizon=(120.0, 300.0))
    server = FloodServer(budget_bytes=2e9, precision="f32")
    summary = server.run(reqs, time_limit=300)
    variant = server.batch.kernel_variant()
    server.close()
    assert summary["completed"] == len(reqs)
    assert summary["max_concurrent"] >= 2          # work of different requests overlapped
    assert summary["p50_s"] <= summary["p99_s"]
    for r in reqs[:4]:
        assert same(r.result_h, _alone(r, variant)), f"request {r.rid} differs from its solo run"


def test_memory_budget_queues_requests():
    reqs = make_requests(rate=1e6, count=6, seed=7, side=(48, 64), horizon=(120.0, 120.0))  # all at once
    server = FloodServer(precision="f32")
    one = max(server.estimate_bytes(r) for r in reqs)
    server.budget = 2 * one                        # at most two catchments resident at once
    summary = server.run(reqs, time_limit=300)
    server.close()
    assert summary["completed"] == len(reqs)
    assert summary["max_concurrent"] <= 2
    # later arrivals had to wait for memory: admission after arrival
    assert any(r.admitted - r.arrival > 1e-3 for r in reqs[2:])


def test_persistent_serving_matches_solo_runs():
    """The server on the persistent batch kernel: requests still overlap, and FP64 results are
    the bits of each request solved alone."""
    reqs = make_requests(rate=50.0, count=8, seed=9, side=(32, 80), horizon=(120.0, 240.0))
    server = FloodServer(budget_bytes=2e9, precision="f64", persistent=True, steps_per_advance=1)
    summary = server.run(reqs, time_limit=300)
    server.close()
    assert summary["completed"] == len(reqs)
    assert summary["max_concurrent"] >= 2
    for r in reqs[:4]:
        assert same(r.result_h, _alone(r, 1, precision="f64")), f"request {r.rid} differs from its solo run"


def test_adopted_solver_matches_its_solo_run():
    """A solver filled on its own and adopted by a batch (the server's preparation path) runs
    as a member bit for bit like its solo run; precision mismatches are refused."""
    from mfcm_b200.batch import SaintVenantBatch
    req = make_requests(rate=1.0, count=1, seed=3, side=(48, 48), horizon=(120.0, 120.0))[0]
    b = SaintVenantBatch("f64")
    wrong = SaintVenantSolver(16, 16, 1.0, precision="f32")
    with pytest.raises(ValueError):
        b.adopt(wrong)
    wrong.close()
    s = SaintVenantSolver(req.nx, req.ny, req.dx, precision="f64", cn_target=0.5, step_duration=60.0,
                          rain_mode="physical")
    s.set_field("Z", req.z)
    s.set_manning(req.n, req.n, 0.1, 0.3)
    m = b.adopt(s)
    assert s._h is None and b.size()[0] == 1
    t = 0.0
    while t < req.horizon - 1e-9:
        b.advance_steps({m: [start_new_step_forcing(t, 60.0, rain=req.rain, rain_kind=RAIN_UNIFORM, head=0.0,
                                                    head_edges=req.head_edges)]})
        t += 60.0
    h = m.get_field("H")
    b.close()
    assert same(h, _alone(req, 1, precision="f64"))
