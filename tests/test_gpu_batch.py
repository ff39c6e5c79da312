"""Batches: uneven catchments advanced in shared launches give, member by member, the same
bits as running each catchment alone (and as the oracle), including after members are
removed and added between steps."""
import numpy as np
import pytest

from mfcm_b200 import SaintVenantSolver, SvError, synth, start_new_step_forcing, RAIN_UNIFORM, EDGE_XMAX, EDGE_YMIN
from mfcm_b200._abi import SV_E_NONFINITE, SV_E_LIMIT
from mfcm_b200.batch import SaintVenantBatch
from oracle.sv_oracle_py import OracleSolver
from tests.scenarios import setup, rain_series, same

pytestmark = pytest.mark.gpu

CASES = [  # nx, ny, dx, rain mm/h, head edges, seed
    (64, 40, 2.0, 60.0, EDGE_XMAX, 1),
    (37, 91, 5.0, 30.0, EDGE_YMIN, 2),
    (128, 17, 1.0, 90.0, EDGE_XMAX | EDGE_YMIN, 3),
]


def _init(b, nx, ny, dx, seed):
    z = synth.plane_with_gaussians(nx, ny, dx, slope=0.01, seed=seed)
    setup(b, z, np.full((ny, nx), 2e-3), np.zeros((ny, nx)), np.zeros((ny, nx)))


def _forcing(t, L, rate, edges):
    return start_new_step_forcing(t, L, rain=rain_series(rate * synth.MM_PER_H, stop=40.0), rain_kind=RAIN_UNIFORM,
                                  head=0.0, head_edges=edges)


def _run_alone(cls, case, steps, L=20.0):
    nx, ny, dx, rate, edges, seed = case
    s = cls(nx, ny, dx, cn_target=0.5, step_duration=L, rain_mode="physical")
    _init(s, nx, ny, dx, seed)
    for i in range(steps):
        s.set_forcing(_forcing(i * L, L, rate, edges))
        s.advance()
    return [s.get_field(f) for f in ("H", "U", "V")], s.stats()


def test_batch_members_match_solo_runs_and_oracle():
    L, steps = 20.0, 3
    batch = SaintVenantBatch("f64")
    mem = []
    for c in CASES:
        m = batch.add(c[0], c[1], c[2], cn_target=0.5, step_duration=L, rain_mode="physical")
        _init(m, c[0], c[1], c[2], c[5])
        mem.append(m)
    for i in range(steps):
        for m, c in zip(mem, CASES):
            m.set_forcing(_forcing(i * L, L, c[3], c[4]))
        batch.advance()
    for m, c in zip(mem, CASES):
        solo, _ = _run_alone(SaintVenantSolver, c, steps, L)
        orc, so = _run_alone(OracleSolver, c, steps, L)
        for k, f in enumerate(("H", "U", "V")):
            got = m.get_field(f)
            assert same(got, solo[k]), f"{c}: {f} differs from the solo run"
            assert same(got, orc[k]), f"{c}: {f} differs from the oracle"
        assert abs(m.stats()["volume"] - so["volume"]) <= 1e-12 * so["volume"]
    batch.close()


def test_members_join_and_leave_between_steps():
    L = 20.0
    batch = SaintVenantBatch("f64")
    a = batch.add(*CASES[0][:3], cn_target=0.5, step_duration=L, rain_mode="physical")
    _init(a, CASES[0][0], CASES[0][1], CASES[0][2], CASES[0][5])
    b = batch.add(*CASES[1][:3], cn_target=0.5, step_duration=L, rain_mode="physical")
    _init(b, CASES[1][0], CASES[1][1], CASES[1][2], CASES[1][5])
    for m, c in ((a, CASES[0]), (b, CASES[1])):
        m.set_forcing(_forcing(0.0, L, c[3], c[4]))
    batch.advance()
    batch.remove(b)
    c = batch.add(*CASES[2][:3], cn_target=0.5, step_duration=L, rain_mode="physical")
    _init(c, CASES[2][0], CASES[2][1], CASES[2][2], CASES[2][5])
    a.set_forcing(_forcing(L, L, CASES[0][3], CASES[0][4]))
    c.set_forcing(_forcing(0.0, L, CASES[2][3], CASES[2][4]))
    batch.advance()
    assert batch.size()[0] == 2
    solo_a, _ = _run_alone(SaintVenantSolver, CASES[0], 2, L)
    solo_c, _ = _run_alone(SaintVenantSolver, CASES[2], 1, L)
    for k, f in enumerate(("H", "U", "V")):
        assert same(a.get_field(f), solo_a[k])
        assert same(c.get_field(f), solo_c[k])
    batch.close()


def test_fp32_batch_close_to_fp64():
    L, steps = 20.0, 2
    b32 = SaintVenantBatch("f32")
    m = b32.add(*CASES[0][:3], cn_target=0.5, step_duration=L, rain_mode="physical")
    _init(m, CASES[0][0], CASES[0][1], CASES[0][2], CASES[0][5])
    for i in range(steps):
        m.set_forcing(_forcing(i * L, L, CASES[0][3], CASES[0][4]))
        b32.advance()
    ref, _ = _run_alone(OracleSolver, CASES[0], steps, L)
    assert np.max(np.abs(m.get_field("H") - ref[0])) <= 1e-3
    b32.close()


def test_a_failing_member_does_not_stop_the_others():
    """One member's time turns NaN (its dt is set to NaN): it alone is reported, and the other
    members complete the same steps with the bits of their solo runs."""
    L, steps = 20.0, 2
    batch = SaintVenantBatch("f64")
    mem = []
    for c in CASES:
        m = batch.add(c[0], c[1], c[2], cn_target=0.5, step_duration=L, rain_mode="physical")
        _init(m, c[0], c[1], c[2], c[5])
        mem.append(m)
    mem[1].set_dt(float("nan"))
    for i in range(steps):
        for m, c in zip(mem, CASES):
            m.set_forcing(_forcing(i * L, L, c[3], c[4]))
        st = batch.advance(raise_on_error=False)
        assert [st[m.slot]["status"] for m in mem] == [0, SV_E_NONFINITE, 0]
    for j in (0, 2):
        solo, _ = _run_alone(SaintVenantSolver, CASES[j], steps, L)
        for k, f in enumerate(("H", "U", "V")):
            assert same(mem[j].get_field(f), solo[k]), f"{CASES[j]}: {f} differs from the solo run"
    with pytest.raises(SvError) as e:
        batch.advance()
    assert e.value.code == SV_E_NONFINITE
    batch.close()


def test_step_limit_leaves_members_part_way():
    """With a cap of 2 timesteps per step every member (each needs more) stops after exactly
    2 timesteps with status SV_E_LIMIT; by default advance raises SV_E_LIMIT."""
    L = 20.0
    batch = SaintVenantBatch("f64")
    mem = []
    for c in CASES:
        m = batch.add(c[0], c[1], c[2], cn_target=0.5, step_duration=L, rain_mode="physical")
        _init(m, c[0], c[1], c[2], c[5])
        m.set_forcing(_forcing(0.0, L, c[3], c[4]))
        mem.append(m)
    batch.set_step_limit(2)
    st = batch.advance(raise_on_error=False)
    for m in mem:
        assert st[m.slot]["status"] == SV_E_LIMIT
        assert st[m.slot]["accepted"] + st[m.slot]["repeated"] == 2
    with pytest.raises(SvError) as e:
        batch.advance()
    assert e.value.code == SV_E_LIMIT
    batch.set_step_limit(0)
    st = batch.advance()
    assert all(st[m.slot]["status"] == 0 for m in mem)
    batch.close()


def test_queued_steps_equal_single_steps():
    """advance_steps runs each member's steps back to back at its own pace; the results are
    bit-identical to one advance() per step, and members with fewer steps queued stop early."""
    L, steps = 20.0, 4
    runs = []
    for queued in (False, True):
        batch = SaintVenantBatch("f64")
        mem = []
        for c in CASES:
            m = batch.add(c[0], c[1], c[2], cn_target=0.5, step_duration=L, rain_mode="physical")
            _init(m, c[0], c[1], c[2], c[5])
            mem.append(m)
        nsteps = [steps, steps - 1, steps]
        per_step = []
        if queued:
            res = batch.advance_steps({m: [_forcing(i * L, L, c[3], c[4]) for i in range(ns)]
                                       for m, c, ns in zip(mem, CASES, nsteps)})
            for m, ns in zip(mem, nsteps):
                assert res[m.slot]["status"] == 0 and len(res[m.slot]["steps"]) == ns
            per_step = [[(s["accepted"], s["repeated"], s["volume"]) for s in res[m.slot]["steps"]] for m in mem]
        else:
            per_step = [[] for _ in mem]
            for i in range(steps):
                for j, (m, c) in enumerate(zip(mem, CASES)):
                    if i == nsteps[j]:
                        batch.remove(m)  # its steps are over: it leaves the batch
                    elif i < nsteps[j]:
                        m.set_forcing(_forcing(i * L, L, c[3], c[4]))
                st = batch.advance()
                for j, m in enumerate(mem):
                    if i < nsteps[j]:
                        s = st[m.slot]
                        per_step[j].append((s["accepted"], s["repeated"], s["volume"]))
        fields = [[m.get_field(f) for f in ("H", "U", "V")] if m.slot in batch.members else None for m in mem]
        runs.append((per_step, fields))
        batch.close()
    (ps_a, f_a), (ps_b, f_b) = runs
    assert ps_a == ps_b
    for j in (0, 2):
        for k in range(3):
            assert same(f_a[j][k], f_b[j][k])
    solo, _ = _run_alone(SaintVenantSolver, CASES[1], steps - 1, L)
    for k in range(3):
        assert same(f_b[1][k], solo[k])


def test_queued_steps_isolate_a_failing_member():
    L = 20.0
    batch = SaintVenantBatch("f64")
    mem = []
    for c in CASES:
        m = batch.add(c[0], c[1], c[2], cn_target=0.5, step_duration=L, rain_mode="physical")
        _init(m, c[0], c[1], c[2], c[5])
        mem.append(m)
    mem[2].set_dt(float("nan"))
    res = batch.advance_steps({m: [_forcing(i * L, L, c[3], c[4]) for i in range(3)] for m, c in zip(mem, CASES)},
                              raise_on_error=False)
    assert [res[m.slot]["status"] for m in mem] == [0, 0, SV_E_NONFINITE]
    assert len(res[mem[0].slot]["steps"]) == 3 and len(res[mem[2].slot]["steps"]) == 1
    solo, _ = _run_alone(SaintVenantSolver, CASES[0], 3, L)
    assert same(mem[0].get_field("H"), solo[0])
    batch.close()


def _persistent_batch(precision, cases, L, spin_limit=0, max_seconds=0.0):
    batch = SaintVenantBatch(precision)
    batch.set_persistent(True, spin_limit, max_seconds)
    mem = []
    for c in cases:
        m = batch.add(c[0], c[1], c[2], cn_target=0.5, step_duration=L, rain_mode="physical")
        _init(m, c[0], c[1], c[2], c[5])
        mem.append(m)
    return batch, mem


def test_persistent_batch_matches_solo_runs():
    """One cooperative launch per advance: every member advances through its queued steps at
    its own dt, and FP64 members keep the bits of their solo runs."""
    L, steps = 20.0, 3
    batch, mem = _persistent_batch("f64", CASES, L)
    res = batch.advance_steps({m: [_forcing(i * L, L, c[3], c[4]) for i in range(steps)] for m, c in zip(mem, CASES)})
    for m, c in zip(mem, CASES):
        assert res[m.slot]["status"] == 0 and len(res[m.slot]["steps"]) == steps
        solo, so = _run_alone(SaintVenantSolver, c, steps, L)
        for k, f in enumerate(("H", "U", "V")):
            assert same(m.get_field(f), solo[k]), f"{c}: {f} differs from the solo run"
        st = res[m.slot]["steps"][-1]
        assert abs(st["volume"] - so["volume"]) <= 1e-12 * so["volume"]
        assert (m.stats()["accepted"], m.stats()["repeated"]) == (so["accepted"], so["repeated"])
    # the next advance carries on from there, one step at a time
    for m, c in zip(mem, CASES):
        m.set_forcing(_forcing(steps * L, L, c[3], c[4]))
    batch.advance()
    for m, c in zip(mem, CASES):
        solo, _ = _run_alone(SaintVenantSolver, c, steps + 1, L)
        assert same(m.get_field("H"), solo[0])
    batch.close()


def test_persistent_fp32_batch_close_to_fp64():
    L, steps = 20.0, 2
    batch, mem = _persistent_batch("f32_datum64", CASES, L)
    batch.advance_steps({m: [_forcing(i * L, L, c[3], c[4]) for i in range(steps)] for m, c in zip(mem, CASES)})
    for m, c in zip(mem, CASES):
        ref, so = _run_alone(OracleSolver, c, steps, L)
        assert np.max(np.abs(m.get_field("H") - ref[0])) <= 1e-3
        st = m.stats()
        v0 = 2e-3 * c[0] * c[1] * c[2] * c[2]
        closure = st["volume"] - (v0 + st["rain_in"] - st["outflow"] + st["wall_in"])
        assert abs(closure) <= 1e-6 * st["volume"], (closure, st)
    batch.close()


def test_persistent_batch_isolates_a_failing_member():
    L = 20.0
    batch, mem = _persistent_batch("f64", CASES, L)
    mem[1].set_dt(float("nan"))
    res = batch.advance_steps({m: [_forcing(i * L, L, c[3], c[4]) for i in range(2)] for m, c in zip(mem, CASES)},
                              raise_on_error=False)
    assert [res[m.slot]["status"] for m in mem] == [0, SV_E_NONFINITE, 0]
    solo, _ = _run_alone(SaintVenantSolver, CASES[2], 2, L)
    assert same(mem[2].get_field("H"), solo[0])
    batch.close()


@pytest.mark.parametrize("bound", ["polls", "wall_clock"])
def test_persistent_wait_bound_gives_up_with_a_status(bound):
    """Every wait of the persistent kernel is bounded. With a bound of one poll without progress,
    or of one microsecond of wall clock, the launch gives up and the call returns SV_E_TIMEOUT.
    The device stays usable, and each member keeps the state of its last completed timestep."""
    from mfcm_b200._abi import SV_E_TIMEOUT
    L = 20.0
    # one member: while its single warp runs a finalize no other item completes anywhere
    cases = CASES[:1] if bound == "polls" else CASES
    kw = dict(spin_limit=1) if bound == "polls" else dict(max_seconds=1e-6)
    batch, mem = _persistent_batch("f64", cases, L, **kw)
    for m, c in zip(mem, cases):
        m.set_forcing(_forcing(0.0, L, c[3], c[4]))
    with pytest.raises(SvError) as e:
        batch.advance()
    assert e.value.code == SV_E_TIMEOUT
    for m in mem:  # the state is still finite
        assert np.isfinite(m.get_field("H")).all()
    batch.close()
    # the device keeps working: a fresh persistent batch with the default bound completes
    batch, mem = _persistent_batch("f64", CASES[:1], L)
    mem[0].set_forcing(_forcing(0.0, L, CASES[0][3], CASES[0][4]))
    batch.advance()
    solo, _ = _run_alone(SaintVenantSolver, CASES[0], 1, L)
    assert same(mem[0].get_field("H"), solo[0])
    batch.close()
