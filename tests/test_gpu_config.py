"""A solve driven by a configuration deck on the GPU: FP64 equals the oracle driven by the same
deck bit for bit; the FP32 datum solver stays within a millimetre."""
import os

import numpy as np
import pytest

from mfcm_b200 import config, SaintVenantSolver
from oracle.sv_oracle_py import OracleSolver
from tests.scenarios import first_diff

pytestmark = pytest.mark.gpu

DECK = os.path.join(os.path.dirname(os.path.abspath(__file__)), "decks", "catchment.mf")


def _run(cls, **kw):
    m = config.load(DECK)
    s = m.build(cls, **kw)
    m.solve(s)
    return {k: s.get_field(k) for k in ("H", "U", "V")}, s.stats()


def test_deck_solve_equals_the_oracle():
    g, gs = _run(SaintVenantSolver)
    o, os_ = _run(OracleSolver)
    for k in ("H", "U", "V"):
        d = first_diff(g[k], o[k])
        assert d is None, f"{k}: first mismatch at {d[0]}: gpu {d[1]!r} oracle {d[2]!r}"
    assert gs["accepted"] == os_["accepted"]
    # the volume is a diagnostic sum: the GPU adds 32 x 8 tile partials in a tree, the oracle
    # sums sequentially with compensation, so the two may differ in the last bit
    assert abs(gs["volume"] - os_["volume"]) <= 1e-13 * os_["volume"]


def test_deck_solve_in_fp32_with_fp64_datums():
    g, _ = _run(SaintVenantSolver, precision="f32_datum64")
    o, _ = _run(OracleSolver)
    assert np.max(np.abs(g["H"] - o["H"])) <= 1e-3
