"""The CPU oracle under AddressSanitizer and UndefinedBehaviorSanitizer (CPU).

oracle/build.py builds oracle/_build/sv_oracle_san: the oracle's C-ABI with a driver
(oracle/sanitize_main.cpp) that calls every entry point on single cells, single rows and
columns, ragged grids and coded-out bed cells, in both precisions, with every tableau, rain
kind, head kind, eddy-viscosity mode and source-term order. Any out-of-bounds access, leak,
use after free or undefined arithmetic (signed overflow, invalid shift, misaligned load) ends
the run with the sanitizer's report and a non-zero status.
"""
import os
import shutil
import subprocess

import pytest

from oracle import build


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_oracle_clean_under_asan_and_ubsan():
    exe = build.build_sanitized()
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, (r.stdout + r.stderr)[-4000:]
    assert "sanitized run ok" in r.stdout
    assert "runtime error" not in r.stderr and "ERROR: AddressSanitizer" not in r.stderr
