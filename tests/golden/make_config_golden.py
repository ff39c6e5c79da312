"""Regenerate tests/golden/configs.json: the oracle's FP64 runs of the benchmark configurations
at their full sizes, recorded as a digest per output time.

At these sizes the state is too large to commit (a 256 x 256 run for an hour, a 1024 x 1024
window of the 4096 x 4096 catchment, the 8192 x 1024 dam break), and the oracle needs minutes
per run. Each output therefore records: the accepted and repeated timestep counts, the FP64
volume, the maximum depth, and a SHA-256 digest of the h, u and v fields (little-endian FP64,
with -0.0 folded into +0.0 and every NaN made the canonical quiet NaN: the CUDA path may differ
from the oracle in the sign of an exact zero, which never changes a value). A GPU run that
reproduces every digest is bit for bit the oracle's run. The scenarios are defined in
tests/config_scenarios.py, shared with the GPU tests.

    python tests/golden/make_config_golden.py [name ...]
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.sv_oracle_py import OracleSolver  # noqa: E402
from tests.config_scenarios import SCENARIOS, run  # noqa: E402

OUT = os.path.join(HERE, "configs.json")


def main(names):
    for name in names or list(SCENARIOS):
        t0 = time.time()
        rec = run(name, lambda *a, **k: OracleSolver(*a, openmp=True, **k))
        data = json.load(open(OUT)) if os.path.exists(OUT) else {}
        data[name] = rec
        with open(OUT, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        print(f"{name}: {len(rec['outputs'])} outputs, {rec['outputs'][-1]['accepted']} accepted timesteps, "
              f"{time.time() - t0:.0f} s", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
