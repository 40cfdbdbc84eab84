"""Time the unmodified reference's RK3 step on this machine's CPU cores.

Usage:  PYWRF_REFERENCE_ROOT=/path/to/PyWRF python tests/golden/time_reference_cpu.py [--threads N]

Runs the reference through tests/golden/refharness.py (its own solver loop,
float32, torch on the CPU with N threads, default all cores) on the
synthetic 240x240x41 workload (1 warm-up step, then 2 timed steps: the
difference of a 3-step and a 1-step solve) and the 64x64x41 workload (1
warm-up step, then 10 timed steps), and writes reference_cpu_timing.json
next to this script with seconds per step, steps/s, the thread count and the
CPU model.  The reference's Python source cannot run where the reference is
absent, so this record is what bench.py reports as the reference's own CPU
step; the per-run CPU baseline of bench.py is the oracle port timed on the
benchmark machine itself.
"""
from __future__ import annotations

import argparse
import json
import os
import platform
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

from pywrf_b200 import synthetic  # noqa: E402


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor() or "unknown"


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    a = ap.parse_args()
    import torch

    torch.set_num_threads(a.threads)
    import refharness

    out = {"threads": a.threads, "cpu": cpu_model(), "logical_cpus": os.cpu_count(), "dtype": "float32",
           "torch": torch.__version__, "workloads": {}}
    for config, (warm, timed) in ((1, (1, 2)), (0, (1, 10))):
        spec = synthetic.spec_for_config(config)
        g = synthetic.grid_for(spec)
        inputs, bdy = synthetic.build(spec)
        t0 = time.perf_counter()
        refharness.run_reference(g, inputs, bdy, warm, dtype="float32")
        t1 = time.perf_counter()
        refharness.run_reference(g, inputs, bdy, warm + timed, dtype="float32")
        t2 = time.perf_counter()
        sec = ((t2 - t1) - (t1 - t0)) / timed
        out["workloads"][f"{g.nx}x{g.ny}x{g.nz}"] = {"seconds_per_step": sec, "steps_per_s": 1.0 / sec,
                                                     "timed_steps": timed, "warmup_steps": warm}
        print(config, sec, flush=True)
    out["solver_sha256"] = refharness.SOLVER_SHA256
    with open(os.path.join(HERE, "reference_cpu_timing.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
