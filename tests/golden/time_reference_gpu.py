"""Time the unmodified reference's RK3 step on a CUDA device.

Usage:  PYWRF_REFERENCE_ROOT=/path/to/PyWRF python tests/golden/time_reference_gpu.py [--device cuda:0]

Runs the reference through tests/golden/refharness.py (its own solver loop
and kernel modules, float32, torch with the default device set to the
given CUDA device) on the synthetic 240x240x41 workload: a solve of W steps
and a solve of W + K steps, each closed by torch.cuda.synchronize(), so that
their difference is K steps of the reference's stepping with its own
host-side control flow and synchronisations (the harness stubs only its
debug prints and debug arg-max blocks, which would add host work).  Writes
reference_gpu_timing.json next to this script with seconds per step,
steps/s and the device name.  The reference is Python source that is not
present where bench.py runs, so this record is what bench.py reports as the
reference's own GPU step (``reference_gpu``), named as recorded, not
measured in that run.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

from pywrf_b200 import synthetic  # noqa: E402


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--device", default="cuda:0")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--steps", type=int, default=10)
    a = ap.parse_args()
    import torch

    import refharness

    if not torch.cuda.is_available():
        raise SystemExit("a CUDA device is required")
    spec = synthetic.spec_for_config(1)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)

    def solve(n):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        refharness.run_reference(g, inputs, bdy, n, dtype="float32", device=a.device)
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    solve(1)  # first-touch: module loads, allocator, kernel caches
    t_w = solve(a.warmup)
    t_wk = solve(a.warmup + a.steps)
    sec = (t_wk - t_w) / a.steps
    out = {"device": torch.cuda.get_device_name(torch.device(a.device)), "dtype": "float32",
           "torch": torch.__version__, "solver_sha256": refharness.SOLVER_SHA256,
           "workloads": {f"{g.nx}x{g.ny}x{g.nz}": {"seconds_per_step": sec, "steps_per_s": 1.0 / sec,
                                                   "timed_steps": a.steps, "warmup_steps": a.warmup}}}
    print(json.dumps(out), flush=True)
    with open(os.path.join(HERE, "reference_gpu_timing.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
