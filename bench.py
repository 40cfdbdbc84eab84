"""Benchmark: ARW RK3 steps/s on the 240x240x41 synthetic moist workload.

``python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]``

One step = one complete ``wrf_rk3_step`` (three RK stages, 1+2+4 acoustic
substeps, moisture transport, WSM6, boundary updates) over the 240x240x41
state built by :mod:`pywrf_b200.synthetic` (the 240x240x41 / dt 45 s / 80-step
workload with seeded boundary tendencies), replayed from one captured CUDA
graph.  The timed region is bracketed by barrier + synchronize; the device
time is measured with CUDA events on the replay stream and the maximum over
ranks is reported.  Multi-GPU runs are independent replicas (different seeds,
no data-path collective): the step is column-local but its lateral boundary
is one domain, so ``value`` = N * K / max-rank time ("weak" scaling).

Extra keys of the JSON line:
  roofline      the dominant kernel's algorithmic bytes / CUDA-event duration
                against the measured HBM copy bandwidth
  phases        per-phase device time of one eager step (probe events)
  e2e           the same metric through the public API with host buffers:
                pinned H2D of the prognostic state, one step, D2H of it back
  cpu_baseline  the numpy oracle (a restatement of the reference's CPU path)
                timed on this host for one step of the same workload
  clocks        SM clock samples taken during the timed region
``--impl reference`` times that CPU path alone (rank 0; other ranks exit).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RK3 steps/s @240x240x41"
UNIT = "steps/s"
WORKLOAD = "240x240x41 synthetic moist ARW, plain WSM6, dt=45 s, 4 acoustic substeps, seeded bdy tendencies"
FALLBACK_HBM_GBS = 6650.0

# prognostic fields a host-driven caller moves in and out each step (e2e)
E2E_FIELDS = ("u", "v", "w", "t", "ph", "mu", "p", "al", "moist")

# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per launch of the
# dominant kernel from one ncu --set full capture of this workload
# (profiles/k_acoustic_col_and_advection_240x240x41.md): the stage-1 launch,
# 202.0 MB read + 72.9 MB written, against 321 MB algorithmic for that launch
NCU_TRAFFIC = {"k_acoustic_col": 274.835456e6}


def parse():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--config", type=int, default=1, help="synthetic workload id (1: 240x240x41)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--phase-steps", type=int, default=3, help="eager steps timed per phase for the roofline")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi samples of one GPU's clocks while the timed region runs."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 8:
                    continue
                try:
                    sm.append(float(parts[0]))
                    smax = float(parts[1])
                except ValueError:
                    continue
                for nm, v in zip(names, parts[4:8]):
                    if v.lower() == "active":
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------------- CPU arm

def cpu_reference_step_time(config: int, nsteps: int, warmup: int):
    """Seconds per step of the numpy oracle (the reference's algorithm on
    the host) on the same workload, plus the sample description."""
    from oracle.model import OracleModel   # the CPU baseline leg only
    from pywrf_b200 import synthetic
    spec = synthetic.spec_for_config(config)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    m = OracleModel(g, inputs, bdy, np.float32)
    for _ in range(warmup):
        m.step(m.step_count + 1)
    t0 = time.perf_counter()
    for _ in range(nsteps):
        m.step(m.step_count + 1)
    dt = (time.perf_counter() - t0) / nsteps
    return dt, f"{nsteps} RK3 step(s) of the {g.nx}x{g.ny}x{g.nz} workload, numpy fp32 oracle, 1 thread"


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # bounded sample: each oracle step of this workload is tens of seconds of
    # CPU work, so at most 1 warm-up and 2 timed steps are run
    k, w = max(1, min(a.steps, 2)), min(a.warmup, 1)
    sec, sample = cpu_reference_step_time(a.config, k, w)
    v = 1.0 / sec
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": k, "warmup": w,
            "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "parallelism": "replicas"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------- GPU arm

# compulsory 3-D field passes of k_acoustic_col (one acoustic substep): reads
# u v u_save v_save t t_tend t_save ww ww1 ph_save phb ph a alpha gamma
# ph_tend w c2a alt cqw rw_tend w_save pm1 (23) + ru_m rv_m ww_m after the
# first substep of a stage (3); writes t t_2save ww ph w ru_m rv_m ww_m al p
# pm1 (11).  A step has 3 first substeps and 4 later ones.
COL_PASSES_PER_STEP = 3 * (23 + 11) + 4 * (26 + 11)
COL_LAUNCHES_PER_STEP = 7


def algorithmic_bytes(g):
    """Compulsory HBM bytes per launch of the dominant kernel: fp32 3-D
    passes x 4 B x points of the allocation."""
    n3 = g.nx * g.ny * g.nz
    return {"k_acoustic_col": COL_PASSES_PER_STEP / COL_LAUNCHES_PER_STEP * 4 * n3}


def run_ours(a):
    import torch
    import torch.distributed as dist
    from pywrf_b200 import _native as N
    from pywrf_b200 import synthetic
    from pywrf_b200.solver import Integrator
    from pywrf_b200.state import DeviceState

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != a.gpus:
        raise SystemExit(f"--gpus {a.gpus} but WORLD_SIZE={world}")
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    from pywrf_b200.replicas import barrier, job_rate, max_over_ranks

    spec = synthetic.spec_for_config(a.config, seed=rank)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    st = DeviceState.from_inputs(g, inputs, bdy, device=f"cuda:{local}")
    it = Integrator(st)

    # one eager step: launch count, then the graph
    it.step()
    launches = N.lib().wrf_last_launch_count()
    it.capture()
    for _ in range(a.warmup):
        it.replay()
    torch.cuda.synchronize()

    stream = it._graph_stream
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as cs:
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(a.steps):
                it._graph.replay()
            e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms)
    value = job_rate(a.steps, ms_max, world)
    clocks = cs.summary()

    # per-phase device time of eager steps (probe events on the launch stream)
    phase_ms: dict[str, float] = {}
    for _ in range(a.phase_steps):
        evs = []
        cur = torch.cuda.current_stream()
        start = torch.cuda.Event(enable_timing=True)
        start.record(cur)

        def probe(name):
            e = torch.cuda.Event(enable_timing=True)
            e.record(cur)
            evs.append((name, e))
        it.step(probe)
        torch.cuda.synchronize()
        prev = start
        for name, e in evs:
            key = name.split(".", 1)[1] if name.startswith("s") and "." in name else name
            if key.startswith("sub"):
                key = "sub." + key.split(".")[1] if key.count(".") else "sub.bc"
            phase_ms[key] = phase_ms.get(key, 0.0) + prev.elapsed_time(e) / a.phase_steps
            prev = e
    nan = it.status()["nan_p"]

    # roofline of the dominant kernel, k_acoustic_col (the "sub.col" phases:
    # that kernel alone, 7 launches per step)
    hbm, peak_kind = peaks()
    ab = algorithmic_bytes(g)
    k_ms = phase_ms.get("sub.col", float("nan")) / COL_LAUNCHES_PER_STEP
    achieved = ab["k_acoustic_col"] / (k_ms / 1e3) / 1e9
    traffic = NCU_TRAFFIC.get("k_acoustic_col")
    roofline = {"kernel": "k_acoustic_col", "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "traffic": traffic, "peak_source": peak_kind,
                "algorithmic_bytes": ab["k_acoustic_col"], "kernel_ms": k_ms}
    step_bytes = 662 * 4 * g.nx * g.ny * g.nz
    step_ms = ms_max / a.steps
    whole = {"ledger_bytes_per_step": step_bytes, "achieved_gbs": step_bytes / (step_ms / 1e3) / 1e9,
             "frac": step_bytes / (step_ms / 1e3) / 1e9 / hbm}

    # end to end through the public API with host buffers
    e2e = None
    if not a.no_e2e:
        host = {k: torch.empty(st[k].shape, dtype=st[k].dtype, pin_memory=True) for k in E2E_FIELDS}
        for k in E2E_FIELDS:
            host[k].copy_(st[k])
        torch.cuda.synchronize()
        cur = torch.cuda.current_stream()
        h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ke = max(1, min(a.steps, 10))
        barrier()
        torch.cuda.synchronize()
        h0.record(cur)
        for _ in range(ke):
            for k in E2E_FIELDS:
                st[k].copy_(host[k], non_blocking=True)
            it.step()
            for k in E2E_FIELDS:
                host[k].copy_(st[k], non_blocking=True)
        h1.record(cur)
        torch.cuda.synchronize()
        barrier()
        e_ms = max_over_ranks(h0.elapsed_time(h1))
        nbytes = sum(host[k].numel() * host[k].element_size() for k in E2E_FIELDS)
        e2e = {"value": job_rate(ke, e_ms, world), "unit": UNIT, "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": nbytes, "steps": ke}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        sec, sample = cpu_reference_step_time(a.config, 1, 0)
        cpu = {"value": 1.0 / sec, "unit": UNIT, "cores": 1, "kind": "port", "sample": sample}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": WORKLOAD, "grid": [g.nz, g.ny, g.nx], "points": g.nx * g.ny * g.nz,
                           "parallelism": "replicas" if world > 1 else "single",
                           "l2": "working set ~1.2 GB of fields >> 126 MB L2; no flush needed",
                           "grid_point_updates_per_s": value * g.nx * g.ny * g.nz},
                "gpu_launches": launches * a.steps, "launches_per_step": launches,
                "roofline": roofline, "step_roofline": whole, "phases_ms": phase_ms,
                "e2e": e2e, "cpu_baseline": cpu, "clocks": clocks, "nan_points": nan}
        print(json.dumps(line), flush=True)
    it._graph = None
    if world > 1:
        dist.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
