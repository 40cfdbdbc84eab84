"""Benchmark: ARW RK3 steps/s on the 240x240x41 synthetic moist workload.

``python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]``

One step = one complete ``wrf_rk3_step`` (three RK stages, 1+2+4 acoustic
substeps, moisture transport, WSM6, boundary updates) over the 240x240x41
state built by :mod:`pywrf_b200.synthetic` (the 240x240x41 / dt 45 s / 80-step
workload with seeded boundary tendencies), replayed from one captured CUDA
graph.  The workload is a 1-h integration: K steps run as integrations of at
most 80 steps, each from the initial state (its seeded boundary tendencies
drive the forced boundary state unstable after ~175 steps); the restore lies
between timed segments and the NaN count of every integration is kept, a NaN
making the run exit non-zero.  The timed region is bracketed by barrier +
synchronize; the device time is measured with CUDA events on the replay
stream and the maximum over ranks is reported.  Multi-GPU runs are
independent replicas (different seeds, no data-path collective): the step is
column-local but its lateral boundary is one domain, so ``value`` = N * K /
max-rank time ("weak" scaling).

Extra keys of the JSON line:
  roofline      the dominant kernel's algorithmic bytes / CUDA-event duration
                against the measured HBM copy bandwidth
  step_roofline the whole step's 662-pass ledger against the same peak
  phases        per-phase device time of one eager step (probe events)
  e2e           the same metric through the public API with host buffers
                (Integrator.run_host): every step the pinned H2D of the
                prognostic state, the step, the D2H of it back
  cpu_baseline  the unmodified reference (installed offline in
                baseline/_ref) on this host's CPU threads, one step of the
                same workload; where the install is absent, the numpy oracle
  cpu_baseline_port  the numpy oracle (a restatement of the reference's
                algorithm) on one host thread, one step
  reference_cpu the unmodified reference's own CPU step, recorded where its
                source lives (tests/golden/reference_cpu_timing.json)
  reference_gpu the unmodified reference's own PyTorch step on a B200,
                recorded by tests/golden/time_reference_gpu.py
                (tests/golden/reference_gpu_timing.json), with this run's
                value and e2e as ratios to it
  config4       the 512x512x61 workload's plain step (36 steps): steps/s,
                ledger fraction, peak device memory
  clocks        SM clock samples taken during the timed region
  surrogate     the per-column network in place of WSM6: trained on the GPU
                on harvested WSM6 increments, then one unseen state run for
                1 h with the plain and the surrogate step (speed, hydrometeor
                mass and precipitation errors, tensor-core roofline)
  adjoint       one whole step forward + reverse (WSM6 included) composed
                from the hand-written operator adjoints, with and without the
                microphysics, beside the fused forward step; and the acoustic
                part of RK stage 3 alone
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

METRIC = "RK3 steps/s @240x240x41: surrogate vs plain WSM6 at <=2% err; fwd+adj steps/s"
UNIT = "steps/s"
WORKLOAD = "240x240x41 synthetic moist ARW, plain WSM6, dt=45 s, 4 acoustic substeps, seeded bdy tendencies"
FALLBACK_HBM_GBS = 6650.0

# prognostic fields a host-driven caller moves in and out each step (e2e)
E2E_FIELDS = ("u", "v", "w", "t", "ph", "mu", "p", "al", "moist")

# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per launch of the
# dominant kernel, from one ncu capture of this workload's step (the third
# k_acoustic_col launch: RK stage 2's second substep): a constant of that
# capture, not a measurement of the run, and labelled so in the bench line
NCU_TRAFFIC = {"k_acoustic_col": 312.6e6}


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
    ap.add_argument("--no-surrogate", action="store_true", help="skip the network (harvest, training, surrogate run)")
    ap.add_argument("--no-config4", action="store_true", help="skip the 512x512x61 plain-step figure")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the composed acoustic-stage forward + adjoint")
    ap.add_argument("--sur-seeds", type=int, default=5, help="integrations harvested for the network's training set")
    ap.add_argument("--sur-harvest-steps", type=int, default=80)
    ap.add_argument("--sur-epochs", type=int, default=200)
    ap.add_argument("--sur-steps", type=int, default=80, help="steps of the surrogate-vs-plain comparison (80 = 1 h)")
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


REF_INSTALL = os.path.join(ROOT, "baseline", "_ref")


def reference_host_step_time(config: int, nsteps: int, warmup: int):
    """Seconds per step of the unmodified reference -- installed offline in
    baseline/_ref, run through its own solver loop by
    tests/golden/refharness.py (float32, torch on the CPU with all host
    threads) -- on the same workload: the difference of a solve of
    ``warmup`` steps and one of ``warmup + nsteps`` steps, after a
    first-touch solve.  Returns (seconds, threads, sample) or None when the
    install is absent."""
    if not os.path.isfile(os.path.join(REF_INSTALL, "pywrf", "solver.py")):
        return None
    import torch
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import refharness
    from pywrf_b200 import synthetic
    refharness.REF_ROOT = REF_INSTALL
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    spec = synthetic.spec_for_config(config)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)

    def solve(n):
        t0 = time.perf_counter()
        refharness.run_reference(g, inputs, bdy, n, dtype="float32", device="cpu")
        return time.perf_counter() - t0

    w = max(1, warmup)
    solve(1)
    t_w = solve(w)
    t_wk = solve(w + nsteps)
    sec = (t_wk - t_w) / nsteps
    return sec, threads, (f"{nsteps} RK3 step(s) of the {g.nx}x{g.ny}x{g.nz} workload after {w} warm-up, the "
                          f"unmodified reference (baseline/_ref, float32) on {threads} host threads")


def reference_cpu_record(grid_key: str):
    """The unmodified reference's own CPU step on this workload, as timed by
    tests/golden/time_reference_cpu.py where the reference's source lives (a
    recorded measurement of another machine, not of this run)."""
    p = os.path.join(ROOT, "tests", "golden", "reference_cpu_timing.json")
    try:
        with open(p) as f:
            d = json.load(f)
        w = d["workloads"][grid_key]
    except (OSError, KeyError, ValueError):
        return None
    return {"value": w["steps_per_s"], "unit": UNIT, "cores": d["threads"], "kind": "reference",
            "machine": f"{d['cpu']} ({d['logical_cpus']} logical CPUs), torch {d['torch']}, {d['dtype']}",
            "sample": f"{w['timed_steps']} timed step(s) after {w['warmup_steps']} warm-up",
            "recorded_in": "tests/golden/reference_cpu_timing.json (not measured in this run)"}


def reference_gpu_record(grid_key: str, value: float, e2e: float | None):
    """The unmodified reference's own PyTorch step on a B200 on this
    workload, as timed by tests/golden/time_reference_gpu.py (its solver
    loop on cuda:0, float32; a recorded measurement, not of this run), with
    the ratios of this run's device-resident and end-to-end figures to it."""
    p = os.path.join(ROOT, "tests", "golden", "reference_gpu_timing.json")
    try:
        with open(p) as f:
            d = json.load(f)
        w = d["workloads"][grid_key]
    except (OSError, KeyError, ValueError):
        return None
    return {"value": w["steps_per_s"], "unit": UNIT, "device": d["device"],
            "machine": f"torch {d['torch']}, {d['dtype']}",
            "sample": f"{w['timed_steps']} timed step(s) after {w['warmup_steps']} warm-up",
            "recorded_in": "tests/golden/reference_gpu_timing.json (not measured in this run)",
            "value_ratio": value / w["steps_per_s"],
            "e2e_ratio": (e2e / w["steps_per_s"]) if e2e else None}


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # bounded sample: each oracle step of this workload is tens of seconds of
    # CPU work, so at most 1 warm-up and 2 timed steps are run
    k, w = max(1, min(a.steps, 2)), min(a.warmup, 1)
    ref = reference_host_step_time(a.config, k, w)
    if ref is not None:
        sec, cores, sample = ref
        kind = "reference"
    else:  # the reference's install is absent: its algorithm by the numpy port
        sec, sample = cpu_reference_step_time(a.config, k, w)
        cores, kind = 1, "port"
    v = 1.0 / sec
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": k, "warmup": w,
            "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "parallelism": "replicas"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
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

    # The workload is a 1-h integration (spec.nsteps = 80 steps): its seeded
    # boundary tendencies push the boundary state linearly away from the
    # initial one, and the forced state is defined (and stable) over that
    # hour, not indefinitely.  K timed steps therefore run as integrations of
    # at most spec.nsteps steps, each from the initial state; the copy back to
    # it lies between the timed segments.  NaN counts of every segment are
    # accumulated on the device before each restore.
    seg = max(1, spec.nsteps)
    init = st.snapshot()
    nan_acc = torch.zeros((), dtype=torch.int64, device=st["status"].device)

    def restart():
        nan_acc.add_(st["status"][N.WRF_ST_NAN_P].to(torch.int64))
        st.restore(init)

    # one eager step: launch count, then the graph
    it.step()
    launches = N.lib().wrf_last_launch_count()
    restart()
    it.capture()
    for w in range(a.warmup):
        if w and w % seg == 0:
            restart()
        it.replay()
    torch.cuda.synchronize()
    restart()

    stream = it._graph_stream
    nseg = (a.steps + seg - 1) // seg
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(nseg)]
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as cs:
        done = 0
        for e0, e1 in evs:
            n = min(seg, a.steps - done)
            with torch.cuda.stream(stream):
                e0.record(stream)
                for _ in range(n):
                    it._graph.replay()
                e1.record(stream)
            done += n
            if done < a.steps:
                with torch.cuda.stream(stream):
                    restart()
        torch.cuda.synchronize()
    barrier()
    ms = sum(e0.elapsed_time(e1) for e0, e1 in evs)
    ms_max = max_over_ranks(ms)
    value = job_rate(a.steps, ms_max, world)
    clocks = cs.summary()
    restart()

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
    restart()

    # roofline of the dominant kernel, k_acoustic_col (the "sub.col" phases:
    # that kernel alone, 7 launches per step)
    hbm, peak_kind = peaks()
    ab = algorithmic_bytes(g)
    k_ms = phase_ms.get("sub.col", float("nan")) / COL_LAUNCHES_PER_STEP
    achieved = ab["k_acoustic_col"] / (k_ms / 1e3) / 1e9
    traffic = NCU_TRAFFIC.get("k_acoustic_col")
    roofline = {"kernel": "k_acoustic_col", "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "traffic": traffic, "peak_source": peak_kind,
                "traffic_source": "ncu capture of the 240x240x41 step (the kernel's third launch, RK stage "
                                  "2's second substep), not measured in this run",
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
        # the public host-driven call: every step copies the fields in from the
        # pinned host buffers, replays the captured step and copies them back
        it.run_host(host, ke)
        h1.record(cur)
        torch.cuda.synchronize()
        barrier()
        e_ms = max_over_ranks(h0.elapsed_time(h1))
        nbytes = sum(host[k].numel() * host[k].element_size() for k in E2E_FIELDS)
        e2e = {"value": job_rate(ke, e_ms, world), "unit": UNIT, "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": nbytes, "steps": ke}
        restart()
    nan = int(nan_acc.item())
    del init

    sur = None
    if world > 1:
        sur = {"unavailable": "measured at one GPU only (the replicas run the plain step)"}
    elif not a.no_surrogate:
        sur = run_surrogate(a, hbm)

    big = None
    if world == 1 and not a.no_config4:
        big = run_config4(hbm, with_adjoint=not a.no_adjoint)
    adj = None
    if world > 1:
        adj = {"unavailable": "measured at one GPU only"}
    elif not a.no_adjoint:
        adj = run_adjoint_step(st, it, ms_max / a.steps)
        adj["acoustic_stage"] = run_adjoint_stage(st, it, phase_ms)

    cpu = cpu_port = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        sec, sample = cpu_reference_step_time(a.config, 1, 0)
        cpu_port = {"value": 1.0 / sec, "unit": UNIT, "cores": 1, "kind": "port", "sample": sample}
        ref = reference_host_step_time(a.config, 1, 1)
        if ref is not None:
            sec, cores, sample = ref
            cpu = {"value": 1.0 / sec, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample}
        else:
            cpu = cpu_port

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
                "e2e": e2e, "cpu_baseline": cpu, "cpu_baseline_port": cpu_port, "clocks": clocks, "nan_points": nan,
                "surrogate": sur, "config4": big,
                "reference_cpu": reference_cpu_record(f"{g.nx}x{g.ny}x{g.nz}"),
                "reference_gpu": reference_gpu_record(f"{g.nx}x{g.ny}x{g.nz}", value,
                                                      e2e["value"] if e2e else None),
                "adjoint": adj}
        line["valid"] = nan == 0
        print(json.dumps(line), flush=True)
    it._graph = None
    if world > 1:
        dist.destroy_process_group()
    if nan:
        raise SystemExit(f"NaN in the diagnosed pressure at {nan} point(s): the timed state is not a result")


def run_adjoint_step(st, it, fused_step_ms, reps=3):
    """Forward + reverse pass of one whole step -- the three RK stages, the
    microphysics (WSM6's reverse over a per-column tape) and the
    end-of-step boundaries -- composed from the hand-written operator
    adjoints (pywrf_b200.adjoint.step) on the 240x240x41 state after one
    step, timed with CUDA events (2 warm-up passes): the fwd+adj steps per
    second of the adjoint configuration's unit of work (eagerly, and
    captured once in a CUDA graph by adjoint.capture and replayed), the same
    without the microphysics, and the composed forward alone, beside the
    fused forward step."""
    import torch
    from pywrf_b200 import adjoint as A

    g = st.g
    it.step()
    torch.cuda.synchronize()
    names = tuple(dict.fromkeys(A.RK_STATE + ("u_1", "w_1", "ph_1", "mu_1", "t_1", "v_1")))
    data = {k: st[k] for k in dict.fromkeys(A.STEP_DATA + A._Microphysics.data)}
    keys = (("bxs", "xs"), ("bxe", "xe"), ("bys", "ys"), ("bye", "ye"), ("btxs", "txs"), ("btxe", "txe"),
            ("btys", "tys"), ("btye", "tye"))
    bd = {f: {key: st[f"{f}_{n}"] for n, key in keys} for f in ("u", "v", "ph", "t", "mu", "qv")}
    sc = dict(epssm=g.epssm, emdiv=g.emdiv, smdiv=g.smdiv, cf1=st.scal["cf1"], cf2=st.scal["cf2"],
              cf3=st.scal["cf3"], cfn=st.scal["cfn"], cfn1=st.scal["cfn1"], rdx=g.rdx, rdy=g.rdy)
    state = {k: st[k].detach().clone().requires_grad_(True) for k in names}
    mp = lambda s: A.microphysics(s, data, g.dt, g.rdx, g.rdy)  # noqa: E731
    gen = torch.Generator(device=st["u"].device).manual_seed(7)
    outs = ("u", "v", "w", "ph", "t", "mu", "p", "al", "moist")
    cot = {k: torch.randn(st[k].shape, generator=gen, device=st[k].device) for k in outs}

    def run(micro, backward):
        for v in state.values():
            v.grad = None
        if backward:
            o = A.step(state, data, bd, 2.0 * g.dt, dt=g.dt, soundsteps=g.soundsteps, microphysics=micro, **sc)
            sum((o[k] * cot[k]).sum() for k in outs).backward()
        else:
            with torch.no_grad():
                A.step(state, data, bd, 2.0 * g.dt, dt=g.dt, soundsteps=g.soundsteps, microphysics=micro, **sc)

    res = {}
    for name, micro, bwd in (("fwd_adj", mp, True), ("fwd_adj_dry", None, True), ("fwd_composed", mp, False)):
        for _ in range(2):
            run(micro, bwd)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            run(micro, bwd)
        e1.record()
        torch.cuda.synchronize()
        res[name] = e0.elapsed_time(e1) / reps
    # the same pass with microphysics, captured once in a CUDA graph and replayed
    graph = A.capture(lambda: run(mp, True))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        graph.replay()
    e1.record()
    torch.cuda.synchronize()
    res["fwd_adj_graph"] = e0.elapsed_time(e1) / reps
    del graph
    peak = torch.cuda.max_memory_allocated() / 2**30
    return {"what": "one whole step (3 RK stages, WSM6 microphysics, end-of-step boundaries) forward and reverse, "
                    "composed from the operator adjoints, 240x240x41",
            "fwd_adj_ms": res["fwd_adj"], "fwd_adj_steps_per_s": 1e3 / res["fwd_adj"],
            "fwd_adj_ms_graph": res["fwd_adj_graph"], "fwd_adj_steps_per_s_graph": 1e3 / res["fwd_adj_graph"],
            "fwd_adj_ms_without_microphysics": res["fwd_adj_dry"], "fwd_composed_ms": res["fwd_composed"],
            "fused_forward_step_ms": fused_step_ms, "peak_gib": peak,
            "reference_autograd": "not comparable: the reference's autograd cannot run backward through its "
                                  "acoustic solve (in-place updates of saved operands in calc_coef_w, advance_uv, "
                                  "advance_w)"}


def run_adjoint_stage(st, it, phase_ms, reps=5):
    """Forward + reverse pass of the acoustic part of RK stage 3 (4
    substeps) composed from the hand-written operator adjoints
    (pywrf_b200.adjoint.acoustic_stage) on the 240x240x41 state after the
    tendencies of a step, timed with CUDA events (3 warm-up passes): stages
    per second, beside the fused forward's time for the same part of a step
    (stage 3's share of the acoustic phases in the step's probe timing)."""
    import torch
    from pywrf_b200 import _native as N_
    from pywrf_b200 import adjoint as A

    g = st.g
    L = N_.lib()
    h = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    gp = ctypes.byref(st.cgrid)
    # a state after one step and the first stage's tendencies of the next
    it.step()
    for fn, args in (("wrf_step_begin", ()), ("wrf_rk_prep", (1,)), ("wrf_diff_stage1", ()), ("wrf_tend_stage", (1,))):
        N_.check(getattr(L, fn)(gp, st.ptr, *args, h), fn)
    torch.cuda.synchronize()
    state = {k: st[k].detach().clone().requires_grad_(True) for k in A.STAGE_STATE}
    data = {k: st[k] for k in A.STAGE_DATA}
    sc = dict(epssm=g.epssm, emdiv=g.emdiv, smdiv=g.smdiv, cf1=st.scal["cf1"], cf2=st.scal["cf2"],
              cf3=st.scal["cf3"], rdx=g.rdx, rdy=g.rdy)
    dts = g.dt / g.soundsteps
    gen = torch.Generator(device=st["u"].device).manual_seed(5)
    outs = ("u", "v", "w", "ph", "t", "mu", "p", "al", "ww", "ru_m", "rv_m", "ww_m")
    cot = {k: torch.randn(st[k].shape, generator=gen, device=st[k].device) for k in outs}

    def one():
        for v in state.values():
            v.grad = None
        o = A.acoustic_stage(state, data, 3, g.soundsteps, dts, **sc)
        sum((o[k] * cot[k]).sum() for k in outs).backward()

    def fwd():
        with torch.no_grad():
            A.acoustic_stage(state, data, 3, g.soundsteps, dts, **sc)

    res = {}
    for name, fn in (("fwd_adj", one), ("fwd_composed", fwd)):
        for _ in range(3):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        res[name] = e0.elapsed_time(e1) / reps
    # stage 3's share of the step's acoustic phases: a third of the prep and
    # finish, four of the seven substeps
    fused = (phase_ms.get("acprep", 0.0) + phase_ms.get("acfinish", 0.0)) / 3.0 + \
        sum(phase_ms.get(k, 0.0) for k in ("sub.uv", "sub.col", "sub.bc")) * 4.0 / 7.0
    return {"what": "acoustic part of RK stage 3 (small_step_prep, calc_p_rho, calc_coef_w, 4 substeps, "
                    "small_step_finish) composed from the operator adjoints, 240x240x41",
            "fwd_adj_ms": res["fwd_adj"], "fwd_adj_stages_per_s": 1e3 / res["fwd_adj"],
            "fwd_composed_ms": res["fwd_composed"],
            "fused_step_forward_ms_per_stage": fused,
            "reference_autograd": "not comparable: the reference's autograd cannot run backward through its "
                                  "acoustic solve (in-place updates of saved operands in calc_coef_w, advance_uv, "
                                  "advance_w)"}


def run_config4(hbm, with_adjoint=True):
    """The 512x512x61 workload (dt 30 s, one 36-step integration) with the
    plain step: steps/s, grid-point updates/s, the step's ledger fraction of
    the HBM peak, peak device memory and the NaN count; with_adjoint adds
    the forward + reverse of whole steps at that size (config4_adjoint)."""
    import torch
    from pywrf_b200 import _native as N_
    from pywrf_b200 import synthetic
    from pywrf_b200.solver import Integrator
    from pywrf_b200.state import DeviceState

    spec = synthetic.spec_for_config(4)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    torch.cuda.synchronize()
    torch.cuda.reset_peak_memory_stats()
    base = torch.cuda.memory_allocated()
    st = DeviceState.from_inputs(g, inputs, bdy, device="cuda")
    del inputs, bdy
    it = Integrator(st)
    init = st.snapshot()
    it.capture()
    for _ in range(3):
        it.replay()
    st.restore(init)
    torch.cuda.synchronize()
    stream = it._graph_stream
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(spec.nsteps):
            it._graph.replay()
        e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / spec.nsteps
    nan = it.status()["nan_p"]
    n3 = g.nx * g.ny * g.nz
    ledger = 662 * 4 * n3
    peak = torch.cuda.max_memory_allocated() - base
    it._graph = None
    adj = None
    if with_adjoint:
        st.restore(init)
        it.step()
        torch.cuda.synchronize()
        adj = config4_adjoint(st, g, base)
    del init, st, it
    torch.cuda.empty_cache()
    return {"workload": f"{g.nx}x{g.ny}x{g.nz} synthetic moist ARW, plain WSM6, dt={spec.dt:g} s, "
                        f"{spec.nsteps} steps from the initial state",
            "steps_per_s": 1e3 / ms, "ms_per_step": ms, "grid_point_updates_per_s": 1e3 / ms * n3,
            "step_roofline": {"ledger_bytes_per_step": ledger, "achieved_gbs": ledger / (ms / 1e3) / 1e9,
                              "frac": ledger / (ms / 1e3) / 1e9 / hbm},
            "peak_device_bytes": peak, "state_plus_snapshot": "the field table and one copy of it",
            "nan_points": nan, "adjoint": adj}


def config4_adjoint(st, g, base, nsteps=2):
    """Forward + reverse of ``nsteps`` whole steps (plain WSM6) at the
    config-4 size under adjoint.rollout with one checkpoint per step (the
    forward keeps each step's input state; the backward recomputes a step and
    runs its operators' adjoints), from the state after one step: seconds
    per step and the peak device memory of the pass (a 1-step pass first as
    warm-up)."""
    import torch
    from pywrf_b200 import adjoint as A

    names = tuple(dict.fromkeys(A.RK_STATE + ("u_1", "w_1", "ph_1", "mu_1", "t_1", "v_1")))
    data = {k: st[k] for k in dict.fromkeys(A.STEP_DATA + A._Microphysics.data)}
    keys = (("bxs", "xs"), ("bxe", "xe"), ("bys", "ys"), ("bye", "ye"), ("btxs", "txs"), ("btxe", "txe"),
            ("btys", "tys"), ("btye", "tye"))
    bd = {f: {key: st[f"{f}_{n}"] for n, key in keys} for f in ("u", "v", "ph", "t", "mu", "qv")}
    sc = dict(epssm=g.epssm, emdiv=g.emdiv, smdiv=g.smdiv, cf1=st.scal["cf1"], cf2=st.scal["cf2"],
              cf3=st.scal["cf3"], cfn=st.scal["cfn"], cfn1=st.scal["cfn1"], rdx=g.rdx, rdy=g.rdy)
    bias = torch.zeros_like(st["t"], requires_grad=True)
    mp = lambda s: A.microphysics(s, data, g.dt, g.rdx, g.rdy)  # noqa: E731

    def one(*xs):
        n = int(round(float(xs[-1].item())))
        s = A.step(dict(zip(names, xs[:-1])), data, bd, g.dt * n, dt=g.dt, soundsteps=g.soundsteps,
                   microphysics=mp, theta_bias=bias, **sc)
        return tuple(s[k] for k in names) + (xs[-1] + 1,)

    def run(k):
        bias.grad = None
        x0 = tuple(st[k2].detach().clone() for k2 in names) + (torch.tensor(2.0, device=st["u"].device),)
        outs = A.rollout(one, x0, k, every=1)
        o = dict(zip(names, outs))
        ((o["t"][:10].double() ** 2).mean() + (o["moist"][1][:10].double() ** 2).mean()).backward()

    try:
        run(1)
        torch.cuda.synchronize()
        torch.cuda.reset_peak_memory_stats()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        run(nsteps)
        e1.record()
        torch.cuda.synchronize()
    except torch.cuda.OutOfMemoryError as e:  # reported, not fatal to the bench
        torch.cuda.empty_cache()
        return {"unavailable": f"out of device memory: {str(e).splitlines()[0]}"}
    sec = e0.elapsed_time(e1) / 1e3 / nsteps
    return {"what": f"{nsteps} whole steps (plain WSM6) forward and reverse under rollout, one checkpoint per "
                    "step, theta-bias gradient of a lowest-10-level loss",
            "seconds_per_step": sec, "fwd_adj_steps_per_s": 1.0 / sec,
            "peak_device_bytes": torch.cuda.max_memory_allocated() - base,
            "surrogate_form": "not composed: the network's reverse is built for its training, not wired into "
                              "the differentiable step"}


def hydrometeor_budget(st, g):
    """Dry-air-mass-weighted totals of qc..qg (kg per m^2, summed over the
    mass points) and the domain sum of accumulated precipitation."""
    import torch
    ids, ide, jds, jde, nz = g.ids, g.ide, g.jds, g.jde, g.nz
    mu = (st["mu"] + st["mub"])[jds:jde - 1, ids:ide - 1].double()
    dnw = st["dnw"][:nz - 1].double().abs()
    out = {}
    for m, name in enumerate(("qc", "qr", "qi", "qs", "qg"), start=2):
        q = st["moist"][m, :nz - 1, jds:jde - 1, ids:ide - 1].double()
        out[name] = float((q * dnw[:, None, None] * mu[None]).sum() / 9.81)
    out["hydrometeors"] = sum(out[k] for k in ("qc", "qr", "qi", "qs", "qg"))
    out["rainnc"] = float(st["rainnc"][jds:jde - 1, ids:ide - 1].double().sum())
    return out


def run_surrogate(a, hbm_peak):
    """Train the per-column network on harvested WSM6 increments (all on the
    tensor-core kernels), then integrate one unseen 240x240x41 state for
    --sur-steps steps with the plain step and with the surrogate step (WSM6
    every 10th step and on rejected columns) and compare their speed and
    their hydrometeor mass and precipitation."""
    import torch
    from pywrf_b200 import _native as N_
    from pywrf_b200 import surrogate, synthetic
    from pywrf_b200.solver import Integrator
    from pywrf_b200.state import DeviceState

    def spec_for(seed):
        return synthetic.spec_for_config(1, seed=seed)

    t0 = time.time()
    raw_in, raw_out, lay = surrogate.harvest(range(a.sur_seeds), a.sur_harvest_steps, spec_for, per_step=5000)
    torch.cuda.synchronize()
    t_harvest = time.time() - t0
    spec = spec_for(100)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    st_plain = DeviceState.from_inputs(g, inputs, bdy, device="cuda")
    net = surrogate.MlpNet(lay, hidden=512, device="cuda", seed=0)
    net.fit_normalisation(raw_in, raw_out)
    x, t = surrogate.standardise(net, st_plain.cgrid, raw_in, raw_out)   # (the grid's layout only)
    nrows = int(raw_in.shape[0])
    del raw_in, raw_out
    tr = surrogate.Trainer(net, batch=8192, splits=4, lr=1e-3)
    torch.cuda.synchronize()
    t0 = time.time()
    losses = tr.fit(x, t, epochs=a.sur_epochs, lr_end=1e-4)
    torch.cuda.synchronize()
    t_train = time.time() - t0
    train_flop = 3 * 2 * (nrows - nrows % tr.batch) * a.sur_epochs * sum(
        net.dims[i] * net.dims[i + 1] for i in range(4))
    del x, t, tr

    def timed(fn, n):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        fn(n)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    it = Integrator(st_plain)
    it.capture()
    ms_plain = timed(lambda n: [it.replay() for _ in range(n)], a.sur_steps)
    bp = hydrometeor_budget(st_plain, g)
    it._graph = None
    del st_plain

    # gate settings, strict to open: (tol_neg kg/kg, tol_sat); each run starts
    # from the same unseen state
    gates = []
    si = None
    for tol_neg, tol_sat in ((1e-6, 0.05), (1e-5, 0.1), (1e-4, 0.25), (1.0, 10.0)):
        st_sur = DeviceState.from_inputs(g, inputs, bdy, device="cuda")
        si = surrogate.SurrogateIntegrator(st_sur, net, judge_every=10, tol_neg=tol_neg, tol_sat=tol_sat)
        si.capture()
        si.capture_mlp()
        ms_sur = timed(lambda n: si.run(n, graph=True), a.sur_steps)
        bs = hydrometeor_budget(st_sur, g)
        rel = {k: abs(bs[k] - bp[k]) / abs(bp[k]) if bp[k] else None for k in bp}
        gates.append({"tol_neg": tol_neg, "tol_sat": tol_sat, "surrogate_steps_per_s": a.sur_steps / (ms_sur / 1e3),
                      "speedup": ms_plain / ms_sur, "rel_err_1h": rel, "surrogate_budget": bs,
                      "columns_last_surrogate_step": si.column_stats(), "nan_p": si.status()["nan_p"]})
        si._graph = None
        si._mlp_graph = None
    ok = [r for r in gates if r["rel_err_1h"]["hydrometeors"] <= 0.02 and r["rel_err_1h"]["rainnc"] <= 0.02]
    best = max(ok, key=lambda r: r["speedup"]) if ok else min(gates, key=lambda r: r["rel_err_1h"]["rainnc"])

    # the four tensor-core products of one surrogate call, alone (the
    # inference chain of the step: bias + GELU fused, bf16 activations)
    L = lay
    flop = 2 * L["ncols"] * sum(net.dims[i] * net.dims[i + 1] for i in range(4))
    lib = N_.lib()
    cs = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def fwd(n):
        for _ in range(n):
            N_.check(lib.wrf_mlp_forward(ctypes.byref(si.netc), ctypes.c_void_p(si.x.data_ptr()), L["ncols"],
                                         ctypes.c_void_p(si.hbuf[0].data_ptr()),
                                         ctypes.c_void_p(si.hbuf[1].data_ptr()), ctypes.c_void_p(si.y.data_ptr()),
                                         ctypes.c_void_p(si.err.data_ptr()), cs), "wrf_mlp_forward")
    fwd(3)
    ms_fwd = timed(fwd, 20) / 20
    peak = peaks_tensor()
    return {
        "plain_steps_per_s": a.sur_steps / (ms_plain / 1e3),
        "surrogate_steps_per_s": best["surrogate_steps_per_s"],
        "speedup": best["speedup"],
        "gate": {"tol_neg": best["tol_neg"], "tol_sat": best["tol_sat"],
                 "chosen": "fastest setting within 2 % on hydrometeor mass and precipitation" if ok else
                           "no setting within 2 % on both: the one with the smallest precipitation error"},
        "judge_every": 10, "steps": a.sur_steps, "eval_seed": 100,
        "rel_err_1h": best["rel_err_1h"], "plain_budget": bp, "gate_sweep": gates,
        "network": {"dims": net.dims, "dtype": "bf16 weights/activations, fp32 accumulate (tcgen05)"},
        "training": {"rows": nrows, "seeds": a.sur_seeds, "harvest_steps": a.sur_harvest_steps,
                     "epochs": a.sur_epochs, "batch": 8192, "loss_first": losses[0], "loss_last": losses[-1],
                     "harvest_s": t_harvest, "train_s": t_train, "train_tflops": train_flop / t_train / 1e12},
        "tensor_roofline": {"kernel": "k_gemm_tc (4 layers, one call)", "bound": "tensor",
                            "achieved": flop / (ms_fwd / 1e3) / 1e12, "peak": peak[0], "unit": "TFLOP/s",
                            "frac": flop / (ms_fwd / 1e3) / 1e12 / peak[0], "peak_source": peak[1],
                            "flop_per_call": flop, "ms_per_call": ms_fwd},
    }


def peaks_tensor():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        if d.get("bf16_tflops"):
            return float(d["bf16_tflops"]), "measured (burst)"
    return 1590.0, "fallback"


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
