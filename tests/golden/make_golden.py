"""Generate the golden fixtures by running the reference PyWRF step on CPU.

Usage:  python tests/golden/make_golden.py [--reference /path/to/PyWRF]

Writes, next to this script:

* ``small_ref64.npz`` / ``small_ref32.npz``: full fields after 2 RK3 steps of
  a 28x28x16 synthetic state with seeded lateral-boundary tendencies, from the
  reference in float64 and float32.
* ``c0_ref64_summary.json``: per-field checksums (sum, L2 norm) and 64 sampled
  values per field after 3 steps of configuration 0 (64x64x41) in float64.
* ``c1_ref64_summary.json``: the same after 1 step of the 240x240x41
  configuration with boundary tendencies.
* ``thbias_ref64.npz``: the adjoint configuration's check on the 28x28x16
  case in float64 - a bias field added to the theta tendency after
  rk_addtend_dry, the loss L = mean (theta - theta*)^2 + mean (qv - qv*)^2
  over the lowest 10 levels of the mass points after 2 steps, against the
  initial state of a second seed - with L at zero bias and its central
  differences (eps 1e-3) in the bias at 16 seeded points.
* ``small_bdyrec_ref64.npz`` / ``small_bdyrec_ref32.npz``: u, v, t, ph, mu,
  qv after 4 steps of the 28x28x16 case with a boundary interval of 2 steps
  and three distinct boundary records (``bdy_records``), so that step 3 runs
  on record 1 after the reference's reload (solver.py:457-703), in float64
  and float32.
* ``c1_80_ref_sample.npz`` (``--only-c1-80``): the 240x240x41 workload after
  80 steps (1 h) in float64 and float32.  A full state is ~170 MB, so the
  fixture keeps, per compared field, the values of both runs at 16384 seeded
  flat indices, the exact full-field norm and sum of the float64 run and the
  exact full-field relative L2 of the float32 run against it (the
  reference's own float32 error), and the dry-mass total (sum of mu + mub
  over the mass points) of both runs and of the initial state.

The reference is read from the source tree named by ``--reference`` or the
PYWRF_REFERENCE_ROOT environment variable (one of them is required); this
script is the only producer of the fixtures and is never run by the tests.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

from pywrf_b200 import synthetic  # noqa: E402

FIELDS = ["u", "v", "w", "t", "ph", "mu", "p", "al", "h_diabatic", "rainnc", "muts", "ww"]
SPECIES = ["qv", "qc", "qr", "qi", "qs", "qg"]
SMALL = dict(n=28, nz=16, nsteps=2, bdy_tend_amp=1.0e-4, seed=3)


def pick(res):
    out = {k: res[k] for k in FIELDS}
    for i, nm in enumerate(SPECIES, start=1):
        out[nm] = res["moist"][i]
    return out


def summary(res, nsample=64, seed=0):
    rng = np.random.default_rng(seed)
    out = {}
    for k, a in pick(res).items():
        a = np.asarray(a, np.float64)
        idx = rng.integers(0, a.size, nsample)
        out[k] = {"sum": float(a.sum()), "l2": float(np.sqrt((a * a).sum())), "idx": idx.tolist(),
                  "val": a.reshape(-1)[idx].tolist(), "shape": list(a.shape)}
    return out


def bdy_records(bdy, n=3):
    """Boundary data with ``n`` distinct records: record r scales the values
    by 1 + 0.002 r and the tendencies by 1 + 0.5 r."""
    out = {}
    for k, v in bdy.items():
        v = np.asarray(v)
        ten = "_BT" in k
        out[k] = np.stack([v[0] * ((1.0 + 0.5 * r) if ten else (1.0 + 0.002 * r)) for r in range(n)]).astype(v.dtype)
    return out


BDYREC = dict(nsteps=4, bdy_interval=2)

LONG = dict(config=1, seed=0, nsteps=80, nsample=16384, sample_seed=80)


def dry_mass(res, g):
    """Sum of the column dry mass mu + mub over the mass points."""
    R = (slice(g.jds, g.jde - 1), slice(g.ids, g.ide - 1))
    return float((np.asarray(res["mu"], np.float64)[R] + np.asarray(res["mub"], np.float64)[R]).sum())


def long_fixture(refharness):
    spec = synthetic.spec_for_config(LONG["config"], seed=LONG["seed"])
    g = synthetic.grid_for(spec)
    inp, bdy = synthetic.build(spec)
    r0 = refharness.run_reference(g, inp, bdy, 0, dtype="float64")
    runs = {}
    for dt in ("float64", "float32"):
        res = refharness.run_reference(g, inp, bdy, LONG["nsteps"], dtype=dt)
        runs[dt] = (pick(res), dry_mass(res, g))
        print("ran", dt, flush=True)
    f64, m64 = runs["float64"]
    f32, m32 = runs["float32"]
    rng = np.random.default_rng(LONG["sample_seed"])
    out = {"mass0": np.array(dry_mass(r0, g)), "mass64": np.array(m64), "mass32": np.array(m32)}
    for k in f64:
        a64 = np.asarray(f64[k], np.float64)
        a32 = np.asarray(f32[k], np.float64)
        idx = rng.integers(0, a64.size, LONG["nsample"])
        nrm = float(np.sqrt((a64 * a64).sum()))
        out[f"{k}__idx"] = idx.astype(np.int64)
        out[f"{k}__v64"] = a64.reshape(-1)[idx]
        out[f"{k}__v32"] = a32.reshape(-1)[idx].astype(np.float32)
        out[f"{k}__l2"] = np.array(nrm)
        out[f"{k}__sum"] = np.array(float(a64.sum()))
        out[f"{k}__floor"] = np.array(float(np.sqrt(((a32 - a64) ** 2).sum())) / (nrm if nrm > 0 else 1.0))
        out[f"{k}__shape"] = np.array(a64.shape)
    np.savez_compressed(os.path.join(HERE, "c1_80_ref_sample.npz"),
                        meta=json.dumps({**LONG, "solver_sha256": refharness.SOLVER_SHA256}), **out)
    print("wrote c1_80_ref_sample", {k[:-7]: float(v) for k, v in out.items() if k.endswith("__floor")})


def bdyrec_case():
    import dataclasses

    spec = synthetic.CaseSpec(**SMALL)
    g = dataclasses.replace(synthetic.grid_for(spec), bdy_interval=BDYREC["bdy_interval"])
    inp, bdy = synthetic.build(spec)
    return g, inp, bdy_records(bdy)


THB = dict(nsteps=2, levels=10, npoints=16, eps=1e-3, point_seed=2024)


def thbias_region(g, levels):
    return (slice(0, levels), slice(g.jds, g.jde - 1), slice(g.ids, g.ide - 1))


def thbias_points(g):
    rng = np.random.default_rng(THB["point_seed"])
    return np.stack([rng.integers(0, THB["levels"], THB["npoints"]), rng.integers(g.jds, g.jde - 1, THB["npoints"]),
                     rng.integers(g.ids, g.ide - 1, THB["npoints"])], axis=1)


def thbias_loss(t, qv, target, g):
    R = thbias_region(g, THB["levels"])
    return float(((t[R] - target["t"]) ** 2).mean() + ((qv[R] - target["qv"]) ** 2).mean())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("PYWRF_REFERENCE_ROOT"))
    ap.add_argument("--skip-c1", action="store_true")
    ap.add_argument("--only-bdyrec", action="store_true", help="write small_bdyrec_ref64.npz only")
    ap.add_argument("--only-thbias", action="store_true", help="write thbias_ref64.npz only")
    ap.add_argument("--only-c1-80", action="store_true", help="write c1_80_ref_sample.npz only")
    args = ap.parse_args()
    if not args.reference:
        ap.error("name the reference source tree with --reference or PYWRF_REFERENCE_ROOT")
    os.environ["PYWRF_REFERENCE_ROOT"] = args.reference
    import refharness
    refharness.REF_ROOT = args.reference

    if args.only_c1_80:
        long_fixture(refharness)
        return

    if args.only_thbias:
        import dataclasses

        spec = synthetic.CaseSpec(**SMALL)
        g = synthetic.grid_for(spec)
        inp, bdy = synthetic.build(spec)
        inp2, bdy2 = synthetic.build(dataclasses.replace(spec, seed=spec.seed + 1))
        t0 = refharness.run_reference(g, inp2, bdy2, 0, dtype="float64")
        R = thbias_region(g, THB["levels"])
        target = {"t": t0["t"][R], "qv": t0["moist"][1][R]}
        nz, ny, nx = g.nz, g.ny, g.nx

        def loss(bias):
            r = refharness.run_reference(g, inp, bdy, THB["nsteps"], dtype="float64", theta_bias=bias)
            return thbias_loss(r["t"], r["moist"][1], target, g)

        zero = np.zeros((nz, ny, nx))
        pts = thbias_points(g)
        fd = []
        for k, j, i in pts:
            b = zero.copy()
            b[k, j, i] = THB["eps"]
            lp = loss(b)
            b[k, j, i] = -THB["eps"]
            fd.append((lp - loss(b)) / (2 * THB["eps"]))
        np.savez_compressed(os.path.join(HERE, "thbias_ref64.npz"), meta=json.dumps({"case": SMALL, **THB}),
                            loss0=np.array(loss(zero)), points=pts, fd=np.array(fd), target_t=target["t"],
                            target_qv=target["qv"])
        print("wrote thbias", fd[:4])
        return

    g, inp, bdy = bdyrec_case()
    for dt in ("float64", "float32"):
        res = refharness.run_reference(g, inp, bdy, BDYREC["nsteps"], dtype=dt)
        keep = {k: np.asarray(v, dt) for k, v in pick(res).items() if k in ("u", "v", "t", "ph", "mu", "qv")}
        np.savez_compressed(os.path.join(HERE, f"small_bdyrec_ref{dt[-2:]}.npz"), meta=json.dumps(
            {"case": SMALL, **BDYREC, "solver_sha256": refharness.SOLVER_SHA256}), **keep)
        print("wrote small_bdyrec", dt)
    if args.only_bdyrec:
        return

    spec = synthetic.CaseSpec(**SMALL)
    g = synthetic.grid_for(spec)
    inp, bdy = synthetic.build(spec)
    meta = {"case": SMALL, "solver_sha256": None}
    for dt in ("float64", "float32"):
        res = refharness.run_reference(g, inp, bdy, spec.nsteps, dtype=dt)
        meta["solver_sha256"] = refharness.SOLVER_SHA256
        np.savez_compressed(os.path.join(HERE, f"small_ref{dt[-2:]}.npz"),
                            meta=json.dumps(meta), **{k: np.asarray(v, dt) for k, v in pick(res).items()})
        print("wrote small", dt)

    spec0 = synthetic.spec_for_config(0)
    g0 = synthetic.grid_for(spec0)
    inp0, bdy0 = synthetic.build(spec0)
    res0 = refharness.run_reference(g0, inp0, bdy0, 3, dtype="float64")
    with open(os.path.join(HERE, "c0_ref64_summary.json"), "w") as f:
        json.dump({"config": 0, "nsteps": 3, "solver_sha256": refharness.SOLVER_SHA256,
                   "fields": summary(res0)}, f)
    print("wrote c0 summary")
    if not args.skip_c1:
        spec1 = synthetic.spec_for_config(1)
        g1 = synthetic.grid_for(spec1)
        inp1, bdy1 = synthetic.build(spec1)
        res1 = refharness.run_reference(g1, inp1, bdy1, 1, dtype="float64")
        with open(os.path.join(HERE, "c1_ref64_summary.json"), "w") as f:
            json.dump({"config": 1, "nsteps": 1, "solver_sha256": refharness.SOLVER_SHA256,
                       "fields": summary(res1)}, f)
        print("wrote c1 summary")


if __name__ == "__main__":
    main()
