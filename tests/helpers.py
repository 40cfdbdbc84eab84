"""Comparison helpers shared by the parity tests."""
from __future__ import annotations

import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

FIELDS = ["u", "v", "w", "t", "ph", "mu", "p", "al", "h_diabatic", "rainnc", "muts", "ww"]
SPECIES = ["qv", "qc", "qr", "qi", "qs", "qg"]

# the small golden case (must match tests/golden/make_golden.py)
SMALL = dict(n=28, nz=16, nsteps=2, bdy_tend_amp=1.0e-4, seed=3)


def pick(get) -> dict[str, np.ndarray]:
    """The compared fields from a state accessor ``get(name) -> array``."""
    out = {k: np.asarray(get(k)) for k in FIELDS}
    moist = np.asarray(get("moist"))
    for i, nm in enumerate(SPECIES, start=1):
        out[nm] = moist[i]
    return out


def rel_l2(a, ref) -> float:
    """||a - ref|| / ||ref|| over the entries where ref is finite (absolute
    norm when ref is identically zero)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(ref, np.float64)
    m = np.isfinite(b)
    nb = float(np.sqrt((b[m] ** 2).sum()))
    d = float(np.sqrt(((a[m] - b[m]) ** 2).sum()))
    return d / nb if nb > 0 else d


def load_npz(name: str) -> dict[str, np.ndarray]:
    with np.load(os.path.join(GOLDEN, name)) as z:
        return {k: z[k] for k in z.files if k != "meta"}


def load_summary(name: str) -> dict:
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def summary_errors(fields: dict[str, np.ndarray], summ: dict) -> dict[str, tuple[float, float]]:
    """(sampled-value error, L2-norm error) of each field against a reference
    checksum record.  Sampled errors are scaled by the larger of the sampled
    magnitude and the field's RMS."""
    out = {}
    for k, s in summ["fields"].items():
        a = np.asarray(fields[k], np.float64).reshape(-1)
        assert list(np.asarray(fields[k]).shape) == s["shape"], k
        idx = np.asarray(s["idx"])
        v = np.asarray(s["val"])
        rms = s["l2"] / np.sqrt(a.size)
        scale = max(float(np.abs(v).max()), rms, 1e-30)
        l2 = float(np.sqrt((a * a).sum()))
        out[k] = (float(np.abs(a[idx] - v).max()) / scale, abs(l2 - s["l2"]) / max(s["l2"], 1e-30))
    return out


def bdy_records(bdy, n=3):
    """The boundary records of tests/golden/make_golden.py's boundary-record
    case: record r scales the values by 1 + 0.002 r and the tendencies by
    1 + 0.5 r."""
    return {k: np.stack([np.asarray(v)[0] * ((1.0 + 0.5 * r) if "_BT" in k else (1.0 + 0.002 * r))
                         for r in range(n)]).astype(np.asarray(v).dtype) for k, v in bdy.items()}
