"""The oracle against the reference's own outputs (golden fixtures made by
tests/golden/make_golden.py from the unmodified reference step).

An fp64 oracle must reproduce the fp64 reference to rounding (1e-10 relative
L2); the fp32 oracle must stay within the reference's own fp32 error (its
fp32 run against its fp64 run), so that the oracle can stand in for the
reference when the CUDA kernels are checked.
"""
from __future__ import annotations

import numpy as np
import pytest

from helpers import SMALL, load_npz, load_summary, pick, rel_l2, summary_errors
from oracle.model import OracleModel
from pywrf_b200 import synthetic


@pytest.fixture(scope="module")
def small_case():
    spec = synthetic.CaseSpec(**SMALL)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    return g, inputs, bdy


def _run(g, inputs, bdy, dtype, nsteps):
    m = OracleModel(g, inputs, bdy, dtype)
    m.run(nsteps)
    return pick(lambda k: m.st[k])


def test_oracle64_matches_reference64_small(small_case):
    g, inputs, bdy = small_case
    ref = load_npz("small_ref64.npz")
    out = _run(g, inputs, bdy, np.float64, SMALL["nsteps"])
    for k, v in out.items():
        assert rel_l2(v, ref[k]) < 1e-10, k


def test_oracle32_within_reference_fp32_error_small(small_case):
    g, inputs, bdy = small_case
    r64, r32 = load_npz("small_ref64.npz"), load_npz("small_ref32.npz")
    out = _run(g, inputs, bdy, np.float32, SMALL["nsteps"])
    for k, v in out.items():
        floor = rel_l2(r32[k], r64[k])
        assert rel_l2(v, r64[k]) <= 2.5 * floor + 1e-9, (k, rel_l2(v, r64[k]), floor)


def test_oracle64_matches_reference64_config0_three_steps():
    summ = load_summary("c0_ref64_summary.json")
    spec = synthetic.spec_for_config(0)
    g = synthetic.grid_for(spec)
    inputs, bdy = synthetic.build(spec)
    out = _run(g, inputs, bdy, np.float64, summ["nsteps"])
    for k, (samp, l2) in summary_errors(out, summ).items():
        # WSM6 thresholds (qs > 0, qi > qmin ...) flip on rounding-level
        # differences, so the norms of h_diabatic and qi agree to ~1e-9 only
        assert samp < 1e-10 and l2 < 1e-8, (k, samp, l2)


def test_golden_fixtures_are_self_consistent():
    """The fp32 and fp64 reference runs agree to the fp32 noise level and
    contain no NaN (a corrupted fixture would fail here first)."""
    r64, r32 = load_npz("small_ref64.npz"), load_npz("small_ref32.npz")
    assert set(r64) == set(r32)
    for k in r64:
        assert np.isfinite(r64[k]).sum() > 0.9 * r64[k].size, k
        assert rel_l2(r32[k], r64[k]) < 1e-3, k


def _bdy_records(bdy, n=3):
    # the records of make_golden.bdy_records: record r scales the values by
    # 1 + 0.002 r and the tendencies by 1 + 0.5 r
    return {k: np.stack([np.asarray(v)[0] * ((1.0 + 0.5 * r) if "_BT" in k else (1.0 + 0.002 * r))
                         for r in range(n)]).astype(np.asarray(v).dtype) for k, v in bdy.items()}


def test_oracle64_reloads_boundary_records_as_the_reference():
    """With a boundary interval of 2 steps and three distinct records, the
    reference reloads every boundary array from record 1 before step 3
    (solver.py:457-703); the oracle, doing the same, matches its fields after
    4 steps, and a run that keeps record 0 does not."""
    import dataclasses

    spec = synthetic.CaseSpec(**SMALL)
    g = dataclasses.replace(synthetic.grid_for(spec), bdy_interval=2)
    inputs, bdy = synthetic.build(spec)
    ref = load_npz("small_bdyrec_ref64.npz")
    m = OracleModel(g, inputs, _bdy_records(bdy), np.float64)
    m.run(4)
    out = pick(lambda k: m.st[k])
    # 4 float64 steps: 1e-9 .. 7e-8 (mu) from the reference's operation order
    for k in ("u", "v", "t", "ph", "mu", "qv"):
        assert rel_l2(out[k], ref[k]) < 1e-6, k
    # the fixture sees the reload: the same run on record 0 throughout is off
    # by 3e-3 .. 4e-2
    same = {k: np.stack([np.asarray(v)[0]] * 3) for k, v in _bdy_records(bdy).items()}
    m0 = OracleModel(g, inputs, same, np.float64)
    m0.run(4)
    for k in ("u", "mu"):
        assert rel_l2(pick(lambda kk: m0.st[kk])[k], ref[k]) > 1e-3, k


def test_oracle32_reloads_boundary_records_within_reference_fp32_error():
    """The float32 oracle on the boundary-record case stays within the
    reference's own float32 error (against its float64 run)."""
    import dataclasses

    spec = synthetic.CaseSpec(**SMALL)
    g = dataclasses.replace(synthetic.grid_for(spec), bdy_interval=2)
    inputs, bdy = synthetic.build(spec)
    r64, r32 = load_npz("small_bdyrec_ref64.npz"), load_npz("small_bdyrec_ref32.npz")
    m = OracleModel(g, inputs, _bdy_records(bdy), np.float32)
    m.run(4)
    out = pick(lambda k: m.st[k])
    for k in ("u", "v", "t", "ph", "mu", "qv"):
        floor = rel_l2(r32[k], r64[k])
        assert rel_l2(out[k], r64[k]) <= 2.5 * floor + 1e-9, (k, rel_l2(out[k], r64[k]), floor)


def test_theta_bias_fixture_pinned_by_the_oracle(small_case):
    """The adjoint configuration's check on the 28x28x16 case
    (tests/golden/thbias_ref64.npz, from the reference with a bias added to
    the theta tendency after rk_addtend_dry): the oracle reproduces the
    reference's loss at zero bias, and its central differences in the bias at
    an interior point and at a specified-row point (where spec_bdytend
    overwrites the tendency: zero) equal the reference's."""
    g, inputs, bdy = small_case
    Z = load_npz("thbias_ref64.npz")
    R = (slice(0, 10), slice(g.jds, g.jde - 1), slice(g.ids, g.ide - 1))

    def loss(bias):
        m = OracleModel(g, inputs, bdy, np.float64, theta_bias=bias)
        m.run(2)
        return float(((m.st["t"][R] - Z["target_t"]) ** 2).mean() + ((m.st["moist"][1][R] - Z["target_qv"]) ** 2).mean())

    zero = np.zeros((g.nz, g.ny, g.nx))
    assert abs(loss(zero) - float(Z["loss0"])) <= 1e-10 * abs(float(Z["loss0"]))
    eps = 1e-3
    for n in (0, 1):
        k, j, i = (int(x) for x in Z["points"][n])
        bp, bm = zero.copy(), zero.copy()
        bp[k, j, i], bm[k, j, i] = eps, -eps
        fd = (loss(bp) - loss(bm)) / (2 * eps)
        ref = float(Z["fd"][n])
        assert abs(fd - ref) <= 1e-4 * abs(ref) + 1e-12, (n, fd, ref)
    assert float(Z["fd"][1]) == 0.0 and int(Z["points"][1][2]) == g.ide - 2
