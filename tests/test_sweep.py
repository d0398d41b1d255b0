"""Threshold sweeps (opo_sweep) and per-round-trip FP64 tallies with the reference's NaN
probe (opo_run_round_trips_tallied, Solver3D.cuh:999-1005).

The scan is the reference's main use case (cuOPO3D.sh:58-80 runs one OPO per pump power
and waist; saveAppendedValues2Columns, Files.cuh:215-233, records the power pairs).  On
the configuration below the signal's round-trip gain crosses 1 between 10 and 30 W (the
oracle gives 0.906 at 10 W and 1.053 at 30 W), and at 3 kW the fields blow up within the
run, which the NaN probe must catch."""
import numpy as np
import pytest

import cuopo3d_b200 as co
from golden_cases import rel_l2
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

BASE = dict(nx=16, ny=16, nt=32, nz=6, LX=300.0, LY=300.0, Lcr=4000.0, w0=40.0, FWHM=4.0, t_window=30.0,
            pump_mode="focused-cw", Rs=0.9, total_rt=12, precision=co.FP64)
TUNING = {"t": dict(threads=128, tile=1024, r1=4), "x": dict(threads=128, tile=1024, r1=8),
          "y": dict(threads=128, tile=1024, r1=8)}
POWERS = [1.0, 10.0, 20.0, 30.0, 100.0, 3000.0]
RT, SEED, SIGMA = 12, 40, 1e-3


def standalone(P, seed):
    cfg = co.make_config(**dict(BASE, P=P))
    params, _ = co.derive(cfg)
    _, w = co.time_freq(cfg.nt, params.t_window)
    sim = co.Simulation(params, w)
    sim.set_tuning(TUNING)
    sim.set_plane_pass(0)
    sim.init_fields(cfg, seed, SIGMA)
    return sim


def test_tallied_round_trips_equal_field_sums():
    """Each round trip's tallies equal the FP64 sums of the fields it leaves, and the run
    is the same as untallied round trips."""
    sim = standalone(30.0, 7)
    t, rc = sim.run_round_trips_tallied(4)
    assert rc == co.OPO_OK and t.shape == (4, 3)
    ref = standalone(30.0, 7)
    for k in range(4):
        ref.run_round_trips(1)
        np.testing.assert_array_equal(t[k], ref.field_sums())
    for which in (co.FIELD_AP, co.FIELD_AS, co.FIELD_AI):
        assert np.array_equal(sim.get_field(which), ref.get_field(which))


def test_tallied_round_trips_stop_at_first_nonfinite():
    sim = standalone(3000.0, 7)
    t, rc = sim.run_round_trips_tallied(RT)
    assert rc == co.OPO_ERR_NONFINITE
    n = len(t)
    assert 1 <= n < RT and sim.round_trip_index == n  # stopped where the probe fired
    assert np.all(np.isfinite(t[:-1])) and not np.all(np.isfinite(t[-1]))
    assert b"round trip" in co.lib().opo_last_error(sim.handle)


def test_sweep_points_equal_standalone_runs_and_bracket_threshold(tmp_path):
    base = co.make_config(**BASE)
    pts, tallies = co.sweep(base, POWERS, [40.0] * len(POWERS), RT, window=4, seed=SEED, noise_sigma=SIGMA,
                            capacity=4, tuning=TUNING)  # capacity 4: two waves
    for k, (P, pt) in enumerate(zip(POWERS, pts)):
        sim = standalone(P, SEED + k)
        t, rc = sim.run_round_trips_tallied(RT)
        assert pt["round_trips"] == len(t)
        assert np.array_equal(tallies[k, :len(t)], t, equal_nan=True), P
        if P < 1000:
            assert pt["status"] == co.OPO_OK and rc == co.OPO_OK
            assert np.array_equal(pt["sums"], t[-1])
            g = (t[-1, 1] / t[-1 - 4, 1]) ** 0.25
            assert pt["gain"] == pytest.approx(g, rel=1e-12) and pt["above"] == (g > 1)
            cfg = co.make_config(**dict(BASE, P=P))
            assert pt["output_power"] == pytest.approx(co.power_cut_xy(cfg, t[-1])[1] * (1 - 0.9), rel=1e-14)
        else:
            assert pt["status"] == co.OPO_ERR_NONFINITE and rc == co.OPO_ERR_NONFINITE and len(t) < RT
    gains = [p["gain"] for p in pts[:-1]]
    assert all(a < b for a, b in zip(gains, gains[1:]))  # parametric gain grows with the pump
    lo, hi, est = co.sweep_threshold(pts)
    assert lo in (10.0, 20.0) and hi == 30.0 and lo < est < hi
    path = tmp_path / "Average_power_Waist_40.txt"
    co.sweep_write(path, pts)
    rows = [ln.split("\t") for ln in open(path).read().splitlines()]
    assert [float(r[0]) for r in rows] == POWERS[:-1]


def test_sweep_point_matches_oracle():
    """One point of the sweep against the FP64 oracle: the signal tally of every round trip."""
    base = co.make_config(**BASE)
    pts, tallies = co.sweep(base, [30.0], [40.0], 5, window=2, seed=SEED, noise_sigma=SIGMA, tuning=TUNING)
    kw = {k: v for k, v in dict(BASE, P=30.0, total_rt=5).items() if k != "precision"}
    st = po.Setup(po.make_phys(**kw))
    api = st.api_complex()
    s = co.noise(SEED, SIGMA, api.size).reshape(api.shape)
    ap, i = api.copy(), np.zeros_like(s)
    for r in range(5):
        ap, s, i = po.round_trips(st, api, ap, s, i, 1)
        assert abs(tallies[0, r, 1] / np.sum(np.abs(s) ** 2) - 1) < 1e-10
    assert rel_l2(np.array([tallies[0, -1, 0]]), np.array([np.sum(np.abs(ap) ** 2)])) < 1e-10
