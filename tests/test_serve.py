"""Served form (opo_serve): requests admitted as slots and memory free up, resident
instances advanced together, retired on steady state, round-trip limit or non-finite
fields.  Each result is the same alone and in the mix (bit-identical: a slot's
arithmetic and its FP64 tally order do not depend on the other slots)."""
import numpy as np
import pytest

import cuopo3d_b200 as co

pytestmark = pytest.mark.gpu

GRIDS = [(16, 16, 32), (24, 24, 48), (32, 32, 64)]


def request(k, total_rt, tol=0.0, **over):
    nx, ny, nt = GRIDS[k % len(GRIDS)]
    kw = dict(nx=nx, ny=ny, nt=nt, nz=5, LX=300.0, LY=300.0, Lcr=3000.0, FWHM=3.0, t_window=25.0,
              pump_mode="focused-pulsed", P=100.0 + 40.0 * k, w0=35.0 + 3.0 * k, detuning=0.1 * k,
              total_rt=total_rt, precision=co.FP32)
    kw.update(over)
    return dict(cfg=co.make_config(**kw), arrival_s=0.0, seed=10 + k, noise_sigma=0.01, tol=tol)


def test_results_same_alone_and_in_mix():
    reqs = [request(k, total_rt=2 + k % 4) for k in range(7)]
    mixed, st = co.serve(reqs, co.FP32, capacity=3, hbm_budget=8 << 30, realtime=False)
    assert all(r["status"] == co.OPO_OK for r in mixed)
    assert st["max_resident"] <= 3 and st["completed"] == 7
    for k, r in enumerate(reqs):
        alone, _ = co.serve([r], co.FP32, capacity=1, hbm_budget=8 << 30, realtime=False)
        assert alone[0]["round_trips"] == mixed[k]["round_trips"] == 2 + k % 4
        assert np.array_equal(alone[0]["power"], mixed[k]["power"])


def test_matches_standalone_solver():
    r = request(1, total_rt=3)
    res, _ = co.serve([r], co.FP32, capacity=2, hbm_budget=8 << 30, realtime=False)
    params, _ = co.derive(r["cfg"])
    _, w = co.time_freq(r["cfg"].nt, params.t_window)
    sim = co.Simulation(params, w)
    sim.set_tuning({"t": dict(threads=128, tile=2048, r1=4), "x": dict(threads=128, tile=2048, r1=8),
                    "y": dict(threads=128, tile=2048, r1=8)})
    sim.init_fields(r["cfg"], r["seed"], r["noise_sigma"])
    sim.run_round_trips(3)
    np.testing.assert_allclose(res[0]["power"], sim.field_sums(), rtol=1e-12)


def test_budget_limits_residency():
    reqs = [request(2, total_rt=2) for _ in range(5)]
    one = 4 * 8 * 32 * 32 * 64 + (1 << 20)
    res, st = co.serve(reqs, co.FP32, capacity=8, hbm_budget=2 * one + 1000, realtime=False)
    assert all(r["status"] == co.OPO_OK for r in res)
    assert st["max_resident"] <= 2


def test_faulty_requests_answered_others_unaffected():
    good = request(0, total_rt=2)
    bad_grid = request(1, total_rt=2, nx=5)                      # malformed
    nan_req = dict(request(2, total_rt=3), noise_sigma=float("nan"))  # fields not finite
    res, _ = co.serve([good, bad_grid, nan_req, request(0, total_rt=2)], co.FP32, capacity=4,
                      hbm_budget=8 << 30, realtime=False)
    assert res[0]["status"] == co.OPO_OK and res[3]["status"] == co.OPO_OK
    assert res[1]["status"] == co.OPO_ERR_INVALID
    assert res[2]["status"] == co.OPO_ERR_NONFINITE and res[2]["round_trips"] == 1
    assert np.array_equal(res[0]["power"], res[3]["power"])
    too_big, _ = co.serve([request(2, total_rt=2)], co.FP32, capacity=1, hbm_budget=1 << 20, realtime=False)
    assert too_big[0]["status"] == co.OPO_ERR_CAPACITY


def test_steady_state_retirement():
    r = request(0, total_rt=50, tol=1.0)  # any change below 100 % counts as steady
    res, _ = co.serve([r], co.FP32, capacity=1, hbm_budget=8 << 30, realtime=False)
    assert res[0]["status"] == co.OPO_OK and res[0]["round_trips"] == 2


def test_realtime_arrivals_admitted_after_arrival():
    reqs = [dict(request(k, total_rt=2), arrival_s=0.05 * k) for k in range(4)]
    res, st = co.serve(reqs, co.FP32, capacity=4, hbm_budget=8 << 30, realtime=True)
    for r, q in zip(res, reqs):
        assert r["status"] == co.OPO_OK
        assert r["admit_s"] >= q["arrival_s"] and r["latency_s"] > 0
    assert st["p99_latency_s"] >= st["p50_latency_s"] > 0


def test_budget_between_fields_and_fields_plus_tables_is_answered():
    """A budget above the request's fields but below fields + tables (the 1 MiB a batch
    charges per instance for plans and tables) cannot ever admit it: the request is
    answered with OPO_ERR_CAPACITY instead of waiting for a retirement that cannot come."""
    r = request(2, total_rt=2)
    fields = 4 * 8 * 32 * 32 * 64
    res, st = co.serve([r, request(0, total_rt=2)], co.FP32, capacity=2, hbm_budget=fields + (512 << 10),
                       realtime=False)
    assert res[0]["status"] == co.OPO_ERR_CAPACITY
    assert res[1]["status"] == co.OPO_OK  # 16 x 16 x 32: 256 KiB of fields + 1 MiB fit
    assert st["completed"] == 1


def test_requests_with_other_step_counts_wait_for_the_batch_to_drain():
    """All resident instances share one round-trip graph, so a request with another number
    of z-steps waits until the resident ones have retired, then runs (not rejected)."""
    reqs = [request(0, total_rt=2), request(1, total_rt=2, nz=7), request(2, total_rt=2)]
    res, st = co.serve(reqs, co.FP32, capacity=3, hbm_budget=8 << 30, realtime=False)
    assert all(x["status"] == co.OPO_OK for x in res)
    assert res[1]["admit_s"] >= res[0]["done_s"]
    alone, _ = co.serve([reqs[1]], co.FP32, capacity=1, hbm_budget=8 << 30, realtime=False)
    assert np.array_equal(alone[0]["power"], res[1]["power"])


C5_GRIDS = [(64, 64, 128), (96, 96, 192), (128, 128, 256)]


def c5_request(k, total_rt):
    nx, ny, nt = C5_GRIDS[k % len(C5_GRIDS)]
    cfg = co.make_config(nx=nx, ny=ny, nt=nt, nz=5, LX=800.0, LY=800.0, Lcr=2000.0, FWHM=2.0, t_window=40.0,
                         pump_mode="focused-pulsed", P=1.0 + 3.0 * k, w0=40.0 + 5.0 * k, detuning=0.2 * k,
                         total_rt=total_rt, precision=co.FP32)
    return dict(cfg=cfg, arrival_s=0.0, seed=50 + k, noise_sigma=1e-3, tol=0.0, return_fields=True)


def test_served_fields_same_alone_and_in_mix_on_c5_grids():
    """The served form's grids (64^2 x 128, 96^2 x 192 with its radix-3 transforms,
    128^2 x 256): every request's final pump, signal and idler fields -- not only its
    tallies -- are the same bit for bit alone and in a mix where requests of other grids
    join and retire around it, and equal a standalone solver's."""
    reqs = [c5_request(k, 2 + k % 3) for k in range(6)]
    mixed, st = co.serve(reqs, co.FP32, capacity=4, hbm_budget=8 << 30, realtime=False)
    assert st["completed"] == 6 and st["max_resident"] == 4
    for k, r in enumerate(reqs):
        alone, _ = co.serve([r], co.FP32, capacity=1, hbm_budget=8 << 30, realtime=False)
        assert alone[0]["round_trips"] == mixed[k]["round_trips"] == 2 + k % 3
        for a, b in zip(alone[0]["fields"], mixed[k]["fields"]):
            assert np.array_equal(a, b), k
    # request 1 (96^2 x 192) against a standalone solver with the batch's kernel variants
    r = reqs[1]
    params, _ = co.derive(r["cfg"])
    _, w = co.time_freq(r["cfg"].nt, params.t_window)
    sim = co.Simulation(params, w)
    sim.set_tuning({"t": dict(threads=128, tile=2048, r1=4), "x": dict(threads=128, tile=2048, r1=8),
                    "y": dict(threads=128, tile=2048, r1=8)})
    sim.set_plane_pass(0)
    sim.init_fields(r["cfg"], r["seed"], r["noise_sigma"])
    sim.run_round_trips(mixed[1]["round_trips"])
    for which, f in zip((co.FIELD_AP, co.FIELD_AS, co.FIELD_AI), mixed[1]["fields"]):
        assert np.array_equal(sim.get_field(which), f)
