"""Warp-specialised passes (a producer warp streaming tiles with TMA into a ring of
shared-memory stages, consumer warps computing): the same results as the classic
kernels and the FP64 oracle on square, non-square, radix-3, long-time-axis and 1-D
grids, in both precisions; variants that do not apply to a grid are refused."""
import numpy as np
import pytest

import cuopo3d_b200 as co
from golden_cases import rel_l2
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def tuning(t, x, y):
    return {"t": dict(zip(("threads", "tile", "r1"), t)), "x": dict(zip(("threads", "tile", "r1"), x)),
            "y": dict(zip(("threads", "tile", "r1"), y))}


def run(cfg, tun, nrt=2, seed=8):
    params, _ = co.derive(cfg)
    _, w = co.time_freq(cfg.nt, params.t_window)
    sim = co.Simulation(params, w)
    sim.set_tuning(tun)
    sim.set_plane_pass(0)
    sim.init_fields(cfg, seed, 0.02, idler_copy=True)
    sim.run_round_trips(nrt)
    out = [sim.get_field(k) for k in (co.FIELD_AP, co.FIELD_AS, co.FIELD_AI)]
    sim.synchronize()  # raises if a pipeline wait had timed out
    return sim, out


def oracle(kw, nrt=2, seed=8):
    st = po.Setup(po.make_phys(**kw))
    api = st.api_complex()
    s0 = co.noise(seed, 0.02, api.size).reshape(api.shape)
    return po.round_trips(st, api, api, s0, s0, nrt)


def base_kw(nx, ny, nt, **over):
    kw = dict(nx=nx, ny=ny, nt=nt, nz=4, LX=300.0, LY=250.0, Lcr=3000.0, P=400.0, w0=40.0, FWHM=3.0,
              t_window=25.0, pump_mode="focused-pulsed", gdd_gamma=0.6, Rs=0.9, total_rt=3)
    kw.update(over)
    return kw


FP64_CASES = [((32, 32, 64), tuning((160, 1024, 4), (160, 1024, 8), (160, 1024, 8))),
              ((64, 32, 128), tuning((288, 2048, 4), (160, 512, 4), (288, 2048, 8))),
              ((24, 48, 96), tuning((160, 1024, 4), (160, 1024, 4), (160, 1024, 8))),
              ((16, 16, 2048), tuning((160, 2048, 4), (160, 1024, 8), (160, 1024, 8)))]


@pytest.mark.parametrize("grid,tun", FP64_CASES)
def test_ws_fp64_equals_classic_and_oracle(grid, tun):
    kw = base_kw(*grid)
    cfg = co.make_config(precision=co.FP64, **kw)
    sim, got = run(cfg, tun)
    assert all(sim.tuning[k]["threads"] in (160, 288) for k in "txy")
    classic = {k: dict(v, threads=v["threads"] - 32) for k, v in tun.items()}
    _, ref_c = run(cfg, classic)
    ref_o = oracle(kw)
    for a, b, c in zip(got, ref_c, ref_o):
        assert rel_l2(a, b) < 1e-13
        assert rel_l2(a, c) < 1e-10


def test_ws_fp32_t_and_y_equal_classic():
    kw = base_kw(64, 64, 128)
    cfg = co.make_config(precision=co.FP32, **kw)
    tun = tuning((160, 2048, 4), (128, 2048, 16), (160, 2048, 16))
    _, got = run(cfg, tun)
    _, ref_c = run(cfg, tuning((128, 2048, 4), (128, 2048, 16), (128, 2048, 16)))
    ref_o = oracle(kw)
    for a, b, c in zip(got, ref_c, ref_o):
        assert rel_l2(a, b) < 1e-6
        assert rel_l2(a, c) < 1e-5


def test_ws_1d_long_time_axis_fp64():
    """One 2048-sample time line per tile, eight tensor boxes per field, two stages."""
    kw = dict(nx=1, ny=1, nt=2048, nz=20, LX=1.0, LY=1.0, Lcr=10000.0, P=2.0, w0=40.0, FWHM=1.0, t_window=20.0,
              pump_mode="waveplane-pulsed", gdd_gamma=0.8, Rs=0.95, total_rt=4, flags=co.DISPERSION,
              eom_beta=0.5, eom_fpm=0.05)
    cfg = co.make_config(precision=co.FP64, **kw)
    _, got = run(cfg, tuning((160, 2048, 4), (128, 1024, 8), (128, 1024, 8)), nrt=3)
    ref = oracle(kw, nrt=3)
    for a, b in zip(got, ref):
        assert rel_l2(a, b) < 1e-10


def test_ws_tables_from_global_memory_fp64():
    """A 1024-point y axis: its twiddles and phase tables (~64 KB) beside the two-stage
    ring would leave one CTA per SM instead of two, so the consumers read them from global
    memory instead of copying them into shared memory; same results as the classic
    kernels and the oracle."""
    kw = base_kw(16, 1024, 16, LY=2000.0, nz=3)
    cfg = co.make_config(precision=co.FP64, **kw)
    tun = tuning((128, 1024, 4), (128, 1024, 8), (160, 1024, 8))
    sim, got = run(cfg, tun)
    assert sim.tuning["y"]["threads"] == 160
    _, ref_c = run(cfg, tuning((128, 1024, 4), (128, 1024, 8), (128, 1024, 8)))
    ref_o = oracle(kw)
    for a, b, c in zip(got, ref_c, ref_o):
        assert rel_l2(a, b) < 1e-13
        assert rel_l2(a, c) < 1e-10


def test_ws_variant_refused_where_it_does_not_apply():
    # FP32 x rows of nx + 1 complex64 are not 16-byte multiples: no warp-specialised x-pass
    cfg = co.make_config(precision=co.FP32, **base_kw(32, 32, 64))
    params, _ = co.derive(cfg)
    _, w = co.time_freq(cfg.nt, params.t_window)
    sim = co.Simulation(params, w)
    before = sim.tuning
    with pytest.raises(co.OpoError):
        sim.set_tuning(dict(before, x=dict(threads=160, tile=2048, r1=8)))
    assert sim.tuning["x"]["threads"] in (128, 256)


@pytest.mark.parametrize("precision", [co.FP64, co.FP32])
def test_wait_expiry_reports_error_and_solver_recovers(precision):
    """The bounded pipeline waits' error path: with a bound of a few clock cycles the
    consumers give up their first ring wait (the producer's tensor / bulk copies take far
    longer), leave together, the producer drains the copies it issued, and the host gets
    OPO_ERR_CUDA at its next synchronisation.  The fields are then lost: reads and runs
    fail until all four are uploaded again; with the default bound restored the same
    solver runs the case again and matches the oracle (the context stays usable)."""
    grid, tun = FP64_CASES[0]
    if precision == co.FP32:  # FP32 rows of 33 complex64 are not 16-byte strided: classic x-pass
        tun = dict(tun, x=dict(threads=128, tile=1024, r1=8))
    kw = base_kw(*grid)
    cfg = co.make_config(precision=precision, **kw)
    params, _ = co.derive(cfg)
    _, w = co.time_freq(cfg.nt, params.t_window)
    sim = co.Simulation(params, w)
    sim.set_tuning(tun)
    sim.set_plane_pass(0)
    assert all(sim.tuning[k]["threads"] == tun[k]["threads"] for k in "txy")
    sim.init_fields(cfg, 8, 0.02, idler_copy=True)
    sim.synchronize()
    sim.set_wait_limit(4)
    sim.run_single_pass()
    with pytest.raises(co.OpoError) as e:
        sim.synchronize()
    assert e.value.code == co.OPO_ERR_CUDA and "timed out" in str(e.value)
    for call in (lambda: sim.get_field(co.FIELD_AS), sim.run_single_pass, sim.field_sums):
        with pytest.raises(co.OpoError) as e:
            call()
        assert e.value.code == co.OPO_ERR_CUDA and "lost" in str(e.value)
    sim.set_wait_limit(0)
    api = co.pump_field(cfg)
    s0 = co.noise(8, 0.02, api.size).reshape(api.shape)
    for which, arr in ((co.FIELD_API, api), (co.FIELD_AP, api), (co.FIELD_AS, s0), (co.FIELD_AI, s0)):
        sim.set_field(which, arr)
    sim.run_round_trips(2)
    got = [sim.get_field(k) for k in (co.FIELD_AP, co.FIELD_AS, co.FIELD_AI)]
    sim.synchronize()
    ref = oracle(kw)
    tol = 1e-10 if precision == co.FP64 else 1e-5
    for a, b in zip(got, ref):
        assert rel_l2(a, b) < tol
