"""Fused (x, y) diffraction plane pass (thread-block clusters with distributed shared
memory) against the separate x and y passes and the FP64 oracle: every cluster size,
CTA size and first-stage radix, square and non-square grids, radix-3 axes, the crystal
step and the free-space return (signal and idler only), FP64 and FP32."""
import numpy as np
import pytest

import cuopo3d_b200 as co
from golden_cases import rel_l2
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def make(nx, ny, nt, prec, **over):
    kw = dict(nx=nx, ny=ny, nt=nt, nz=4, LX=300.0, LY=250.0, Lcr=3000.0, P=400.0, w0=40.0, FWHM=3.0,
              t_window=25.0, pump_mode="focused-pulsed", gdd_gamma=0.6, Rs=0.9, total_rt=3)
    kw.update(over)
    return kw, co.make_config(precision=prec, **kw)


def run(cfg, plane, nrt=2, seed=4):
    params, _ = co.derive(cfg)
    _, w = co.time_freq(cfg.nt, params.t_window)
    sim = co.Simulation(params, w)
    if plane is not None:
        sim.set_plane_pass(*plane)
    sim.init_fields(cfg, seed, 0.02, idler_copy=True)
    sim.run_round_trips(nrt)
    return sim, [sim.get_field(k) for k in (co.FIELD_AP, co.FIELD_AS, co.FIELD_AI)]


def oracle(kw, cfg, nrt=2, seed=4):
    kw = dict(kw)
    st = po.Setup(po.make_phys(**kw))
    api = st.api_complex()
    s0 = co.noise(seed, 0.02, api.size).reshape(api.shape)
    return po.round_trips(st, api, api, s0, s0, nrt)


VARIANTS = [(2, 256, 8), (4, 256, 8), (8, 256, 4), (4, 512, 8), (2, 512, 4), (8, 512, 8)]


@pytest.mark.parametrize("K,threads,r1", VARIANTS)
def test_plane_variants_fp64_equal_separate_passes_and_oracle(K, threads, r1):
    kw, cfg = make(32, 32, 64, co.FP64)
    sim, got = run(cfg, (K, threads, r1))
    assert sim.plane_pass["cluster"] == K
    _, sep = run(cfg, (0,))
    ref = oracle(kw, cfg)
    for a, b, c in zip(got, sep, ref):
        assert rel_l2(a, b) < 1e-13
        assert rel_l2(a, c) < 1e-10


@pytest.mark.parametrize("nx,ny,nt", [(16, 8, 32), (24, 48, 32), (96, 32, 16), (64, 128, 16)])
def test_plane_non_square_and_radix3_fp64(nx, ny, nt):
    kw, cfg = make(nx, ny, nt, co.FP64)
    for K in (2, 4, 8):
        if nx % K or ny % K:
            continue
        sim, got = run(cfg, (K, 256, 8))
        ref = oracle(kw, cfg)
        for a, c in zip(got, ref):
            assert rel_l2(a, c) < 1e-10, (K, rel_l2(a, c))


@pytest.mark.parametrize("K,threads,r1", [(2, 256, 16), (4, 256, 8), (4, 512, 16), (8, 256, 4)])
def test_plane_variants_fp32(K, threads, r1):
    kw, cfg = make(64, 64, 32, co.FP32)
    sim, got = run(cfg, (K, threads, r1))
    assert sim.plane_pass["cluster"] == K
    _, sep = run(cfg, (0,))
    kw64, cfg64 = make(64, 64, 32, co.FP64)
    _, ref = run(cfg64, (0,))
    for a, b, c in zip(got, sep, ref):
        assert rel_l2(a, b) < 2e-6
        assert rel_l2(a, c) < 1e-5


def test_plane_last_round_trip_and_resume():
    """The free-space plane pass runs on signal and idler only and is skipped on the run's
    last round trip: 2 + 1 round trips equal 3 at once and match the oracle."""
    kw, cfg = make(32, 16, 32, co.FP64, total_rt=3)
    sim_a, got_a = run(cfg, (4, 256, 8), nrt=3)
    params, _ = co.derive(cfg)
    _, w = co.time_freq(cfg.nt, params.t_window)
    sim = co.Simulation(params, w)
    sim.set_plane_pass(4, 256, 8)
    sim.init_fields(cfg, 4, 0.02, idler_copy=True)
    sim.run_round_trips(2)
    sim.run_round_trips(1)
    got_b = [sim.get_field(k) for k in (co.FIELD_AP, co.FIELD_AS, co.FIELD_AI)]
    for a, b in zip(got_a, got_b):
        assert np.array_equal(a, b)
    ref = oracle(kw, cfg, nrt=3)
    for a, c in zip(got_a, ref):
        assert rel_l2(a, c) < 1e-10


def test_plane_rejects_bad_configurations_and_keeps_current():
    _, cfg = make(24, 16, 16, co.FP64)
    params, _ = co.derive(cfg)
    _, w = co.time_freq(cfg.nt, params.t_window)
    sim = co.Simulation(params, w)
    sim.set_plane_pass(4, 256, 8)
    for bad in ((3, 256, 8), (4, 384, 8), (16, 256, 8)):  # cluster size, CTA size, cluster size
        with pytest.raises(co.OpoError) as e:
            sim.set_plane_pass(*bad)
        assert e.value.code == co.OPO_ERR_INVALID
        assert sim.plane_pass == dict(cluster=4, threads=256, r1=8)
    _, cfg2 = make(12, 12, 16, co.FP64)
    params2, _ = co.derive(cfg2)
    _, w2 = co.time_freq(cfg2.nt, params2.t_window)
    sim2 = co.Simulation(params2, w2)
    with pytest.raises(co.OpoError):
        sim2.set_plane_pass(8, 256, 8)  # 12 is not a multiple of 8
    sim2.set_plane_pass(0)
    assert sim2.plane_pass["cluster"] == 0


def test_autotune_keeps_faster_diffraction():
    _, cfg = make(64, 64, 64, co.FP64)
    params, _ = co.derive(cfg)
    _, w = co.time_freq(cfg.nt, params.t_window)
    sim = co.Simulation(params, w)
    sim.autotune()
    pp = sim.plane_pass
    assert pp["cluster"] in (0, 2, 4, 8)
    sim.init_fields(cfg, 4, 0.02, idler_copy=True)
    sim.run_round_trips(1)
    assert np.isfinite(sim.field_sums()).all()
