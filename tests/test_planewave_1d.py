"""Plane-wave 1-D solver (the reference's Solver1D.cuh / EFields1D.cuh / Cavity1D.cuh,
which do not compile as shipped): nx = ny = 1 without diffraction, the 1-D pump
amplitude, and the intracavity electro-optic modulator (EOM) -- on the 1-D and on the
3-D path -- against the FP64 oracle; batches of 1-D instances against standalone ones."""
import numpy as np
import pytest

import cuopo3d_b200 as co
from golden_cases import rel_l2
from oracle import pyoracle as po

FLAGS_1D = co.DISPERSION


def kw_1d(nt, **over):
    kw = dict(nx=1, ny=1, nt=nt, nz=20, LX=1.0, LY=1.0, Lcr=10000.0, P=2.0, w0=40.0, FWHM=1.0, t_window=20.0,
              pump_mode="waveplane-pulsed", gdd_gamma=0.8, Rs=0.95, total_rt=4, flags=FLAGS_1D)
    kw.update(over)
    return kw


def test_1d_configuration_rules():
    # 1-D needs the (x, y) step off; nx = 2 is not a grid either way
    with pytest.raises(co.OpoError):
        co.derive(co.make_config(**kw_1d(256, flags=co.DISPERSION | co.DIFFRACTION)))
    with pytest.raises(co.OpoError):
        co.derive(co.make_config(**kw_1d(256, nx=2, ny=2)))
    p, sc = co.derive(co.make_config(**kw_1d(256)))
    assert p.nx == 1 and p.ny == 1 and sc["dx"] == 0 and sc["dy"] == 0
    # 1-D pump amplitude sqrt(2P/(eps0 c pi np w0^2)) (EFields1D.cuh:145-148) at the pulse peak
    cfg = co.make_config(**kw_1d(256, pump_mode="waveplane-cw"))
    api = co.pump_field(cfg)
    eps0, c = 8.8541878128E-12 * 1E12 / 1E6, 299792458 * 1E6 / 1E12
    a0 = np.sqrt(2 * 2.0 / (eps0 * c * np.pi * sc["np"] * 40.0 ** 2))
    assert np.allclose(np.abs(api), a0, rtol=1e-14)
    # the oracle builds the same pump; focused modes do not exist in 1-D
    st = po.Setup(po.make_phys(**kw_1d(256, pump_mode="waveplane-pulsed")))
    api_l = co.pump_field(co.make_config(**kw_1d(256, pump_mode="waveplane-pulsed")))
    assert rel_l2(api_l, st.api_complex()) < 1e-14
    with pytest.raises(co.OpoError):
        co.pump_field(co.make_config(**kw_1d(256, pump_mode="focused-cw")))


def run_lib(cfg, seed, nrt, tuning=None):
    params, _ = co.derive(cfg)
    _, w = co.time_freq(cfg.nt, params.t_window)
    sim = co.Simulation(params, w)
    if tuning:
        sim.set_tuning(tuning)
    sim.init_fields(cfg, seed, 1e-3, idler_copy=True)
    sim.run_round_trips(nrt)
    return [sim.get_field(k) for k in (co.FIELD_AP, co.FIELD_AS, co.FIELD_AI)]


def run_oracle(kw, seed, nrt):
    st = po.Setup(po.make_phys(**kw))
    api = st.api_complex()
    s0 = co.noise(seed, 1e-3, api.size).reshape(api.shape)
    return po.round_trips(st, api, api, s0, s0, nrt)


@pytest.mark.gpu
@pytest.mark.parametrize("nt", [256, 2048, 4096])
@pytest.mark.parametrize("eom", [(0.0, 0.0), (0.6, 0.05)])
def test_1d_round_trips_fp64_vs_oracle(nt, eom):
    kw = kw_1d(nt, eom_beta=eom[0], eom_fpm=eom[1])
    got = run_lib(co.make_config(precision=co.FP64, **kw), 3, 4)
    ref = run_oracle(kw, 3, 4)
    for a, b in zip(got, ref):
        assert rel_l2(a, b) < 1e-10


@pytest.mark.gpu
def test_1d_eom_changes_the_result_and_physics_flag():
    kw = kw_1d(1024, eom_beta=0.6, eom_fpm=0.05, flags=co.DISPERSION | co.PHYSICS, Lambda=6.5)
    got = run_lib(co.make_config(precision=co.FP64, **kw), 5, 3)
    ref = run_oracle(kw, 5, 3)
    ref0 = run_oracle(dict(kw, eom_beta=0.0), 5, 3)
    for a, b in zip(got, ref):
        assert rel_l2(a, b) < 1e-10
    assert rel_l2(ref[1], ref0[1]) > 1e-3


@pytest.mark.gpu
def test_1d_fp32_long_time_axis():
    """FP32 with nt = 8192 (one tile of the three fields per CTA) against FP64."""
    kw = kw_1d(8192, eom_beta=0.3, eom_fpm=0.1)
    got = run_lib(co.make_config(precision=co.FP32, **kw), 7, 3)
    ref = run_oracle(kw, 7, 3)
    for a, b in zip(got, ref):
        assert rel_l2(a, b) < 1e-5


@pytest.mark.gpu
def test_eom_on_the_3d_path_vs_oracle():
    kw = dict(nx=16, ny=16, nt=64, nz=5, LX=300.0, LY=300.0, Lcr=3000.0, P=400.0, w0=40.0, FWHM=2.0, t_window=20.0,
              pump_mode="focused-pulsed", gdd_gamma=0.5, Rs=0.9, total_rt=3, eom_beta=0.4, eom_fpm=0.08)
    got = run_lib(co.make_config(precision=co.FP64, **kw), 9, 3)
    ref = run_oracle(kw, 9, 3)
    for a, b in zip(got, ref):
        assert rel_l2(a, b) < 1e-10


@pytest.mark.gpu
def test_batch_of_1d_instances_equals_standalone():
    tuning = {"t": dict(threads=128, tile=1024, r1=4), "x": dict(threads=128, tile=1024, r1=8),
              "y": dict(threads=128, tile=1024, r1=8)}
    b = co.Batch(co.FP64, 8, 1 << 30, tuning=tuning)
    cfgs = [co.make_config(precision=co.FP64, **kw_1d(1024, P=p, eom_beta=beta, eom_fpm=0.05))
            for p, beta in ((1.0, 0.0), (2.0, 0.5), (4.0, 0.2), (3.0, 0.0))]
    slots = []
    for k, c in enumerate(cfgs):
        s = b.add(c)
        b.init_fields(s, c, 20 + k, 1e-3, idler_copy=True)
        slots.append(s)
    b.run_round_trips(3)
    for k, (s, c) in enumerate(zip(slots, cfgs)):
        solo = run_lib(c, 20 + k, 3, tuning)
        for w_, ref in zip((co.FIELD_AP, co.FIELD_AS, co.FIELD_AI), solo):
            assert np.array_equal(b.get_field(s, w_), ref)
