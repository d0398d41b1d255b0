"""Line-specialised t-pass (tuning r1 + co.LINE): compiled bodies for the time axes 64,
128 and 256, tiles of 8 FP32 pixels (two per packed f32x2 instruction) or 4 FP64 pixels.
It must match the FP64 oracle within the form's tolerance (FP32 1e-5, FP64 1e-10; round
trips with GDD, mirrors, EOM, the corrected physics with a phase mismatch, the closing
pass's untransformed pump), agree with the generic kernel to rounding, fall back to the
generic kernel with the setting's fallback radix (FP32: its r1, FP64: 4) on grids it does
not cover, and give bit-identical results in a batch and in a standalone solver (the
batched kernel runs the same tile bodies per instance)."""
import numpy as np
import pytest

import cuopo3d_b200 as co
from golden_cases import rel_l2
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

TOL = {co.FP32: 1e-5, co.FP64: 1e-10}
# against the generic kernel: FP32 / FP64 rounding apart
GEN_TOL = {co.FP32: 2e-6, co.FP64: 1e-12}
AXES = {"x": dict(threads=128, tile=1024, r1=8), "y": dict(threads=128, tile=1024, r1=8)}


def tuning(r1, line=True, nt=256):
    return {"t": dict(threads=128, tile=max(nt * 8, 1024), r1=r1 + (co.LINE if line else 0)), **AXES}


def run(grid, over, tun, precision, nrt=2, seed=31):
    nx, ny, nt = grid
    kw = dict(nx=nx, ny=ny, nt=nt, nz=4, LX=300.0, LY=250.0, Lcr=3000.0, P=400.0, w0=40.0, FWHM=3.0, t_window=25.0,
              pump_mode="focused-pulsed", gdd_gamma=0.6, Rs=0.9, total_rt=3, **over)
    flags = kw.pop("flags", co.DISPERSION | co.DIFFRACTION)
    cfg = co.make_config(precision=precision, flags=flags, **kw)
    params, _ = co.derive(cfg)
    _, w = co.time_freq(nt, params.t_window)
    sim = co.Simulation(params, w)
    sim.set_tuning(tun)
    sim.set_plane_pass(0)
    s0 = co.noise(seed, 0.02, nx * ny * nt).reshape(nt, ny, nx)
    api = co.pump_field(cfg)
    for which, arr in ((co.FIELD_API, api), (co.FIELD_AP, api), (co.FIELD_AS, s0), (co.FIELD_AI, s0)):
        sim.set_field(which, arr)
    sim.run_round_trips(nrt)
    out = (sim.get_field(co.FIELD_AP), sim.get_field(co.FIELD_AS), sim.get_field(co.FIELD_AI))
    t = sim.tuning["t"]
    sim.close()
    return out, kw, flags, s0, t


def oracle(kw, flags, s0, nrt=2):
    st = po.Setup(po.make_phys(flags=flags, **kw))
    api = st.api_complex()
    return po.round_trips(st, api, api, s0, s0, nrt)


LINE_CASES = [
    ((32, 32, 256), 16, {}),
    ((16, 8, 128), 16, dict(eom_beta=0.4, eom_fpm=0.05)),
    ((24, 16, 64), 8, {}),
    ((16, 16, 256), 16, dict(flags=co.DISPERSION | co.DIFFRACTION | co.PHYSICS, Lambda=6.5)),
    ((8, 8, 128), 16, dict(flags=co.DISPERSION)),
]


@pytest.mark.parametrize("precision", [co.FP32, co.FP64])
@pytest.mark.parametrize("grid,r1,over", LINE_CASES)
def test_line_tpass_vs_oracle_and_generic(grid, r1, over, precision):
    out, kw, flags, s0, t = run(grid, over, tuning(r1, nt=grid[2]), precision)
    assert t["r1"] == r1 + co.LINE
    for a, b in zip(out, oracle(kw, flags, s0)):
        assert rel_l2(a, b) < TOL[precision]
    # the generic kernel (FP64: its radix-4 register form): the same arithmetic up to
    # rounding, but not bit for bit (so the line kernel is the one that ran)
    gen, *_ = run(grid, over, tuning(4 if precision == co.FP64 else r1, line=False, nt=grid[2]), precision)
    diff = [rel_l2(a, b) for a, b in zip(out, gen)]
    assert max(diff) < GEN_TOL[precision], diff
    assert any(not np.array_equal(a, b) for a, b in zip(out, gen))


@pytest.mark.parametrize("precision", [co.FP32, co.FP64])
@pytest.mark.parametrize("grid,over", [((16, 8, 96), {}), ((6, 8, 128), dict(flags=co.DISPERSION)),
                                       ((16, 16, 256), dict(flags=co.DISPERSION | co.DIFFRACTION | co.ASIS_Q2))])
def test_line_tuning_falls_back_to_generic_kernel(grid, over, precision):
    """Grids without a line body (time axis 96, nx not a multiple of the tile, the shipped
    Q2 launch grid) keep the line setting but run the generic tile body with the fallback
    radix (FP32 the setting's 16, FP64 4 whatever the setting): bit for bit the generic
    kernel's results, and the oracle's within the form's tolerance."""
    out, kw, flags, s0, t = run(grid, over, tuning(16, nt=grid[2]), precision)
    assert t["r1"] == 16 + co.LINE
    for a, b in zip(out, oracle(kw, flags, s0)):
        assert rel_l2(a, b) < TOL[precision]
    gen, *_ = run(grid, over, tuning(4 if precision == co.FP64 else 16, line=False, nt=grid[2]), precision)
    for a, b in zip(out, gen):
        assert np.array_equal(a, b)


def test_line_tpass_full_size_vs_fp64():
    """128 x 128 x 256, the benchmark's physics, one full round trip (100 z-steps): the
    FP32 line t-pass within 1e-5 of the FP64 line t-pass, which is within 1e-12 of the
    generic FP64 kernels."""
    kw = dict(nx=128, ny=128, nt=256, nz=100, LX=800.0, LY=800.0, Lcr=20000.0, t_window=40.0, P=5.0,
              w0=60.0, FWHM=2.0, Rs=0.98, alpha=(-1.0, 2e-7, 2e-7), pump_mode="focused-pulsed",
              gdd_gamma=1.0, total_rt=200)
    tunings = {"fp32": (co.FP32, {"t": dict(threads=128, tile=2048, r1=16 + co.LINE),
                                  "x": dict(threads=128, tile=2048, r1=8), "y": dict(threads=128, tile=2048, r1=16)}),
               "fp64": (co.FP64, {"t": dict(threads=128, tile=1024, r1=16 + co.LINE),
                                  "x": dict(threads=160, tile=1024, r1=8), "y": dict(threads=160, tile=1024, r1=8)}),
               "fp64_generic": (co.FP64, {"t": dict(threads=128, tile=1024, r1=4),
                                          "x": dict(threads=160, tile=1024, r1=8),
                                          "y": dict(threads=160, tile=1024, r1=8)})}
    outs = {}
    for name, (prec, tun) in tunings.items():
        cfg = co.make_config(precision=prec, **kw)
        params, _ = co.derive(cfg)
        _, w = co.time_freq(cfg.nt, params.t_window)
        sim = co.Simulation(params, w)
        sim.set_tuning(tun)
        assert sim.tuning["t"]["r1"] == tun["t"]["r1"]
        sim.init_fields(cfg, 1, 1e-3, idler_copy=True)
        sim.run_round_trips(1)
        outs[name] = [sim.get_field(k) for k in (co.FIELD_AP, co.FIELD_AS, co.FIELD_AI)]
        sim.close()
    for a, b, c in zip(outs["fp32"], outs["fp64"], outs["fp64_generic"]):
        assert rel_l2(a, b) < TOL[co.FP32]
        assert rel_l2(b, c) < 1e-12


@pytest.mark.parametrize("precision", [co.FP32, co.FP64])
def test_line_tpass_batch_equals_standalone(precision):
    """A batch tuned to the line form, with instances on every line axis (256, 128, 64) and
    one without (96: the generic body with the fallback radix in the same launch): every
    slot bit for bit its standalone solver."""
    base = dict(nz=4, LX=300.0, LY=300.0, Lcr=3000.0, FWHM=3.0, t_window=25.0, pump_mode="focused-pulsed",
                total_rt=3, precision=precision)
    insts = [dict(nx=16, ny=16, nt=256, P=300.0, w0=40.0, gdd_gamma=1.0),
             dict(nx=32, ny=16, nt=128, P=150.0, w0=60.0, detuning=0.7, Rs=0.9),
             dict(nx=24, ny=24, nt=128, P=80.0, w0=50.0, flags=co.DISPERSION | co.DIFFRACTION | co.PHYSICS,
                  Lambda=6.5),
             dict(nx=16, ny=32, nt=64, P=200.0, w0=45.0, detuning=0.3),
             dict(nx=16, ny=16, nt=96, P=500.0, w0=35.0, detuning=-1.2)]
    tun = {"t": dict(threads=128, tile=2048, r1=16 + co.LINE), **AXES}
    b = co.Batch(precision, 8, 8 << 30, tuning=tun)
    slots = []
    for k, inst in enumerate(insts):
        cfg = co.make_config(**{**base, **inst})
        s = b.add(cfg)
        b.init_fields(s, cfg, 100 + k, 0.02, idler_copy=True)
        slots.append((s, cfg))
    b.run_round_trips(3)
    for k, (s, cfg) in enumerate(slots):
        got = [b.get_field(s, w) for w in (co.FIELD_AP, co.FIELD_AS, co.FIELD_AI)]
        params, _ = co.derive(cfg)
        _, w = co.time_freq(cfg.nt, params.t_window)
        sim = co.Simulation(params, w)
        sim.set_tuning(tun)
        sim.set_plane_pass(0)
        sim.init_fields(cfg, 100 + k, 0.02, idler_copy=True)
        sim.run_round_trips(3)
        for which, a in zip((co.FIELD_AP, co.FIELD_AS, co.FIELD_AI), got):
            assert np.array_equal(a, sim.get_field(which))
        sim.close()


@pytest.mark.parametrize("precision", [co.FP32, co.FP64])
def test_line_tpass_batch_groups_follow_admission_and_retirement(precision):
    """Under the line setting a batch runs one kernel per line body and one generic
    kernel, each over its group's share of the descriptors: slots admitted and retired
    between round trips move instances in and out of the groups (a group emptied, one
    filled that was empty) without breaking the captured round trip; every surviving slot
    stays bit for bit its standalone solver."""
    base = dict(nz=4, LX=300.0, LY=300.0, Lcr=3000.0, FWHM=3.0, t_window=25.0, pump_mode="focused-pulsed",
                total_rt=4, precision=precision)
    first = [dict(nx=16, ny=16, nt=256, P=300.0, w0=40.0), dict(nx=16, ny=16, nt=96, P=500.0, w0=35.0),
             dict(nx=16, ny=32, nt=64, P=200.0, w0=45.0)]
    later = [dict(nx=32, ny=16, nt=128, P=150.0, w0=60.0, detuning=0.7), dict(nx=16, ny=16, nt=64, P=90.0, w0=30.0)]
    tun = {"t": dict(threads=128, tile=2048, r1=16 + co.LINE), **AXES}
    b = co.Batch(precision, 8, 8 << 30, tuning=tun)
    live = {}
    for k, inst in enumerate(first):
        cfg = co.make_config(**{**base, **inst})
        s = b.add(cfg)
        b.init_fields(s, cfg, 200 + k, 0.02, idler_copy=True)
        live[s] = (cfg, 200 + k, 0)
    b.run_round_trips(1)
    live = {s: (c, seed, n + 1) for s, (c, seed, n) in live.items()}
    # retire the 64-sample instance (its group empties), admit a 128-sample one (a group
    # that was empty) and another 64-sample one
    gone = [s for s, (c, _, _) in live.items() if c.nt == 64][0]
    b.remove(gone)
    del live[gone]
    for k, inst in enumerate(later):
        cfg = co.make_config(**{**base, **inst})
        s = b.add(cfg)
        b.init_fields(s, cfg, 300 + k, 0.02, idler_copy=True)
        live[s] = (cfg, 300 + k, 0)
    b.run_round_trips(2)
    for s, (cfg, seed, n) in live.items():
        got = [b.get_field(s, w) for w in (co.FIELD_AP, co.FIELD_AS, co.FIELD_AI)]
        params, _ = co.derive(cfg)
        _, w = co.time_freq(cfg.nt, params.t_window)
        sim = co.Simulation(params, w)
        sim.set_tuning(tun)
        sim.set_plane_pass(0)
        sim.init_fields(cfg, seed, 0.02, idler_copy=True)
        sim.run_round_trips(n + 2)
        for which, a in zip((co.FIELD_AP, co.FIELD_AS, co.FIELD_AI), got):
            assert np.array_equal(a, sim.get_field(which))
        sim.close()
    b.close()
