"""Batched form (opo_batch_*): many instances with uneven grids and parameters advanced
by one persistent launch per pass.  Every slot must give exactly what a standalone
solver with the same kernel configuration gives (bit-identical: the same kernels run
the same arithmetic on the slot's tiles), be the same alone and mixed with others, and
match the FP64 oracle; admission respects the HBM budget; slots can leave and join
between round trips."""
import numpy as np
import pytest

import cuopo3d_b200 as co
from golden_cases import rel_l2
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

TUNING = {"t": dict(threads=128, tile=1024, r1=4), "x": dict(threads=128, tile=1024, r1=8),
          "y": dict(threads=128, tile=1024, r1=8)}

BASE = dict(nz=5, LX=300.0, LY=300.0, Lcr=3000.0, FWHM=3.0, t_window=25.0, pump_mode="focused-pulsed",
            total_rt=3, precision=co.FP64)
INSTANCES = [
    dict(nx=16, ny=16, nt=32, P=300.0, w0=40.0, gdd_gamma=1.0),
    dict(nx=32, ny=16, nt=64, P=150.0, w0=60.0, detuning=0.7, Rs=0.9),
    dict(nx=24, ny=24, nt=48, P=500.0, w0=35.0, detuning=-1.2),
    dict(nx=32, ny=32, nt=96, P=80.0, w0=50.0, gdd_gamma=0.5, flags=co.DISPERSION | co.DIFFRACTION | co.PHYSICS,
         Lambda=6.5),
]


def cfg_of(inst, **over):
    kw = dict(BASE)
    kw.update(inst)
    kw.update(over)
    return co.make_config(**kw)


def seed_of(k):
    return 100 + k


def run_solo(cfg, seed, nrt):
    params, _ = co.derive(cfg)
    _, w = co.time_freq(cfg.nt, params.t_window)
    sim = co.Simulation(params, w)
    sim.set_tuning(TUNING)
    sim.set_plane_pass(0)  # the batched kernels run the x and y passes
    sim.init_fields(cfg, seed, 0.02, idler_copy=True)
    sim.run_round_trips(nrt)
    return [sim.get_field(k) for k in (co.FIELD_AP, co.FIELD_AS, co.FIELD_AI)]


def make_batch(cap=8, budget=8 << 30):
    return co.Batch(co.FP64, cap, budget, tuning=TUNING)


def test_device_init_matches_host_pump_and_noise():
    cfg = cfg_of(INSTANCES[2])
    params, _ = co.derive(cfg)
    _, w = co.time_freq(cfg.nt, params.t_window)
    sim = co.Simulation(params, w)
    sim.init_fields(cfg, 7, 0.02)
    api = sim.get_field(co.FIELD_API)
    assert rel_l2(api, co.pump_field(cfg)) < 1e-13
    s = sim.get_field(co.FIELD_AS)
    assert np.array_equal(s.ravel(), co.noise(7, 0.02, s.size))
    assert not np.any(sim.get_field(co.FIELD_AI))


def test_batch_slots_equal_standalone_and_oracle():
    b = make_batch()
    slots = []
    for k, inst in enumerate(INSTANCES):
        cfg = cfg_of(inst)
        s = b.add(cfg)
        b.init_fields(s, cfg, seed_of(k), 0.02, idler_copy=True)
        slots.append((s, cfg))
    b.run_round_trips(3)
    for k, (s, cfg) in enumerate(slots):
        got = [b.get_field(s, w) for w in (co.FIELD_AP, co.FIELD_AS, co.FIELD_AI)]
        solo = run_solo(cfg, seed_of(k), 3)
        for a, c in zip(got, solo):
            assert np.array_equal(a, c)
        # FP64 oracle on the same inputs
        kw = dict(BASE)
        kw.update(INSTANCES[k])
        kw.pop("precision")
        st = po.Setup(po.make_phys(**kw))
        api = st.api_complex()
        s0 = co.noise(seed_of(k), 0.02, api.size).reshape(api.shape)
        ref = po.round_trips(st, api, api, s0, s0, 3)
        for a, c in zip(got, ref):
            assert rel_l2(a, c) < 1e-10


def test_instance_alone_equals_instance_in_mix():
    cfg = cfg_of(INSTANCES[1])
    b1 = make_batch()
    s1 = b1.add(cfg)
    b1.init_fields(s1, cfg, 5, 0.02, idler_copy=True)
    b1.run_round_trips(2)
    alone = b1.get_field(s1, co.FIELD_AS)
    b2 = make_batch()
    for k in (0, 2, 3):
        c = cfg_of(INSTANCES[k])
        s = b2.add(c)
        b2.init_fields(s, c, seed_of(k), 0.02)
    s2 = b2.add(cfg)
    b2.init_fields(s2, cfg, 5, 0.02, idler_copy=True)
    b2.run_round_trips(2)
    assert np.array_equal(alone, b2.get_field(s2, co.FIELD_AS))


def test_admission_respects_budget_and_slots():
    cfg = cfg_of(INSTANCES[3])
    b = co.Batch(co.FP64, 2, 1 << 20, tuning=TUNING)  # 1 MiB: nothing fits
    with pytest.raises(co.OpoError) as e:
        b.add(cfg)
    assert e.value.code == co.OPO_ERR_CAPACITY
    b = co.Batch(co.FP64, 1, 8 << 30, tuning=TUNING)
    b.add(cfg)
    with pytest.raises(co.OpoError) as e:
        b.add(cfg)
    assert e.value.code == co.OPO_ERR_CAPACITY
    st = b.stats()
    assert st["instances"] == 1 and st["used"] <= st["budget"]


def test_slots_leave_and_join_between_round_trips():
    b = make_batch()
    ca, cb, cc = cfg_of(INSTANCES[0]), cfg_of(INSTANCES[1]), cfg_of(INSTANCES[2])
    sa = b.add(ca)
    b.init_fields(sa, ca, 1, 0.02, idler_copy=True)
    sb = b.add(cb)
    b.init_fields(sb, cb, 2, 0.02, idler_copy=True)
    b.run_round_trips(1)
    b.remove(sb)
    sc = b.add(cc)
    b.init_fields(sc, cc, 3, 0.02, idler_copy=True)
    b.run_round_trips(2)
    assert b.info(sa)["round_trips"] == 3 and b.info(sc)["round_trips"] == 2
    assert np.array_equal(b.get_field(sa, co.FIELD_AS), run_solo(ca, 1, 3)[1])
    assert np.array_equal(b.get_field(sc, co.FIELD_AS), run_solo(cc, 3, 2)[1])


def test_per_slot_last_round_trip_and_tallies():
    """Slots with different run lengths: each skips the free-space return on its own last
    round trip (Solver3D.cuh:987); batched FP64 tallies equal the per-field sums."""
    b = make_batch()
    ca = cfg_of(INSTANCES[0], total_rt=2)
    cb = cfg_of(INSTANCES[1], total_rt=4)
    sa = b.add(ca)
    b.init_fields(sa, ca, 1, 0.02, idler_copy=True)
    sb = b.add(cb)
    b.init_fields(sb, cb, 2, 0.02, idler_copy=True)
    b.run_round_trips(2)
    fa = b.get_field(sa, co.FIELD_AS)
    assert np.array_equal(fa, run_solo(ca, 1, 2)[1])
    b.remove(sa)
    b.run_round_trips(2)
    fields = [b.get_field(sb, w) for w in (co.FIELD_AP, co.FIELD_AS, co.FIELD_AI)]
    assert np.array_equal(fields[1], run_solo(cb, 2, 4)[1])
    sums = b.sums()
    for k in range(3):
        ref = float(np.sum(np.abs(fields[k]) ** 2))
        assert abs(sums[sb, k] - ref) <= 1e-12 * ref
    assert np.all(sums[sa] == 0)


def test_incompatible_grid_rejected():
    b = make_batch()
    with pytest.raises(co.OpoError):
        b.add(cfg_of(dict(nx=12, ny=12, nt=24, P=10.0, w0=40.0)))  # 12 has no radix-8 first stage


def c4_instances(n=9, seed=2024):
    """Instances over the batched form's grid set, N x N x NT with N in {32, 64, 128} and
    NT in {64, 128, 256} (every pair once), P log-uniform 0.5-20 W, waist U[30, 100] um,
    detuning U[-pi, pi]; a 2 mm crystal over a 1600 um window in 4 slices keeps the
    oracle's run to seconds (the 128 x 128 x 256 instances dominate)."""
    rng = np.random.default_rng(seed)
    pairs = [(N, NT) for N in (32, 64, 128) for NT in (64, 128, 256)][:n]
    out = []
    for N, NT in pairs:
        out.append(dict(nx=N, ny=N, nt=NT, nz=4, LX=1600.0, LY=1600.0, Lcr=2000.0, t_window=40.0,
                        P=float(np.exp(rng.uniform(np.log(0.5), np.log(20.0)))), w0=float(rng.uniform(30, 100)),
                        detuning=float(rng.uniform(-np.pi, np.pi)), FWHM=2.0, focal=1000.0, Rs=0.98,
                        alpha=(2e-7, 2e-7, 2e-7), pump_mode="focused-pulsed", total_rt=2))
    return out


@pytest.mark.parametrize("precision,tol", [(co.FP64, 1e-10), (co.FP32, 1e-5)])
def test_batch_c4_grid_set_vs_oracle(precision, tol):
    """Every grid of the batched form's set in one batch (FP64: the plain form, FP32: the
    precision form) against the FP64 oracle on the same inputs, two round trips; once
    with the generic t-pass and once with the line-specialised one (one batched kernel
    per line body: the time axes 64, 128 and 256 of the set), the setting the batch tuner
    picks for the C4 mix."""
    insts = c4_instances()
    generic = TUNING if precision == co.FP64 else {"t": dict(threads=128, tile=2048, r1=8),
                                                   "x": dict(threads=128, tile=2048, r1=8),
                                                   "y": dict(threads=128, tile=2048, r1=16)}
    line_t = dict(threads=128, tile=512, r1=4 + co.LINE) if precision == co.FP64 else \
        dict(threads=128, tile=2048, r1=16 + co.LINE)
    refs = []
    for k, kw in enumerate(insts):
        st = po.Setup(po.make_phys(**kw))
        api = st.api_complex()
        s0 = co.noise(300 + k, 0.01, api.size).reshape(api.shape)
        refs.append(po.round_trips(st, api, api, s0, np.zeros_like(s0), 2))
    for tuning in (generic, {**generic, "t": line_t}):
        b = co.Batch(precision, len(insts), 16 << 30, tuning=tuning)
        slots = []
        for k, kw in enumerate(insts):
            cfg = co.make_config(precision=precision, **kw)
            s = b.add(cfg)
            b.init_fields(s, cfg, 300 + k, 0.01)
            slots.append(s)
        b.run_round_trips(2)
        for k, kw in enumerate(insts):
            got = [b.get_field(slots[k], w) for w in (co.FIELD_AP, co.FIELD_AS, co.FIELD_AI)]
            for name, a, c in zip(("Ap", "As", "Ai"), got, refs[k]):
                assert rel_l2(a, c) < tol, (tuning["t"], kw["nx"], kw["nt"], name, rel_l2(a, c))
        b.close()


@pytest.mark.parametrize("mode", sorted(co.PUMP_MODES))
@pytest.mark.parametrize("precision,tol", [(co.FP64, 1e-13), (co.FP32, 1e-6)])
def test_device_init_every_pump_mode(mode, precision, tol):
    """Device field initialisation (init_fields.cu) against the host pump (opo_pump_field,
    EFields3D.cuh:72-137, 244-296, plus the sech^2 modes) for every mode, on a 3-D grid and,
    for the plane-wave modes, the 1-D solver's grid (nx = ny = 1, EFields1D.cuh:143-170)."""
    grids = [(24, 16, 48)] + ([(1, 1, 256)] if mode.startswith("waveplane") else [])
    for nx, ny, nt in grids:
        flags = co.DISPERSION | (co.DIFFRACTION if nx > 1 else 0)
        cfg = co.make_config(nx=nx, ny=ny, nt=nt, nz=4, LX=300.0, LY=300.0, Lcr=3000.0, P=120.0, w0=35.0,
                             FWHM=3.0, t_window=25.0, pump_mode=mode, flags=flags, precision=precision)
        params, _ = co.derive(cfg)
        _, w = co.time_freq(cfg.nt, params.t_window)
        sim = co.Simulation(params, w)
        sim.init_fields(cfg, 11, 0.01)
        for which in (co.FIELD_API, co.FIELD_AP):
            assert rel_l2(sim.get_field(which), co.pump_field(cfg)) < tol, (mode, nx, which)
        s = sim.get_field(co.FIELD_AS).ravel()
        ref = co.noise(11, 0.01, s.size)
        assert rel_l2(s, ref) < (0 if precision == co.FP64 else 1e-7) or np.array_equal(s, ref)
        sim.close()
