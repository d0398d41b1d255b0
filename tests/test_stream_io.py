"""Streamed round trips (opo_stream_put / opo_stream_run / opo_stream_get /
opo_stream_wait): a host feeding one solver step after step, with the uploads of the next
step and the downloads of the last one on copy streams while the round trips run.  Every
step's results must equal, bit for bit, the blocking set_field / run_round_trips /
get_field sequence on the same inputs, with all steps enqueued before any is waited for;
misuse is refused."""
import ctypes

import numpy as np
import pytest
import torch

import cuopo3d_b200 as co

pytestmark = pytest.mark.gpu

KW = dict(nx=32, ny=16, nt=64, nz=5, LX=300.0, LY=300.0, Lcr=3000.0, P=300.0, w0=40.0, FWHM=3.0, t_window=25.0,
          pump_mode="focused-pulsed", gdd_gamma=0.7, Rs=0.9, total_rt=20)
IN = (co.FIELD_API, co.FIELD_AS, co.FIELD_AI)
OUT = (co.FIELD_AP, co.FIELD_AS, co.FIELD_AI)


def solver(precision):
    cfg = co.make_config(precision=precision, **KW)
    params, _ = co.derive(cfg)
    _, w = co.time_freq(cfg.nt, params.t_window)
    return cfg, co.Simulation(params, w)


def step_inputs(cfg, k):
    api = co.pump_field(cfg) * (1.0 + 0.1 * k)
    s = co.noise(40 + k, 0.02, api.size).reshape(api.shape)
    i = co.noise(80 + k, 0.01, api.size).reshape(api.shape)
    return api, s, i


@pytest.mark.parametrize("precision", [co.FP64, co.FP32])
def test_streamed_steps_equal_blocking_steps(precision):
    steps = 4
    cfg, ref = solver(precision)
    expect = []
    for k in range(steps):
        for which, a in zip(IN, step_inputs(cfg, k)):
            ref.set_field(which, a)
        ref.run_round_trips(2)
        expect.append([ref.get_field(w) for w in OUT])
    ref.close()

    dt = torch.complex128 if precision == co.FP64 else torch.complex64
    _, sim = solver(precision)
    ins = [[torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).to(dt).pin_memory() for a in step_inputs(cfg, k)]
           for k in range(steps)]
    outs = [[torch.zeros(cfg.nt * cfg.ny * cfg.nx, dtype=dt).pin_memory() for _ in OUT] for _ in range(steps)]
    for k in range(steps):  # everything enqueued before the first wait
        for which, t in zip(IN, ins[k]):
            sim.stream_put(which, t.data_ptr())
        sim.stream_run(2)
        for which, t in zip(OUT, outs[k]):
            sim.stream_get(which, t.data_ptr())
    sim.stream_wait()
    assert sim.round_trip_index == 2 * steps
    for k in range(steps):
        for got, want in zip(outs[k], expect[k]):
            g = got.numpy().reshape(want.shape).astype(np.complex128)
            w = want if precision == co.FP64 else want.astype(np.complex64).astype(np.complex128)
            assert np.array_equal(g, w), k
    sim.close()


def test_stream_misuse_is_refused():
    cfg, sim = solver(co.FP64)
    buf = torch.zeros(cfg.nt * cfg.ny * cfg.nx, dtype=torch.complex128).pin_memory()
    with pytest.raises(co.OpoError):
        sim.stream_get(co.FIELD_AS, buf.data_ptr())  # no run yet
    # host data in the other precision
    assert co.lib().opo_stream_put(sim.handle, co.FIELD_AS, ctypes.c_void_p(buf.data_ptr()), co.FP32) == co.OPO_ERR_INVALID
    sim.close()
