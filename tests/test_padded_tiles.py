"""Padded t / y tiles: when a tile's line group is narrower than a shared-memory wavefront,
one padding row follows every R rows of the tile (R the radix of the last forward stage).
The arithmetic does not depend on the layout, so tiles of 1, 2 and 4 lines (padded) give
the same fields as tiles of 16 lines (unpadded), on power-of-two and radix-3 time axes,
in both precisions, and the FP64 result still matches the oracle."""
import numpy as np
import pytest

import cuopo3d_b200 as co
from golden_cases import rel_l2
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def tuning(t, x, y):
    return {k: dict(zip(("threads", "tile", "r1"), v)) for k, v in (("t", t), ("x", x), ("y", y))}


def base_kw(nx, ny, nt):
    return dict(nx=nx, ny=ny, nt=nt, nz=4, LX=300.0, LY=250.0, Lcr=3000.0, P=400.0, w0=40.0, FWHM=3.0,
                t_window=25.0, pump_mode="focused-pulsed", gdd_gamma=0.6, Rs=0.9, total_rt=3)


def run(cfg, tun, nrt=2, seed=5):
    params, _ = co.derive(cfg)
    _, w = co.time_freq(cfg.nt, params.t_window)
    sim = co.Simulation(params, w)
    sim.set_tuning(tun)
    sim.set_plane_pass(0)
    sim.init_fields(cfg, seed, 0.02, idler_copy=True)
    sim.run_round_trips(nrt)
    out = [sim.get_field(k) for k in (co.FIELD_AP, co.FIELD_AS, co.FIELD_AI)]
    sim.synchronize()
    return sim, out


@pytest.mark.parametrize("prec,tol", [(co.FP64, 1e-13), (co.FP32, 1e-6)])
@pytest.mark.parametrize("nt", [128, 96, 48])
def test_padded_tiles_equal_unpadded(prec, tol, nt):
    nx = ny = 16
    cfg = co.make_config(precision=prec, **base_kw(nx, ny, nt))
    _, ref = run(cfg, tuning((128, 16 * nt, 4), (128, 2048, 8), (128, 16 * ny, 8)))
    for lines in (1, 2, 4):
        tun = tuning((128, lines * nt, 4), (128, 2048, 8), (128, lines * ny, 8))
        sim, got = run(cfg, tun)
        assert sim.tuning["t"]["tile"] == lines * nt and sim.tuning["y"]["tile"] == lines * ny
        for a, b in zip(got, ref):
            assert np.all(np.isfinite(a))
            assert rel_l2(a, b) < tol, (lines, rel_l2(a, b))


def test_padded_tiles_match_oracle_fp64():
    kw = base_kw(16, 16, 96)
    cfg = co.make_config(precision=co.FP64, **kw)
    _, got = run(cfg, tuning((128, 2 * 96, 4), (128, 2048, 8), (128, 2 * 16, 8)))
    st = po.Setup(po.make_phys(**kw))
    api = st.api_complex()
    s0 = co.noise(5, 0.02, api.size).reshape(api.shape)
    ref = po.round_trips(st, api, api, s0, s0, 2)
    for a, c in zip(got, ref):
        assert rel_l2(a, c) < 1e-10
