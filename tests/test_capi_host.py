"""CPU tests of the C-ABI library: it loads, exports every entry point declared in
include/cuopo3d.h, and its host physics (the reference constructors, grids, pump and
noise) matches the reference fixtures and the oracle.  No GPU needed."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import cuopo3d_b200 as co
from golden_cases import Golden, fixture_names, rel_l2
from oracle import pyoracle as po

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "cuopo3d.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(opo_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = co.lib()
    names = declared_symbols()
    assert len(names) >= 16
    for n in names:
        assert hasattr(L, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", co.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (opo_[a-z0-9_]+)", out))
    assert set(names) <= exported


def test_version_string():
    assert co.lib().opo_version().startswith(b"cuopo3d-b200")


@pytest.mark.parametrize("name", fixture_names())
def test_host_physics_matches_reference(name):
    g = Golden(name)
    kw = g.config_kwargs()
    flags = co.DISPERSION | co.DIFFRACTION | ((co.ASIS_Q1 | co.ASIS_Q2) if g.asis else 0)
    cfg = co.make_config(flags=flags, precision=co.FP64, **kw)
    params, sc = co.derive(cfg)
    tol = 1e-12 if g.fp64 else 2e-6
    for k, v in sc.items():
        ref = g.scalars[k]
        assert abs(v - ref) <= tol * abs(ref) or (ref == 0 and abs(v) < 1e-15), (k, v, ref)
    t, w = co.time_freq(g.nt, params.t_window)
    assert rel_l2(t, g.t) < (1e-13 if g.fp64 else 1e-6)
    assert rel_l2(w, g.w) < (1e-13 if g.fp64 else 1e-6)
    api = co.pump_field(cfg)
    assert rel_l2(api[g.tidx], g.Api) < (1e-12 if g.fp64 else 1e-6)


def test_noise_matches_oracle_bitwise():
    a = co.noise(12345, 1e-6, 5000)
    b = po.noise(12345, 1e-6, 5000)
    assert np.array_equal(a, b)
    assert abs(np.std(co.noise(7, 1.0, 100000).real) - 1.0) < 0.01


@pytest.mark.parametrize("mode", list(co.PUMP_MODES))
def test_pump_modes_match_oracle(mode):
    kw = dict(nx=16, ny=12, nt=24, nz=5, P=3.0, FWHM=1.5, w0=40.0, t_window=10.0, pump_mode=mode)
    api = co.pump_field(co.make_config(**kw))
    st = po.Setup(po.make_phys(**kw))
    assert rel_l2(api, st.api_complex()) < 1e-13


def test_sech2_average_power():
    """sech^2 envelope: the window average of the on-axis power equals P."""
    kw = dict(nx=8, ny=8, nt=512, nz=5, P=1.0, FWHM=2.0, w0=50.0, t_window=20.0,
              pump_mode="waveplane-sech2")
    api = co.pump_field(co.make_config(**kw))
    prof = np.abs(api[:, 4, 4]) ** 2
    peak = prof.max()
    # average of sech^2 over the window relative to its peak: 2 ts / T
    ts = 2.0 / (2 * np.arccosh(np.sqrt(2.0)))
    assert abs(prof.mean() / peak - 2 * ts / 20.0) < 1e-3


def test_crystal_dispersion_api():
    out = np.zeros(4)
    assert co.lib().opo_crystal_dispersion(0, 27.0, 1.064, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 0
    assert 2.1 < out[0] < 2.2 and 130 < out[1] < 140 and out[2] > 0
    assert co.lib().opo_crystal_dispersion(9, 27.0, 1.064, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) != 0


@pytest.mark.parametrize("bad", [dict(nx=2), dict(nt=0), dict(nz=1), dict(ls=0.4), dict(crystal=7),
                                 dict(precision=3), dict(nx=2048, ny=2048, nt=1024)])  # 2^32 voxels
def test_invalid_configs_rejected(bad):
    with pytest.raises(co.OpoError):
        co.derive(co.make_config(**bad))


def test_largest_volume_accepted():
    """2^31 - 1 voxels is the largest grid the 32-bit field indexing takes."""
    p, _ = co.derive(co.make_config(nx=1024, ny=1024, nt=2047))
    assert p.nx * p.ny * p.nt < 2 ** 31


def test_zloop_step_counts():
    """Step counts of the reference's float loop (Solver3D.cuh:949) for the benchmark crystals."""
    for Lcr, nz, f32, expect in ((5000.0, 50, 1, 49), (20000.0, 100, 1, 100), (29000.0, 100, 1, 99)):
        _, sc = co.derive(co.make_config(Lcr=Lcr, nz=nz, zloop_f32=f32))
        assert sc["nsteps"] == expect
        assert po.lib().or_zloop_steps(Lcr, Lcr / (nz - 1.0), f32) == expect


def test_power_cut_xy_formula():
    """opo_power_cut_xy: the reference's averagePowerCutXY (Solver3D.cuh:527-536),
    0.5 eps0 c ns dx dy / (LX LY) sum |A|^2, with its constants (DtypesConsts.cuh:55-57)."""
    cfg = co.make_config(nx=32, ny=16, nt=64, nz=5, LX=400.0, LY=300.0, P=2.0)
    _, sc = co.derive(cfg)
    sums = np.array([3.0, 0.25, 1e-3])
    c_um_ps = 299792458 * 1e6 / 1e12
    eps0 = 8.8541878128e-12 * 1e12 / 1e6
    want = 0.5 * eps0 * c_um_ps * sc["ns"] * sc["dx"] * sc["dy"] / (400.0 * 300.0) * sums
    np.testing.assert_allclose(co.power_cut_xy(cfg, sums), want, rtol=1e-14)


def _pt(P, gain, status=0, out_p=1.0):
    return dict(P=P, w0=40.0, status=status, round_trips=12, sums=[0, 0, 0], power_xy=[0, 0, 0],
                output_power=out_p, gain=gain, above=gain > 1)


def test_sweep_threshold_bracket_and_estimate():
    pts = [_pt(30.0, 1.05), _pt(1.0, 0.90), _pt(10.0, 0.95), _pt(100.0, 2.5), _pt(3000.0, float("nan"), status=4)]
    lo, hi, est = co.sweep_threshold(pts)
    assert (lo, hi) == (10.0, 30.0)
    # ln g linear between the bracket: ln 0.95 + (ln 1.05 - ln 0.95) (P - 10) / 20 = 0
    want = 10.0 + 20.0 * (0 - np.log(0.95)) / (np.log(1.05) - np.log(0.95))
    assert est == pytest.approx(want, rel=1e-12) and lo < est < hi
    assert co.sweep_threshold([_pt(1.0, 0.9), _pt(2.0, 0.95)]) is None  # never crosses


def test_sweep_write_reference_format(tmp_path):
    """'value1 <tab> value2' lines in default stream formatting (saveAppendedValues2Columns,
    Files.cuh:218-233), completed points only, appended."""
    path = tmp_path / "Average_power_Waist_40.txt"
    pts = [_pt(10.0, 0.95, out_p=1.25e-7), _pt(30.0, 1.05, out_p=0.125), _pt(50.0, 1.2, status=4)]
    co.sweep_write(path, pts, append=True)
    co.sweep_write(path, pts[:1], append=True)
    assert open(path).read() == "10\t1.25e-07\n30\t0.125\n10\t1.25e-07\n"
    co.sweep_write(path, pts[1:2], append=False)
    assert open(path).read() == "30\t0.125\n"
