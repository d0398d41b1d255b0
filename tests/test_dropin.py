"""Drop-in headers (src/headers): a program written against cuOPO3D's headers -- its
cuOPO3D.cu, unchanged -- compiles against them and links to libcuopo3d.so (CPU test,
needs the reference checkout), and the binary built by __graft_entry__.build() runs on a
GPU and writes the same fields as the library called directly (GPU test)."""
import glob
import os
import subprocess

import numpy as np
import pytest

import cuopo3d_b200 as co
from oracle.refharness.locate import reference_root

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_MAIN = os.path.join(reference_root(), "src", "cuOPO3D.cu")
DEMO = os.path.join(ROOT, "src", "_build", "cuOPO3D_g16")
DEMO_FLAGS = ["-DOPO_NX=16", "-DOPO_NT=32", "-DOPO_NZ=12", "-DOPO_NRT=3"]


@pytest.mark.skipif(not os.path.exists(REF_MAIN), reason="reference checkout not present")
def test_reference_main_compiles_unchanged(tmp_path):
    out = tmp_path / "cuOPO3D"
    subprocess.run([os.path.join(ROOT, "src", "build_dropin.sh"), REF_MAIN, str(out)] + DEMO_FLAGS, check=True,
                   capture_output=True)
    assert out.exists() and os.access(out, os.X_OK)


@pytest.mark.skipif(not os.path.exists(REF_MAIN), reason="reference checkout not present")
@pytest.mark.parametrize("crystal", ["ZGP", "MgOPPLN"])
def test_reference_main_other_crystals_compile(tmp_path, crystal):
    """The reference main with its crystal switched the way its own comments show
    (cuOPO3D.cu:21-23: the ZGP alternative with a polarisation tuple; MgOPPLN takes
    MgOsPPLT's constructor arguments)."""
    src = open(REF_MAIN).read()
    if crystal == "ZGP":
        src = src.replace("MgOsPPLT * cr1 = new MgOsPPLT(LX, LY, Lcr, T, Lambda, lp, ls, li);", "")
        src = src.replace("// std::tuple<char, char, char> pol", "std::tuple<char, char, char> pol")
        src = src.replace("// ZGP * cr1 = new ZGP(", "ZGP * cr1 = new ZGP(")
    src = src.replace("MgOsPPLT", crystal)
    main = tmp_path / "main.cu"
    main.write_text(src)
    out = tmp_path / "cuOPO3D"
    r = subprocess.run([os.path.join(ROOT, "src", "build_dropin.sh"), str(main), str(out)] + DEMO_FLAGS,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    assert out.exists() and os.access(out, os.X_OK)


def read_slice(path):
    re_ = np.loadtxt(path + "_r.dat")
    im = np.loadtxt(path + "_i.dat")
    return re_ + 1j * im


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(DEMO), reason="drop-in demo binary not built")
def test_dropin_binary_runs_and_matches_library(tmp_path):
    r = subprocess.run([DEMO, "500", "31"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "criteria: passed" in r.stdout
    slices = sorted(glob.glob(str(tmp_path / "OutputSignalPower_PumpPower500_W_slice*_r.dat")))
    traces = glob.glob(str(tmp_path / "As_temporal_x_*_r.dat"))
    assert len(slices) == 32 and len(traces) == 16 * 16
    # the same run through the library: MgOsPPLT 29 mm, Lcav = 4 Lcr, R = 0.98, GDD 100 %,
    # 0.5 W focused CW pump, 31 um waist, seeded noise (seed 1, 1e-15), idler = signal
    cfg = co.make_config(crystal="mgosplt", LX=1e3, LY=1e3, Lcr=29e3, T=27.0, Lambda=6.97, lp=0.532, ls=1.064,
                         nx=16, ny=16, nt=32, nz=12, Lcav=4 * 29e3, Rs=0.98, gdd_gamma=1.0, P=0.5, FWHM=0.2,
                         w0=31.0, focal=29e3 / 2, pump_mode="focused-cw", zloop_f32=1, total_rt=3,
                         precision=co.FP32)
    params, _ = co.derive(cfg)
    _, w = co.time_freq(cfg.nt, params.t_window)
    sim = co.Simulation(params, w)
    api = co.pump_field(cfg)
    s0 = co.noise(1, 1e-15, api.size).reshape(api.shape)
    for which, arr in ((co.FIELD_API, api), (co.FIELD_AP, api), (co.FIELD_AS, s0), (co.FIELD_AI, s0)):
        sim.set_field(which, arr)
    sim.run_round_trips(3)
    As = sim.get_field(co.FIELD_AS)
    # every slice file and every pixel's trace file (written from one host snapshot of As)
    files = np.zeros_like(As)
    for t in range(32):
        files[t] = read_slice(str(tmp_path / f"OutputSignalPower_PumpPower500_W_slice{t}"))
        assert np.linalg.norm(files[t] - As[t]) <= 1e-4 * np.linalg.norm(As[t])
    for x in range(16):
        for y in range(16):
            base = str(tmp_path / f"As_temporal_x_{x}_y_{y}")
            tr = np.loadtxt(base + "_r.dat") + 1j * np.loadtxt(base + "_i.dat")
            assert np.array_equal(tr, files[:, y, x])  # the traces hold the slices' values
