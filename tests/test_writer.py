"""Output files (opo_save_fields): the reference's text dumps of a field -- NT (x, y) slice
files and NX NY time-trace files, "_r.dat" / "_i.dat" pairs at 20 significant digits
(Files.cuh:73-211 as cuOPO3D.cu:75-85 calls them) -- and the one-file binary form, written
from one device-to-host copy.  Every file is read back and compared with opo_get_field."""
import numpy as np
import pytest

import cuopo3d_b200 as co

pytestmark = pytest.mark.gpu


def solver(precision, nx=12, ny=8, nt=24):
    cfg = co.make_config(nx=nx, ny=ny, nt=nt, nz=4, LX=300.0, LY=250.0, Lcr=3000.0, P=400.0, w0=40.0, FWHM=3.0,
                         t_window=25.0, pump_mode="focused-pulsed", precision=precision)
    params, _ = co.derive(cfg)
    _, w = co.time_freq(nt, params.t_window)
    sim = co.Simulation(params, w)
    sim.init_fields(cfg, 3, 0.05)
    sim.run_single_pass()
    return sim


def read_pair(base):
    re = open(str(base) + "_r.dat").read()
    im = open(str(base) + "_i.dat").read()
    return re, im


@pytest.mark.parametrize("precision", [co.FP64, co.FP32])
def test_text_slices_and_traces_hold_the_field(tmp_path, precision):
    sim = solver(precision)
    nt, ny, nx = sim.shape
    sim.save_fields(co.FIELD_AS, tmp_path / "OutputSignal_slice", tmp_path / "As_temporal_x_")
    ref = sim.get_field(co.FIELD_AS)  # FP32 values widened exactly
    for t in range(nt):
        re, im = read_pair(tmp_path / f"OutputSignal_slice{t}")
        for text, part in ((re, ref[t].real), (im, ref[t].imag)):
            rows = text.split("\n")
            assert rows[-1] == "" and len(rows) == ny + 1
            for y in range(ny):
                assert rows[y].endswith("\t")
                vals = rows[y][:-1].split("\t")
                assert len(vals) == nx
                assert np.array_equal(np.array(vals, dtype=np.float64), part[y])
                assert vals[0] == "%.20g" % part[y, 0]  # the reference's setprecision(20) digits
    for x in range(nx):
        for y in range(ny):
            re, im = read_pair(tmp_path / f"As_temporal_x_{x}_y_{y}")
            assert np.array_equal(np.array(re.split(), dtype=np.float64), ref[:, y, x].real)
            assert np.array_equal(np.array(im.split(), dtype=np.float64), ref[:, y, x].imag)
    assert len(list(tmp_path.iterdir())) == 2 * (nt + nx * ny)


@pytest.mark.parametrize("precision", [co.FP64, co.FP32])
def test_binary_field_file(tmp_path, precision):
    sim = solver(precision, nx=16, ny=16, nt=32)
    for which in (co.FIELD_AP, co.FIELD_AS, co.FIELD_AI):
        sim.save_fields(which, tmp_path / f"field{which}", binary=True)
        hdr, a = co.read_field_file(tmp_path / f"field{which}.bin")
        assert hdr == dict(version=1, nx=16, ny=16, nt=32, bytes=16 if precision == co.FP64 else 8, which=which)
        assert np.array_equal(a.astype(np.complex128), sim.get_field(which))


def test_bad_arguments_rejected(tmp_path):
    sim = solver(co.FP32)
    for args in ((co.FIELD_AS, None, None, co.FILES_TEXT), (7, str(tmp_path / "a"), None, co.FILES_TEXT),
                 (co.FIELD_AS, None, str(tmp_path / "a"), co.FILES_BINARY),
                 (co.FIELD_AS, str(tmp_path / "no_such_dir" / "a"), None, co.FILES_BINARY)):
        enc = [a.encode() if isinstance(a, str) else a for a in args]
        assert co.lib().opo_save_fields(sim.handle, *enc) == co.OPO_ERR_INVALID
