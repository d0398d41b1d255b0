"""The allocation-free tally entry point (opo_field_sums_noalloc), for callers that
cannot call cudaMalloc (hosts whose own allocator has reserved the device memory, loops
that cannot afford an allocation's implicit synchronisation).  Its output must equal the
allocating entry point's (opo_field_sums) within the tallies' FP64 tolerance, on two
calls in a row (the shared scratch array keeps the previous call's contents), and it must
reject sizes beyond its fixed capacity.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

import cuopo3d_b200 as co

pytestmark = pytest.mark.gpu

CAPACITY = 65536 * 4096


def noalloc_sums(ptrs, n, precision, stream=0):
    out = np.zeros(3)
    rc = co.lib().opo_field_sums_noalloc(ctypes.c_void_p(ptrs[0]), ctypes.c_void_p(ptrs[1]),
                                         ctypes.c_void_p(ptrs[2]), n, precision,
                                         ctypes.c_void_p(stream), co._dptr(out))
    return rc, out


@pytest.mark.parametrize("precision", [co.FP64, co.FP32])
def test_noalloc_matches_allocating_entry_point(precision):
    torch = pytest.importorskip("torch")
    nx, ny, nt = 64, 32, 96
    V = nx * ny * nt
    cfg = co.make_config(nx=nx, ny=ny, nt=nt, nz=4, precision=precision)
    params, _ = co.derive(cfg)
    _, w = co.time_freq(nt, params.t_window)
    sim = co.Simulation(params, w)
    dtype = torch.complex128 if precision == co.FP64 else torch.complex64
    for call in range(2):
        fields = [torch.from_numpy(co.noise(100 * call + k + 1, 0.5 + k, V)).to(dtype).cuda()
                  for k in range(3)]
        for which, t in zip((co.FIELD_AP, co.FIELD_AS, co.FIELD_AI), fields):
            sim.set_field_device(which, t.data_ptr(), precision)
        ref = sim.field_sums()
        torch.cuda.synchronize()
        rc, got = noalloc_sums([t.data_ptr() for t in fields], V, precision)
        assert rc == co.OPO_OK
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=0)


def test_noalloc_rejects_sizes_beyond_capacity():
    torch = pytest.importorskip("torch")
    t = torch.zeros(8, dtype=torch.complex128, device="cuda")
    p = t.data_ptr()
    rc, _ = noalloc_sums([p, p, p], CAPACITY + 1, co.FP64)
    assert rc == co.OPO_ERR_CAPACITY
    rc, out = noalloc_sums([p, p, p], 8, co.FP64)
    assert rc == co.OPO_OK and np.all(out == 0)


def test_noalloc_messages_nonfinite_and_many_chunks():
    """More chunks than blocks (each block strides over several 8,192-value chunks), two
    calls in a row against the allocating entry point; a NaN gives OPO_ERR_NONFINITE like
    opo_field_sums; a rejected size leaves a message readable through
    opo_noalloc_last_error and a good call clears it."""
    torch = pytest.importorskip("torch")
    V = 1024 * 8192 + 12345  # 1,026 chunks over 1,024 blocks
    for call in range(2):
        fields = [torch.from_numpy(co.noise(7 * call + k + 1, 1.0 + k, V)).to(torch.complex64).cuda()
                  for k in range(3)]
        rc, got = noalloc_sums([t.data_ptr() for t in fields], V, co.FP32)
        assert rc == co.OPO_OK
        assert co.lib().opo_noalloc_last_error() == b""
        ref = [float(np.sum(np.abs(t.cpu().numpy().astype(np.complex128)) ** 2)) for t in fields]
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=0)
    fields[1][12345] = float("nan")
    rc, _ = noalloc_sums([t.data_ptr() for t in fields], V, co.FP32)
    assert rc == co.OPO_ERR_NONFINITE
    assert b"non-finite" in co.lib().opo_noalloc_last_error()
    p = fields[0].data_ptr()
    rc, _ = noalloc_sums([p, p, p], CAPACITY + 1, co.FP32)
    assert rc == co.OPO_ERR_CAPACITY
    assert b"capacity" in co.lib().opo_noalloc_last_error()
