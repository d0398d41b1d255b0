"""cuopo3d_b200 -- B200-native split-step Fourier solver for three coupled chi(2)
fields (pump, signal, idler) in an optical parametric oscillator.

The compute path is the in-tree CUDA library ``libcuopo3d.so`` (sm_100a kernels and
the C-ABI of include/cuopo3d.h).  This module binds that C-ABI with ctypes and mirrors
the reference's classes (alfredos84/cuOPO3D src/headers: crystals, Cavity, EFields,
Solver) so that scripts written against the reference read the same.  There is no
CPU fallback: importing works without a GPU, but creating a solver without the
library or without a CUDA device raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcuopo3d.so")

# status codes
OPO_OK, OPO_ERR_INVALID, OPO_ERR_CUDA, OPO_ERR_NOMEM, OPO_ERR_NONFINITE = 0, 1, 2, 3, 4
OPO_ERR_COURANT, OPO_ERR_CAPACITY = 5, 6
# flags
DISPERSION, DIFFRACTION, PHYSICS, ASIS_Q1, ASIS_Q2, TOD = 1, 2, 4, 8, 16, 32
FP32, FP64 = 0, 1
# added to a t-pass "r1" in a tuning: the line-specialised t-pass (OPO_TUNE_LINE)
LINE = 256
PPLN_ID, MGOSPPLT_ID, MGOPPLN_ID, ZGP_ID = 0, 1, 2, 3
CRYSTALS = {"ppln": PPLN_ID, "mgospplt": MGOSPPLT_ID, "mgosplt": MGOSPPLT_ID, "mgoppln": MGOPPLN_ID,
            "zgp": ZGP_ID}
FIELD_API, FIELD_AP, FIELD_AS, FIELD_AI = 0, 1, 2, 3
MEM_HOST, MEM_DEVICE = 0, 1
FILES_TEXT, FILES_BINARY = 0, 1
PUMP_MODES = {"waveplane-cw": 0, "waveplane-pulsed": 1, "focused-cw": 2, "focused-pulsed": 3,
              "focused-sech2": 4, "waveplane-sech2": 5}
SCALAR_NAMES = ("np ns ni vp vs vi b2p b2s b2i b3p b3s b3i dQ dk dx dy dz kp ks ki "
                "kappa_p kappa_s kappa_i trt dt nsteps").split()

_d = ctypes.c_double
_i = ctypes.c_int
_u = ctypes.c_uint


class OpoConfig(ctypes.Structure):
    _fields_ = [("crystal", _i), ("LX", _d), ("LY", _d), ("Lcr", _d), ("T", _d), ("Lambda", _d),
                ("lp", _d), ("ls", _d), ("nx", _i), ("ny", _i), ("nt", _i), ("nz", _i), ("dQ", _d),
                ("alpha", _d * 3), ("Lcav", _d), ("Rs", _d), ("Ri", _d), ("gdd_gamma", _d),
                ("detuning", _d), ("P", _d), ("FWHM", _d), ("w0", _d), ("focal", _d),
                ("pump_mode", _i), ("t_window", _d), ("flags", _u), ("zloop_f32", _i),
                ("n_steps", _i), ("total_rt", _i), ("precision", _i), ("resonant", _u), ("pol", _u),
                ("eom_beta", _d), ("eom_fpm", _d)]


class OpoParams(ctypes.Structure):
    _fields_ = [("nx", _i), ("ny", _i), ("nt", _i), ("n_steps", _i), ("flags", _u),
                ("precision", _i), ("dz", _d), ("Lcr", _d), ("dx", _d), ("dy", _d),
                ("kappa", _d * 3), ("kdiff", _d * 3), ("vinv", _d * 3), ("beta2", _d * 3),
                ("alpha", _d * 3), ("dk", _d), ("Rs", _d), ("Ri", _d), ("detuning", _d),
                ("gdd", _d), ("free_len", _d), ("resonant", _u), ("total_rt", _i),
                ("t_window", _d), ("beta3", _d * 3), ("eom_beta", _d), ("eom_fpm", _d)]


class OpoError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"cuopo3d error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    """Load libcuopo3d.so (built in-tree by cuopo3d_b200.build); raises if absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: build it with `python -m cuopo3d_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        dp = ctypes.POINTER(ctypes.c_double)
        L.opo_params_from_config.argtypes = [ctypes.POINTER(OpoConfig), ctypes.POINTER(OpoParams), dp]
        L.opo_crystal_dispersion.argtypes = [_i, _d, _d, dp]
        L.opo_crystal_dispersion_pol.argtypes = [_i, _d, _i, _d, dp]
        L.opo_fp64_peak.argtypes = [dp]
        L.opo_time_freq.argtypes = [_i, _d, dp, dp]
        L.opo_pump_field.argtypes = [ctypes.POINTER(OpoConfig), dp]
        L.opo_noise.argtypes = [ctypes.c_uint64, _d, ctypes.c_size_t, dp]
        L.opo_create.argtypes = [ctypes.POINTER(OpoParams), dp, ctypes.POINTER(vp)]
        L.opo_destroy.argtypes = [vp]
        L.opo_destroy.restype = None
        L.opo_set_field.argtypes = [vp, _i, vp, _i, _i]
        L.opo_get_field.argtypes = [vp, _i, vp, _i, _i]
        L.opo_run_single_pass.argtypes = [vp]
        L.opo_run_round_trips.argtypes = [vp, _i]
        L.opo_stream_put.argtypes = [vp, _i, vp, _i]
        L.opo_stream_run.argtypes = [vp, _i]
        L.opo_stream_get.argtypes = [vp, _i, vp, _i]
        L.opo_stream_wait.argtypes = [vp]
        L.opo_field_sums.argtypes = [vp, dp]
        L.opo_synchronize.argtypes = [vp]
        L.opo_get_stream.argtypes = [vp, ctypes.POINTER(vp)]
        L.opo_init_fields.argtypes = [vp, ctypes.POINTER(OpoConfig), ctypes.c_uint64, _d, _i]
        L.opo_batch_create.argtypes = [_i, _i, ctypes.c_size_t, ctypes.POINTER(_i), ctypes.POINTER(vp)]
        L.opo_batch_destroy.argtypes = [vp]
        L.opo_batch_destroy.restype = None
        L.opo_batch_add.argtypes = [vp, ctypes.POINTER(OpoParams), dp, ctypes.POINTER(_i)]
        L.opo_batch_remove.argtypes = [vp, _i]
        L.opo_batch_set_field.argtypes = [vp, _i, _i, vp, _i, _i]
        L.opo_batch_get_field.argtypes = [vp, _i, _i, vp, _i, _i]
        L.opo_batch_init_fields.argtypes = [vp, _i, ctypes.POINTER(OpoConfig), ctypes.c_uint64, _d, _i]
        L.opo_batch_run_round_trips.argtypes = [vp, _i]
        L.opo_batch_sums.argtypes = [vp, dp]
        L.opo_batch_info.argtypes = [vp, _i, ctypes.POINTER(ctypes.c_longlong)]
        L.opo_batch_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
        L.opo_batch_get_stream.argtypes = [vp, ctypes.POINTER(vp)]
        L.opo_batch_synchronize.argtypes = [vp]
        L.opo_batch_last_error.argtypes = [vp]
        L.opo_batch_last_error.restype = ctypes.c_char_p
        L.opo_serve.argtypes = [vp, _i, vp, vp, dp]
        L.opo_autotune.argtypes = [vp]
        L.opo_get_tuning.argtypes = [vp, ctypes.POINTER(_i)]
        L.opo_set_tuning.argtypes = [vp, ctypes.POINTER(_i)]
        L.opo_field_sums_noalloc.argtypes = [vp, vp, vp, ctypes.c_size_t, _i, vp, dp]
        L.opo_noalloc_last_error.argtypes = []
        L.opo_noalloc_last_error.restype = ctypes.c_char_p
        L.opo_run_round_trips_tallied.argtypes = [vp, _i, dp, ctypes.POINTER(_i)]
        L.opo_power_cut_xy.argtypes = [ctypes.POINTER(OpoConfig), dp, dp]
        L.opo_sweep.argtypes = [ctypes.POINTER(OpoConfig), vp, _i, vp, dp]
        L.opo_sweep_threshold.argtypes = [vp, _i, dp, dp, dp]
        L.opo_sweep_write.argtypes = [ctypes.c_char_p, vp, _i, _i]
        L.opo_save_fields.argtypes = [vp, _i, ctypes.c_char_p, ctypes.c_char_p, _i]
        L.opo_set_wait_limit.argtypes = [vp, ctypes.c_longlong]
        L.opo_set_pass_timing.argtypes = [vp, _i]
        L.opo_pass_times.argtypes = [vp, dp, ctypes.POINTER(ctypes.c_longlong)]
        L.opo_round_trip_index.argtypes = [vp]
        L.opo_kernel_launches.argtypes = [vp]
        L.opo_kernel_launches.restype = ctypes.c_longlong
        L.opo_last_error.argtypes = [vp]
        L.opo_last_error.restype = ctypes.c_char_p
        L.opo_version.restype = ctypes.c_char_p
        _lib = L
    return _lib


def _dptr(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def make_config(**kw):
    """OpoConfig with the reference main()'s defaults (cuOPO3D.cu:15-46) overridden by kw."""
    d = dict(crystal=PPLN_ID, LX=400.0, LY=400.0, Lcr=5000.0, T=27.0, Lambda=6.97, lp=0.532,
             ls=1.064, nx=16, ny=16, nt=32, nz=10, dQ=-1.0, alpha=(-1.0, -1.0, -1.0), Lcav=-1.0,
             Rs=0.98, Ri=None, gdd_gamma=0.0, detuning=0.0, P=1.0, FWHM=2.0, w0=50.0, focal=None,
             pump_mode="focused-pulsed", t_window=0.0, flags=DISPERSION | DIFFRACTION,
             zloop_f32=0, n_steps=0, total_rt=1, precision=FP64, resonant=6, pol="eeo", eom_beta=0.0,
             eom_fpm=0.0)
    d.update(kw)
    if d["Ri"] is None:
        d["Ri"] = d["Rs"]
    if d["focal"] is None:
        d["focal"] = d["Lcr"] / 2
    if isinstance(d["pump_mode"], str):
        d["pump_mode"] = PUMP_MODES[d["pump_mode"]]
    if isinstance(d["crystal"], str):
        d["crystal"] = CRYSTALS[d["crystal"].lower()]
    if isinstance(d["pol"], str):
        # polarisation tuple of the reference (ZGP.cuh:24), e.g. "eeo": bit f = wave f is 'e'
        d["pol"] = sum(1 << f for f, ch in enumerate(d["pol"]) if ch == "e")
    c = OpoConfig()
    for k, v in d.items():
        if k == "alpha":
            c.alpha = (_d * 3)(*v)
        else:
            setattr(c, k, v)
    return c


def fp64_peak():
    """Measured FP64 FMA throughput of the current device (TFLOP/s)."""
    out = np.zeros(1)
    rc = lib().opo_fp64_peak(_dptr(out))
    if rc:
        raise OpoError(rc, "opo_fp64_peak")
    return float(out[0])


def derive(cfg):
    """(OpoParams, scalars dict) of a config (the reference constructors)."""
    p = OpoParams()
    sc = np.zeros(len(SCALAR_NAMES))
    rc = lib().opo_params_from_config(ctypes.byref(cfg), ctypes.byref(p), _dptr(sc))
    if rc:
        raise OpoError(rc, "opo_params_from_config rejected the configuration")
    return p, dict(zip(SCALAR_NAMES, sc))


def time_freq(nt, window):
    t, w = np.zeros(nt), np.zeros(nt)
    rc = lib().opo_time_freq(nt, window, _dptr(t), _dptr(w))
    if rc:
        raise OpoError(rc, "opo_time_freq")
    return t, w


def pump_field(cfg):
    a = np.zeros(2 * cfg.nx * cfg.ny * cfg.nt)
    rc = lib().opo_pump_field(ctypes.byref(cfg), _dptr(a))
    if rc:
        raise OpoError(rc, "opo_pump_field")
    return a.view(np.complex128).reshape(cfg.nt, cfg.ny, cfg.nx)


def noise(seed, sigma, n):
    a = np.zeros(2 * n)
    lib().opo_noise(seed, sigma, n, _dptr(a))
    return a.view(np.complex128)


class Simulation:
    """One resident solver (fields, tables, plans) on the current CUDA device."""

    def __init__(self, params, w):
        self.params = params
        self.shape = (params.nt, params.ny, params.nx)
        self._h = ctypes.c_void_p()
        w = np.ascontiguousarray(w, dtype=np.float64)
        rc = lib().opo_create(ctypes.byref(params), _dptr(w), ctypes.byref(self._h))
        if rc:
            raise OpoError(rc, "opo_create failed (no CUDA device, or unsupported grid)")

    def _check(self, rc):
        if rc:
            raise OpoError(rc, lib().opo_last_error(self._h).decode())

    @property
    def handle(self):
        return self._h

    def set_field(self, which, arr):
        a = np.ascontiguousarray(arr, dtype=np.complex128).reshape(-1)
        self._check(lib().opo_set_field(self._h, which, a.ctypes.data_as(ctypes.c_void_p), MEM_HOST, FP64))

    def set_field_device(self, which, ptr, precision):
        self._check(lib().opo_set_field(self._h, which, ctypes.c_void_p(ptr), MEM_DEVICE, precision))

    def get_field(self, which):
        a = np.zeros(int(np.prod(self.shape)), dtype=np.complex128)
        self._check(lib().opo_get_field(self._h, which, a.ctypes.data_as(ctypes.c_void_p), MEM_HOST, FP64))
        return a.reshape(self.shape)

    def get_field_device(self, which, ptr, precision):
        self._check(lib().opo_get_field(self._h, which, ctypes.c_void_p(ptr), MEM_DEVICE, precision))

    def run_single_pass(self):
        self._check(lib().opo_run_single_pass(self._h))

    def run_round_trips(self, n):
        self._check(lib().opo_run_round_trips(self._h, n))

    def field_sums(self):
        s = np.zeros(3)
        self._check(lib().opo_field_sums(self._h, _dptr(s)))
        return s

    def run_round_trips_tallied(self, n):
        """n round trips with the FP64 tallies (pump, signal, idler sums of |A|^2) after
        each; stops at the first non-finite round trip.  Returns (tallies [done, 3], rc):
        rc is OPO_OK or OPO_ERR_NONFINITE (other errors raise)."""
        t = np.zeros(3 * max(n, 1))
        done = _i(0)
        rc = lib().opo_run_round_trips_tallied(self._h, n, _dptr(t), ctypes.byref(done))
        if rc not in (OPO_OK, OPO_ERR_NONFINITE):
            self._check(rc)
        return t[:3 * done.value].reshape(done.value, 3), rc

    def save_fields(self, which, slice_prefix=None, trace_prefix=None, binary=False):
        """The reference's field dumps from one device-to-host copy (opo_save_fields):
        text slice / trace files, or one binary file '<slice_prefix>.bin'."""
        enc = lambda x: None if x is None else str(x).encode()
        self._check(lib().opo_save_fields(self._h, which, enc(slice_prefix), enc(trace_prefix),
                                          FILES_BINARY if binary else FILES_TEXT))

    def set_wait_limit(self, cycles):
        """Bound of the warp-specialised passes' pipeline waits (SM cycles; 0: ~2 s)."""
        self._check(lib().opo_set_wait_limit(self._h, int(cycles)))

    @property
    def stream(self):
        """The solver's cudaStream_t as an integer (e.g. for torch.cuda.ExternalStream)."""
        st = ctypes.c_void_p()
        self._check(lib().opo_get_stream(self._h, ctypes.byref(st)))
        return st.value or 0

    def autotune(self):
        """Pick the fastest kernel variant and tile per pass (timed on scratch fields; the
        solver's fields are left as they were)."""
        self._check(lib().opo_autotune(self._h))
        return self.tuning

    def set_tuning(self, tuning):
        flat = []
        for k in ("t", "x", "y"):
            flat += [tuning[k]["threads"], tuning[k]["tile"], tuning[k]["r1"]]
        self._check(lib().opo_set_tuning(self._h, (_i * 9)(*flat)))

    @property
    def tuning(self):
        out = (_i * 9)()
        self._check(lib().opo_get_tuning(self._h, out))
        return {k: dict(threads=out[3 * i], tile=out[3 * i + 1], r1=out[3 * i + 2])
                for i, k in enumerate(("t", "x", "y"))}

    def set_plane_pass(self, cluster, threads=256, r1=8):
        """Diffraction as one fused (x, y) plane pass on clusters of `cluster` CTAs (2, 4, 8),
        or as separate x and y passes (cluster=0)."""
        self._check(lib().opo_set_plane_pass(self._h, int(cluster), int(threads), int(r1)))

    @property
    def plane_pass(self):
        out = (_i * 3)()
        self._check(lib().opo_get_plane_pass(self._h, out))
        return dict(cluster=out[0], threads=out[1], r1=out[2])

    def init_fields(self, cfg, seed, sigma, idler_copy=False):
        """Api = Ap = pump, As = seeded noise, Ai = 0 (or As), computed on the device."""
        self._check(lib().opo_init_fields(self._h, ctypes.byref(cfg), seed, sigma, 1 if idler_copy else 0))

    def set_pass_timing(self, enable):
        self._check(lib().opo_set_pass_timing(self._h, 1 if enable else 0))

    def pass_times(self):
        """{kind: (total_ms, launches)} for t/x/y passes and other kernels since the last call."""
        ms = np.zeros(4)
        cnt = (ctypes.c_longlong * 4)()
        self._check(lib().opo_pass_times(self._h, _dptr(ms), cnt))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(("t", "x", "y", "other"))}

    def synchronize(self):
        self._check(lib().opo_synchronize(self._h))

    # Streamed round trips (opo_stream_*): `ptr` is the address of pinned host memory
    # holding (put) or receiving (get) one field in the solver's precision; the calls
    # return at once and the buffers stay in use until stream_wait().
    def stream_put(self, which, ptr):
        self._check(lib().opo_stream_put(self._h, which, ctypes.c_void_p(ptr), self.params.precision))

    def stream_run(self, n=1):
        self._check(lib().opo_stream_run(self._h, n))

    def stream_get(self, which, ptr):
        self._check(lib().opo_stream_get(self._h, which, ctypes.c_void_p(ptr), self.params.precision))

    def stream_wait(self):
        self._check(lib().opo_stream_wait(self._h))

    @property
    def round_trip_index(self):
        return lib().opo_round_trip_index(self._h)

    @property
    def kernel_launches(self):
        return lib().opo_kernel_launches(self._h)

    def close(self):
        if self._h:
            lib().opo_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class OpoServeRequest(ctypes.Structure):
    _fields_ = [("cfg", OpoConfig), ("arrival_s", _d), ("seed", ctypes.c_uint64), ("noise_sigma", _d),
                ("tol", _d), ("out_fields", ctypes.c_void_p * 3)]


class OpoServeOptions(ctypes.Structure):
    _fields_ = [("precision", _i), ("capacity", _i), ("hbm_budget", ctypes.c_size_t), ("realtime", _i),
                ("tuning_set", _i), ("tuning", _i * 9)]


class OpoServeResult(ctypes.Structure):
    _fields_ = [("status", _i), ("round_trips", _i), ("admit_s", _d), ("done_s", _d), ("latency_s", _d),
                ("power", _d * 3), ("voxel_steps", ctypes.c_longlong)]


SERVE_STATS = ("p50_latency_s", "p99_latency_s", "wall_s", "voxel_steps_per_s", "max_resident",
               "kernel_launches", "voxel_steps", "completed")


def serve(requests, precision, capacity, hbm_budget, realtime=True, tuning=None):
    """Run a request stream with continuous batching (opo_serve).  requests: list of
    dicts with cfg (OpoConfig), arrival_s, seed, noise_sigma, tol and, optionally,
    return_fields=True for the final (pump, signal, idler) of that request in its result
    ("fields").  Returns (results, stats)."""
    n = len(requests)
    reqs = (OpoServeRequest * max(n, 1))()
    bufs = {}
    for k, r in enumerate(requests):
        reqs[k].cfg = r["cfg"]
        reqs[k].arrival_s = r.get("arrival_s", 0.0)
        reqs[k].seed = r.get("seed", 1)
        reqs[k].noise_sigma = r.get("noise_sigma", 1e-6)
        reqs[k].tol = r.get("tol", 0.0)
        if r.get("return_fields"):
            c = r["cfg"]
            bufs[k] = [np.zeros((c.nt, c.ny, c.nx), np.complex128) for _ in range(3)]
            for f in range(3):
                reqs[k].out_fields[f] = bufs[k][f].ctypes.data
    opt = OpoServeOptions()
    opt.precision, opt.capacity, opt.hbm_budget, opt.realtime = precision, capacity, int(hbm_budget), int(realtime)
    if tuning is not None:
        opt.tuning_set = 1
        flat = []
        for k in ("t", "x", "y"):
            flat += [tuning[k]["threads"], tuning[k]["tile"], tuning[k]["r1"]]
        opt.tuning = (_i * 9)(*flat)
    out = (OpoServeResult * max(n, 1))()
    stats = np.zeros(8)
    rc = lib().opo_serve(reqs, n, ctypes.byref(opt), out, _dptr(stats))
    if rc:
        raise OpoError(rc, lib().opo_batch_last_error(None).decode())
    res = [dict(status=o.status, round_trips=o.round_trips, admit_s=o.admit_s, done_s=o.done_s,
                latency_s=o.latency_s, power=np.array(o.power[:]), voxel_steps=o.voxel_steps)
           for o in out[:n]]
    for k, b in bufs.items():
        res[k]["fields"] = tuple(b)
    return res, dict(zip(SERVE_STATS, stats))


class OpoSweepOptions(ctypes.Structure):
    _fields_ = [("precision", _i), ("round_trips", _i), ("window", _i), ("seed", ctypes.c_uint64),
                ("noise_sigma", _d), ("hbm_budget", ctypes.c_size_t), ("capacity", _i), ("tuning_set", _i),
                ("tuning", _i * 9)]


class OpoSweepPoint(ctypes.Structure):
    _fields_ = [("P", _d), ("w0", _d), ("status", _i), ("round_trips", _i), ("sums", _d * 3),
                ("power_xy", _d * 3), ("output_power", _d), ("gain", _d), ("above", _i)]


def _point_dict(p):
    return dict(P=p.P, w0=p.w0, status=p.status, round_trips=p.round_trips, sums=np.array(p.sums[:]),
                power_xy=np.array(p.power_xy[:]), output_power=p.output_power, gain=p.gain, above=bool(p.above))


def _points(points):
    arr = (OpoSweepPoint * max(len(points), 1))()
    for k, q in enumerate(points):
        for name, _ in OpoSweepPoint._fields_:
            v = q[name]
            if name in ("sums", "power_xy"):
                getattr(arr[k], name)[:] = list(v)
            else:
                setattr(arr[k], name, int(v) if name in ("status", "round_trips", "above") else float(v))
    return arr


def power_cut_xy(cfg, sums):
    """The reference's averagePowerCutXY of each field from FP64 tallies (opo_power_cut_xy)."""
    s = np.ascontiguousarray(sums, dtype=np.float64)
    out = np.zeros(3)
    rc = lib().opo_power_cut_xy(ctypes.byref(cfg), _dptr(s), _dptr(out))
    if rc:
        raise OpoError(rc, "opo_power_cut_xy")
    return out


def sweep(base_cfg, powers, waists, round_trips, window=3, seed=1, noise_sigma=1e-3, hbm_budget=8 << 30,
          capacity=0, tuning=None):
    """Threshold sweep (opo_sweep): one OPO per (P, w0) point of base_cfg, each run for
    round_trips with FP64 tallies after every round trip.  Returns (points, tallies) with
    tallies[k, r] = the sums after round trip r + 1 of point k."""
    n = len(powers)
    assert len(waists) == n
    pts = (OpoSweepPoint * max(n, 1))()
    for k in range(n):
        pts[k].P, pts[k].w0 = float(powers[k]), float(waists[k])
    opt = OpoSweepOptions()
    opt.precision, opt.round_trips, opt.window, opt.seed = base_cfg.precision, round_trips, window, seed
    opt.noise_sigma, opt.hbm_budget, opt.capacity = noise_sigma, int(hbm_budget), capacity
    if tuning is not None:
        opt.tuning_set = 1
        flat = []
        for k in ("t", "x", "y"):
            flat += [tuning[k]["threads"], tuning[k]["tile"], tuning[k]["r1"]]
        opt.tuning = (_i * 9)(*flat)
    tallies = np.zeros(max(n, 1) * round_trips * 3)
    rc = lib().opo_sweep(ctypes.byref(base_cfg), pts, n, ctypes.byref(opt), _dptr(tallies))
    if rc:
        raise OpoError(rc, "opo_sweep")
    return [_point_dict(pts[k]) for k in range(n)], tallies[:n * round_trips * 3].reshape(n, round_trips, 3)


def sweep_threshold(points):
    """(P below, P above, estimate) of the threshold among sweep points of one waist, or None."""
    arr = _points(points)
    lo, hi, est = _d(), _d(), _d()
    rc = lib().opo_sweep_threshold(arr, len(points), ctypes.byref(lo), ctypes.byref(hi), ctypes.byref(est))
    return None if rc else (lo.value, hi.value, est.value)


def sweep_write(path, points, append=True):
    """The reference's saveAppendedValues2Columns format: 'P <tab> output power' per line."""
    rc = lib().opo_sweep_write(str(path).encode(), _points(points), len(points), 1 if append else 0)
    if rc:
        raise OpoError(rc, f"opo_sweep_write({path})")


class Batch:
    """Many instances advanced together by one persistent launch per pass
    (opo_batch_* of the C-ABI).  Instances are admitted into slots while they fit the
    HBM budget; all take the same number of z-steps."""

    def __init__(self, precision, capacity, hbm_budget, tuning=None):
        self._h = ctypes.c_void_p()
        self.capacity = capacity
        self.precision = precision
        t = None
        if tuning is not None:
            flat = []
            for k in ("t", "x", "y"):
                flat += [tuning[k]["threads"], tuning[k]["tile"], tuning[k]["r1"]]
            t = (_i * 9)(*flat)
        rc = lib().opo_batch_create(precision, capacity, int(hbm_budget), t, ctypes.byref(self._h))
        if rc:
            raise OpoError(rc, lib().opo_batch_last_error(None).decode())
        self.shapes = {}

    def _check(self, rc):
        if rc:
            raise OpoError(rc, lib().opo_batch_last_error(self._h).decode())

    def add(self, cfg):
        """Admit the instance of config `cfg`; returns its slot (OpoError code 6 if full)."""
        params, _ = derive(cfg)
        _, w = time_freq(cfg.nt, params.t_window)
        slot = ctypes.c_int(-1)
        self._check(lib().opo_batch_add(self._h, ctypes.byref(params), _dptr(np.ascontiguousarray(w)),
                                        ctypes.byref(slot)))
        self.shapes[slot.value] = (cfg.nt, cfg.ny, cfg.nx)
        return slot.value

    def remove(self, slot):
        self._check(lib().opo_batch_remove(self._h, slot))
        self.shapes.pop(slot, None)

    def init_fields(self, slot, cfg, seed, sigma, idler_copy=False):
        self._check(lib().opo_batch_init_fields(self._h, slot, ctypes.byref(cfg), seed, sigma,
                                                1 if idler_copy else 0))

    def set_field(self, slot, which, arr):
        a = np.ascontiguousarray(arr, dtype=np.complex128).reshape(-1)
        self._check(lib().opo_batch_set_field(self._h, slot, which, a.ctypes.data_as(ctypes.c_void_p),
                                              MEM_HOST, FP64))

    def get_field(self, slot, which):
        shape = self.shapes[slot]
        a = np.zeros(int(np.prod(shape)), dtype=np.complex128)
        self._check(lib().opo_batch_get_field(self._h, slot, which, a.ctypes.data_as(ctypes.c_void_p),
                                              MEM_HOST, FP64))
        return a.reshape(shape)

    def run_round_trips(self, n):
        self._check(lib().opo_batch_run_round_trips(self._h, n))

    def sums(self):
        s = np.zeros(3 * self.capacity)
        self._check(lib().opo_batch_sums(self._h, _dptr(s)))
        return s.reshape(self.capacity, 3)

    def info(self, slot):
        out = (ctypes.c_longlong * 4)()
        self._check(lib().opo_batch_info(self._h, slot, out))
        return dict(round_trips=out[0], total_rt=out[1], voxels=out[2], bytes=out[3])

    def stats(self):
        out = (ctypes.c_longlong * 4)()
        self._check(lib().opo_batch_stats(self._h, out))
        return dict(instances=out[0], used=out[1], budget=out[2], launches=out[3])

    @property
    def stream(self):
        st = ctypes.c_void_p()
        self._check(lib().opo_batch_get_stream(self._h, ctypes.byref(st)))
        return st.value or 0

    def synchronize(self):
        self._check(lib().opo_batch_synchronize(self._h))

    def close(self):
        if self._h:
            lib().opo_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


from .reference_api import Cavity, EFields, MgOsPPLT, PPLN, Solver  # noqa: E402,F401


def read_field_file(path):
    """A field written by opo_save_fields in binary form: (header dict, array [t][y][x])."""
    with open(path, "rb") as f:
        raw = f.read()
    if raw[:8] != b"OPO3DFLD":
        raise ValueError(f"{path}: not a field file")
    version, nx, ny, nt, esz, which = np.frombuffer(raw[8:32], dtype=np.int32)
    dt = np.complex128 if esz == 16 else np.complex64
    a = np.frombuffer(raw[32:], dtype=dt).reshape(nt, ny, nx)
    return dict(version=int(version), nx=int(nx), ny=int(ny), nt=int(nt), bytes=int(esz), which=int(which)), a
