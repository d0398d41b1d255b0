"""Test infrastructure, NOT product code: ctypes binding of the FP64 CPU oracle
(oracle/libopo_oracle.so, built from opo_oracle.cpp by oracle/Makefile).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import this
module, as the checker.  Parity status: pinned by the fixtures in tests/golden,
which hold outputs of the reference itself (its own headers compiled by
oracle/refharness and run on a B200).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libopo_oracle.so")

OR_DISPERSION = 1 << 0
OR_DIFFRACTION = 1 << 1
OR_PHYSICS = 1 << 2
OR_ASIS_Q1 = 1 << 3
OR_ASIS_Q2 = 1 << 4
OR_TOD = 1 << 5

OR_PPLN, OR_MGOSPPLT, OR_MGOPPLN, OR_ZGP = 0, 1, 2, 3
PUMP_MODES = {
    "waveplane-cw": 0,
    "waveplane-pulsed": 1,
    "focused-cw": 2,
    "focused-pulsed": 3,
    "focused-sech2": 4,
    "waveplane-sech2": 5,
}
SCALAR_NAMES = ("np ns ni vp vs vi b2p b2s b2i b3p b3s b3i dQ dk dx dy dz kp ks ki "
                "kappa_p kappa_s kappa_i trt dt nsteps").split()


class OrPhys(ctypes.Structure):
    _fields_ = [
        ("crystal", ctypes.c_int),
        ("LX", ctypes.c_double), ("LY", ctypes.c_double), ("Lcr", ctypes.c_double),
        ("T", ctypes.c_double), ("Lambda", ctypes.c_double), ("lp", ctypes.c_double),
        ("ls", ctypes.c_double),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nt", ctypes.c_int), ("nz", ctypes.c_int),
        ("dQ", ctypes.c_double),
        ("alpha", ctypes.c_double * 3),
        ("Lcav", ctypes.c_double), ("Rs", ctypes.c_double), ("Ri", ctypes.c_double),
        ("gdd_gamma", ctypes.c_double), ("detuning", ctypes.c_double),
        ("P", ctypes.c_double), ("FWHM", ctypes.c_double), ("w0", ctypes.c_double),
        ("focal", ctypes.c_double),
        ("pump_mode", ctypes.c_int),
        ("t_window", ctypes.c_double),
        ("flags", ctypes.c_uint),
        ("zloop_f32", ctypes.c_int),
        ("n_steps", ctypes.c_int),
        ("total_rt", ctypes.c_int),
        ("pol", ctypes.c_uint),
        ("eom_beta", ctypes.c_double), ("eom_fpm", ctypes.c_double),
        ("resonant", ctypes.c_uint),
    ]


class OrParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nt", ctypes.c_int),
        ("n_steps", ctypes.c_int),
        ("flags", ctypes.c_uint),
        ("dz", ctypes.c_double), ("Lcr", ctypes.c_double), ("dx", ctypes.c_double),
        ("dy", ctypes.c_double),
        ("kappa", ctypes.c_double * 3), ("kdiff", ctypes.c_double * 3),
        ("vinv", ctypes.c_double * 3), ("beta2", ctypes.c_double * 3),
        ("alpha", ctypes.c_double * 3),
        ("dk", ctypes.c_double),
        ("Rs", ctypes.c_double), ("Ri", ctypes.c_double), ("detuning", ctypes.c_double),
        ("gdd", ctypes.c_double), ("free_len", ctypes.c_double),
        ("total_rt", ctypes.c_int), ("rt_index", ctypes.c_int),
        ("beta3", ctypes.c_double * 3),
        ("eom_beta", ctypes.c_double), ("eom_fpm", ctypes.c_double), ("t_window", ctypes.c_double),
        ("resonant", ctypes.c_uint),
    ]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        L.or_setup.argtypes = [ctypes.POINTER(OrPhys), ctypes.POINTER(OrParams), dp, dp, dp, dp]
        L.or_setup.restype = ctypes.c_int
        L.or_zloop_steps.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int]
        L.or_zloop_steps.restype = ctypes.c_int
        L.or_fft.argtypes = [ctypes.c_int, ctypes.c_int, dp]
        L.or_noise.argtypes = [ctypes.c_uint64, ctypes.c_double, ctypes.c_size_t, dp]
        L.or_single_pass.argtypes = [ctypes.POINTER(OrParams), dp, dp, dp, dp]
        L.or_round_trips.argtypes = [ctypes.POINTER(OrParams), dp, dp, dp, dp, dp, ctypes.c_int]
        L.or_set_threads.argtypes = [ctypes.c_int]
        L.or_crystal_dispersion.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double, dp]
        _lib = L
    return _lib


def _ptr(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def make_phys(**kw):
    """OrPhys with the reference main()'s defaults (cuOPO3D.cu:15-46) overridden by kw."""
    d = dict(crystal=OR_PPLN, LX=400.0, LY=400.0, Lcr=5000.0, T=27.0, Lambda=6.97,
             lp=0.532, ls=1.064, nx=16, ny=16, nt=32, nz=10, dQ=-1.0,
             alpha=(-1.0, -1.0, -1.0), Lcav=-1.0, Rs=0.98, Ri=None, gdd_gamma=0.0,
             detuning=0.0, P=1.0, FWHM=2.0, w0=50.0, focal=None, pump_mode="focused-pulsed",
             t_window=0.0, flags=OR_DISPERSION | OR_DIFFRACTION, zloop_f32=0, n_steps=0,
             total_rt=1, pol="eeo", eom_beta=0.0, eom_fpm=0.0, resonant=6)
    d.update(kw)
    if isinstance(d["pol"], str):
        d["pol"] = sum(1 << f for f, ch in enumerate(d["pol"]) if ch == "e")
    if d["Ri"] is None:
        d["Ri"] = d["Rs"]
    if d["focal"] is None:
        d["focal"] = d["Lcr"] / 2
    if d["Lcav"] is None or d["Lcav"] < 0:
        d["Lcav"] = 4 * d["Lcr"]
    if isinstance(d["pump_mode"], str):
        d["pump_mode"] = PUMP_MODES[d["pump_mode"]]
    ph = OrPhys()
    for k, v in d.items():
        if k == "alpha":
            ph.alpha = (ctypes.c_double * 3)(*v)
        else:
            setattr(ph, k, v)
    return ph


def crystal_dispersion(crystal, T, L, extraordinary=True):
    """(n, vg, b2, b3 as the reference prints it, exact b3) of one crystal index."""
    out = np.zeros(5)
    rc = lib().or_crystal_dispersion(crystal, T, 1 if extraordinary else 0, L, _ptr(out))
    if rc:
        raise ValueError(f"or_crystal_dispersion: {rc}")
    return out


class Setup:
    """Derived parameters, scalars, grids and pump of one run (oracle's own)."""

    def __init__(self, phys):
        L = lib()
        self.phys = phys
        self.params = OrParams()
        self.scalars_arr = np.zeros(len(SCALAR_NAMES))
        nt, V = phys.nt, phys.nx * phys.ny * phys.nt
        self.t = np.zeros(nt)
        self.w = np.zeros(nt)
        self.Api = np.zeros(2 * V)
        rc = L.or_setup(ctypes.byref(phys), ctypes.byref(self.params), _ptr(self.scalars_arr),
                        _ptr(self.t), _ptr(self.w), _ptr(self.Api))
        if rc != 0:
            raise ValueError(f"or_setup failed: {rc}")
        self.scalars = dict(zip(SCALAR_NAMES, self.scalars_arr))

    @property
    def shape(self):
        return (self.phys.nt, self.phys.ny, self.phys.nx)

    def api_complex(self):
        return self.Api.view(np.complex128).reshape(self.shape)


def noise(seed, sigma, n):
    out = np.zeros(2 * n)
    lib().or_noise(seed, sigma, n, _ptr(out))
    return out.view(np.complex128)


def fft(x, sign):
    a = np.ascontiguousarray(np.asarray(x, dtype=np.complex128)).copy()
    buf = a.view(np.float64)
    lib().or_fft(len(a), sign, _ptr(buf))
    return a


def _f(a):
    return np.ascontiguousarray(a, dtype=np.complex128).reshape(-1).view(np.float64).copy()


def single_pass(setup, Ap, As, Ai):
    """Run the crystal once; returns new (Ap, As, Ai) complex arrays [t][y][x]."""
    p, s, i = _f(Ap), _f(As), _f(Ai)
    lib().or_single_pass(ctypes.byref(setup.params), _ptr(setup.w), _ptr(p), _ptr(s), _ptr(i))
    sh = setup.shape
    return (p.view(np.complex128).reshape(sh), s.view(np.complex128).reshape(sh),
            i.view(np.complex128).reshape(sh))


def round_trips(setup, Api, Ap, As, Ai, n_rt):
    """Run n_rt cavity round trips; setup.params.rt_index advances."""
    a0 = _f(Api)
    p, s, i = _f(Ap), _f(As), _f(Ai)
    lib().or_round_trips(ctypes.byref(setup.params), _ptr(setup.w), _ptr(a0), _ptr(p), _ptr(s),
                         _ptr(i), n_rt)
    sh = setup.shape
    return (p.view(np.complex128).reshape(sh), s.view(np.complex128).reshape(sh),
            i.view(np.complex128).reshape(sh))


def set_threads(n):
    lib().or_set_threads(n)
