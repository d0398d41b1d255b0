"""Python mirror of the reference's classes (alfredos84/cuOPO3D src/headers): crystals
(CrystalsBase/PPLN.cuh, MgOsPPLT.cuh, MgOPPLN.cuh, ZGP.cuh), Cavity (Cavity3D.cuh), EFields (EFields3D.cuh)
and Solver (Solver3D.cuh), with the same names, arguments and members, driving the
CUDA library through the C-ABI.

The reference fixes the grid at compile time (DtypesConsts.cuh:30-54: NX, NY, NT, NZ,
NRT); here the crystal takes them as keyword arguments and the other objects read
them from it.  Field members (Api, Ap, As, Ai) are host numpy arrays [t][y][x]; the
solver uploads them, runs on the GPU and downloads the results.
"""
import ctypes

import numpy as np

from . import (DIFFRACTION, DISPERSION, FIELD_AI, FIELD_AP, FIELD_API, FIELD_AS, FP64,
               MGOPPLN_ID, MGOSPPLT_ID, PPLN_ID, PUMP_MODES, ZGP_ID, OpoError, Simulation, _dptr, derive,
               lib, make_config, noise, time_freq)

PI = 3.14159265358979323846
C = 299792458 * 1E6 / 1E12          # um/ps, DtypesConsts.cuh:56
EPS0 = 8.8541878128E-12 * 1E12 / 1E6  # DtypesConsts.cuh:57


class _Crystal:
    kind = None
    name = None
    d33 = None
    alphas = None
    QPM = True
    pol_bits = 0

    def __init__(self, LX, LY, Lcr, T, Lambda, lp, ls, li, NX=128, NY=128, NT=256, NZ=100):
        self.LX, self.LY, self.Lcr, self.T, self.Lambda = LX, LY, Lcr, T, Lambda
        self.lp, self.ls, self.li = lp, ls, li
        self.NX, self.NY, self.NT, self.NZ = NX, NY, NT, NZ
        self.dQ = 2.0 * self.d33 / PI
        self.alpha_crp, self.alpha_crs, self.alpha_cri = self.alphas
        self.dx = LX / (NX - 1.0)
        self.dy = LY / (NY - 1.0)
        self.dz = Lcr / (NZ - 1.0)
        out = np.zeros(4)
        vals = []
        for f, lam in enumerate((lp, ls, li)):
            rc = lib().opo_crystal_dispersion_pol(self.kind, T, (self.pol_bits >> f) & 1, lam, _dptr(out))
            if rc:
                raise OpoError(rc, "opo_crystal_dispersion_pol")
            vals.append(out.copy())
        (self.np, self.vp, self.b2p, self.b3p), (self.ns, self.vs, self.b2s, self.b3s), \
            (self.ni, self.vi, self.b2i, self.b3i) = vals
        # PPLN.cuh:74-77: kp and ki use the signal index and ls as shipped
        self.kp = 2.0 * PI * self.ns / lp
        self.ks = 2.0 * PI * self.ns / ls
        self.ki = 2.0 * PI * self.ni / ls
        self.dk = self.kp - self.ks - self.ki - (2.0 * PI / Lambda if self.QPM else 0.0)

    def getCrystalProp(self):
        print(f"Crystal name = {self.name}\n        ---> Temp = {self.T} C\n"
              f"        ---> np, ns, ni = {self.np}, {self.ns}, {self.ni}\n"
              f"        ---> dz = {self.dz} um, dx = {self.dx} um")


class PPLN(_Crystal):
    kind, name, d33 = PPLN_ID, "PPLN", 25.20e-6
    alphas = (0.025e-4, 0.002e-4, 0.002e-4)


class MgOsPPLT(_Crystal):
    kind, name, d33 = MGOSPPLT_ID, "MgOsPPLT", 11.0e-6
    alphas = (1.57e-4, 0.17e-6, 0.17e-6)


class MgOPPLN(_Crystal):
    """MgO:PPLN (Gayer), CrystalsBase/MgOPPLN.cuh:20-78."""
    kind, name, d33 = MGOPPLN_ID, "MgO:PPLN", 25.20e-6
    alphas = (0.025e-4, 0.002e-4, 0.002e-4)


class ZGP(_Crystal):
    """ZnGeP2 (Zelmon), CrystalsBase/ZGP.cuh:17-80: birefringent phase matching with a
    polarisation tuple such as ('e', 'e', 'o'); no temperature or grating period."""
    kind, name, d33 = ZGP_ID, "ZPG", 75.0e-6
    alphas = (1.57e-4, 0.17e-6, 0.17e-6)
    QPM = False

    def __init__(self, LX, LY, Lcr, pol, lp, ls, li, **grid):
        self.pol = tuple(pol)
        self.pol_bits = sum(1 << f for f, ch in enumerate(self.pol) if ch == "e")
        super().__init__(LX, LY, Lcr, 0.0, 1.0, lp, ls, li, **grid)

    def setPolarizations(self, p, s, i):
        """ZGP.cuh:98-102: stores the tuple only; the indices keep their constructed values."""
        self.pol = (p, s, i)


class Cavity:
    """Ring cavity, Cavity3D.cuh:31-62."""

    def __init__(self, Cr, Lcav, Rs, Ri):
        self.Cr, self.Lcav, self.Rs, self.Ri = Cr, Lcav, Rs, Ri
        self.trt = (Lcav + Cr.Lcr * (Cr.ns - 1)) / C
        self.dt = self.trt / (Cr.NT - 1)
        self.fsr = 1.0 / self.trt
        self.Lfs = Lcav - Cr.Lcr
        self.gdd, self.gamma = False, 0.0
        self.detuning = 0.0
        self.eom, self.beta, self.fpm = False, 0.0, 0.0

    def setGDDCompensation(self, gamma):
        self.gdd, self.gamma = True, gamma

    def setEOM(self, beta, fpm):
        """Intracavity electro-optic modulator, Cavity1D.cuh:75-84: after each pass,
        signal and idler x exp(i beta sin(2 pi fpm t)) (Solver1D.cuh:63-72, 467)."""
        self.eom, self.beta, self.fpm = True, beta, fpm

    def getCavityProp(self):
        print(f"Set OPO cavity:\n        ---> Round trip time = {self.trt} ps\n"
              f"        ---> Signal reflectivity = {self.Rs * 100} %")


class EFields:
    """Field state, EFields3D.cuh:174-239."""

    def __init__(self, lp, ls, li, Power, waist, Cr):
        self.lp, self.ls, self.li, self.Power, self.waist, self.Cr = lp, ls, li, Power, waist, Cr
        shape = (Cr.NT, Cr.NY, Cr.NX)
        self.Api = np.zeros(shape, np.complex128)
        self.Ap = np.zeros(shape, np.complex128)
        self.As = np.zeros(shape, np.complex128)
        self.Ai = np.zeros(shape, np.complex128)
        self.resFields = (False, True, True)
        self.window = None
        self.pump = None
        self.t = self.w = None

    def setTimeFreqVectors(self, trt):
        self.window = trt
        self.t, self.w = time_freq(self.Cr.NT, trt)

    def setPumpField(self, Power, FWHM, waist, focalpoint, mode):
        if mode not in PUMP_MODES:
            raise ValueError(f"Invalid option for pump electric field: {mode}")
        self.pump = dict(P=Power, FWHM=FWHM, w0=waist, focal=focalpoint, pump_mode=mode)
        cfg = _config(self.Cr, None, self)
        a = np.zeros(2 * self.Api.size)
        rc = lib().opo_pump_field(ctypes.byref(cfg), _dptr(a))
        if rc:
            raise OpoError(rc, "opo_pump_field")
        self.Api = a.view(np.complex128).reshape(self.Api.shape)

    def noiseGenerator(self, Vec, seed=1, sigma=1.0e-15):
        """Seeded replacement of EFields3D.cuh:300-315 (fills Vec in place)."""
        Vec[...] = noise(seed, sigma, Vec.size).reshape(Vec.shape)


def _config(Cr, Cav, A, flags=DISPERSION | DIFFRACTION, precision=FP64, total_rt=1, **kw):
    pump = A.pump or dict(P=A.Power, FWHM=1.0, w0=A.waist, focal=Cr.Lcr / 2,
                          pump_mode="focused-cw")
    res = (2 if A.resFields[1] else 0) | (4 if A.resFields[2] else 0)
    d = dict(crystal=Cr.kind, pol=Cr.pol_bits, LX=Cr.LX, LY=Cr.LY, Lcr=Cr.Lcr, T=Cr.T, Lambda=Cr.Lambda,
             lp=Cr.lp, ls=Cr.ls, nx=Cr.NX, ny=Cr.NY, nt=Cr.NT, nz=Cr.NZ, dQ=Cr.dQ,
             alpha=(Cr.alpha_crp, Cr.alpha_crs, Cr.alpha_cri),
             t_window=A.window or 0.0, flags=flags, precision=precision,
             total_rt=total_rt, resonant=res, **pump)
    if Cav is not None:
        d.update(Lcav=Cav.Lcav, Rs=Cav.Rs, Ri=Cav.Ri, gdd_gamma=Cav.gamma if Cav.gdd else 0.0,
                 detuning=Cav.detuning, eom_beta=Cav.beta if Cav.eom else 0.0, eom_fpm=Cav.fpm if Cav.eom else 0.0)
    d.update(kw)
    return make_config(**d)


class Solver:
    """Split-step solver, Solver3D.cuh:429-491, running on the GPU."""

    def __init__(self, Cr, Cav, A=None, precision=FP64, flags=DISPERSION | DIFFRACTION):
        if A is None:  # Solver(Cr, A) form, Solver3D.cuh:442
            Cav, A = None, Cav
        self.Cr, self.Cav, self.A = Cr, Cav, A
        self.precision, self.flags = precision, flags
        self.sim = None

    def _start(self, total_rt):
        cfg = _config(self.Cr, self.Cav, self.A, flags=self.flags, precision=self.precision,
                      total_rt=total_rt)
        params, self.scalars = derive(cfg)
        w = self.A.w if self.A.w is not None else time_freq(cfg.nt, params.t_window)[1]
        self.sim = Simulation(params, w)
        for which, arr in ((FIELD_API, self.A.Api), (FIELD_AP, self.A.Ap), (FIELD_AS, self.A.As),
                           (FIELD_AI, self.A.Ai)):
            self.sim.set_field(which, arr)

    def _finish(self):
        self.A.Ap = self.sim.get_field(FIELD_AP)
        self.A.As = self.sim.get_field(FIELD_AS)
        self.A.Ai = self.sim.get_field(FIELD_AI)

    def checkCourantStability(self, dz, kpdxdy):
        return dz < kpdxdy

    def runOPO(self, save_roundtrips=None, NRT=10000):
        """NRT round trips (Solver3D.cuh:964-1023), after the reference's step-size gate."""
        if not self.checkCourantStability(self.Cr.dz, 0.2 * self.Cr.kp * self.Cr.dx * self.Cr.dy):
            raise OpoError(5, "Courant convergence criteria: failed")
        self._start(NRT)
        self.sim.run_round_trips(NRT)
        self._finish()

    def runSinglePass(self):
        self._start(1)
        self.sim.run_single_pass()
        self._finish()

    def averagePowerCutXY(self, field):
        """0.5 eps0 c ns dx dy / (LX LY) sum |A|^2, Solver3D.cuh:529-545 (FP64 sum)."""
        s = float(np.sum(np.abs(field) ** 2))
        return 0.5 * EPS0 * C * self.Cr.ns * self.Cr.dx * self.Cr.dy / (self.Cr.LX * self.Cr.LY) * s
