"""Helpers to replay the golden fixtures (outputs of the reference cuOPO3D built by
oracle/refharness and run on a B200) through the oracle or the CUDA library."""
import glob
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MAX_ORACLE_VOXEL_STEPS = 2e8


def fixture_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


class Golden:
    def __init__(self, name):
        z = np.load(os.path.join(GOLDEN, name + ".npz"))
        self.name = name
        self.meta = json.loads(str(z["meta"]))
        self.args = self.meta["args"]
        self.scalars = dict(zip([str(s) for s in z["scalar_names"]], z["scalar_values"]))
        self.t, self.w, self.tidx = z["t"], z["w"], z["tidx"]
        self.Api, self.Ap, self.As, self.Ai = z["Api"], z["Ap"], z["As"], z["Ai"]
        self.norms = z["norms"]
        # energy of every t-slice of Ap, As, Ai (newer fixtures), else None
        self.tprof = z["tprof"] if "tprof" in z.files else None
        nx, ny, nt = self.meta["shape"]
        self.nx, self.ny, self.nt = nx, ny, nt
        self.fp64 = bool(self.scalars["fp64"])
        self.asis = not bool(self.scalars["fix"])
        self.nz = int(self.scalars["NZ"])
        self.nrt = int(self.scalars["NRT"])
        self.mode = self.args["mode"]

    @property
    def heavy(self):
        """Whether replaying this fixture through the CPU oracle takes more than a few
        seconds (the 128 x 128 x 256, 10-round-trip benchmark case: ~4e9 voxel-steps);
        such fixtures are compared with the FP64 CUDA path only."""
        return self.nx * self.ny * self.nt * int(self.scalars["nsteps"]) * max(1, self.nrt) > MAX_ORACLE_VOXEL_STEPS

    def initial_fields(self, noise_fn):
        """(s0, i0) regenerated from the recorded seed with the given noise function."""
        V = self.nx * self.ny * self.nt
        s0 = noise_fn(self.meta["seed"], self.meta["sigma"], V).reshape(self.nt, self.ny, self.nx)
        i0 = s0.copy() if self.meta["idler"] == "copy" else np.zeros_like(s0)
        return s0, i0

    def config_kwargs(self):
        """Keyword arguments shared by the oracle's OrPhys and the library's OpoConfig."""
        a = self.args
        extra = {}
        if "alpha_p" in a:
            extra["alpha"] = (a["alpha_p"], a["alpha_s"], a["alpha_i"])
        if "resonant" in a:
            extra["resonant"] = a["resonant"]
        return dict(extra, crystal=0 if a["crystal"] == "ppln" else 1, LX=a["LX"], LY=a["LY"],
                    Lcr=a["Lcr"], T=a["T"], Lambda=a["Lambda"], lp=a["lp"], ls=a["ls"],
                    nx=self.nx, ny=self.ny, nt=self.nt, nz=self.nz, dQ=a.get("dQ", -1.0),
                    Lcav=a.get("Lcav", 4 * a["Lcr"]), Rs=a.get("Rs", 0.98),
                    gdd_gamma=a.get("gdd", 0.0), P=a["P"], FWHM=a["FWHM"], w0=a["w0"],
                    focal=a["focal"], pump_mode=a["pump"], t_window=a.get("twin", 0.0),
                    zloop_f32=0 if self.fp64 else 1, total_rt=self.nrt)


def rel_l2(a, b):
    a, b = np.asarray(a), np.asarray(b)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))
