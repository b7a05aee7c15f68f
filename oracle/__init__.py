"""ctypes front end of the CPU oracle (test infrastructure, never the product path).

Only the test-suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
use this package, and only as the checker. ``Oracle`` wraps ``liboracle.so`` (the C
restatement in ``pawsim_oracle.c``); :func:`reference_exe` locates the reference's own
serial build produced by ``oracle/Makefile`` in ``oracle/_ref``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")


class OrcCfg(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in (
        "Nx", "Ny", "Nlay", "wall_ew", "wall_ns", "ts_scheme", "mom_scheme", "thick_scheme",
        "use_rl", "ocean_surf_drag", "wind_feedback", "use_wind", "use_fbaro", "use_relax",
        "use_wdia", "use_diavisc", "use_wdia_file", "tau_nrecs", "wdia_nrecs", "solver",
        "use_full_mg", "maxiters", "pressure_timing")] + [(n, ctypes.c_double) for n in (
        "Lx", "Ly", "dt", "tmin", "A2", "A4", "A2smag", "A4smag", "h0", "hsml", "hmin_surf",
        "hbbl", "hmin_bot", "KT00_sigma", "lin_drag", "quad_drag", "lin_drag_surf",
        "quad_drag_surf", "tau_period", "wdia_period", "conv_diff", "pi_tol", "sor_rp",
        "omega_mg")] + [("serial_corners", ctypes.c_int)]


class OrcPstats(ctypes.Structure):
    _fields_ = [("iters", ctypes.c_int), ("residual_max", ctypes.c_double),
                ("residual_rms", ctypes.c_double), ("div_max", ctypes.c_double),
                ("div_rms", ctypes.c_double)]


def reference_source() -> str:
    """The reference's model_code directory: $PAWSIM_REF_SRC, or model_code of a directory
    named `reference` beside this repository."""
    return os.environ.get("PAWSIM_REF_SRC") or os.path.join(
        os.path.dirname(os.path.dirname(HERE)), "reference", "model_code")


def build(ref: bool = True) -> None:
    """Compile liboracle.so, and the reference build when its sources are present."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    src = reference_source()
    if ref and os.path.isdir(src):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={src}"], check=True)


def _lib():
    if not os.path.exists(LIB_PATH):
        build(ref=False)
    lib = ctypes.CDLL(LIB_PATH)
    lib.orc_create.restype = ctypes.c_void_p
    lib.orc_create.argtypes = [ctypes.POINTER(OrcCfg)]
    lib.orc_destroy.argtypes = [ctypes.c_void_p]
    for fn in ("orc_set", "orc_get"):
        getattr(lib, fn).argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_double)]
        getattr(lib, fn).restype = ctypes.c_int
    lib.orc_init.argtypes = [ctypes.c_void_p]
    lib.orc_tendency.argtypes = [ctypes.c_void_p]
    lib.orc_prepare_and_core.argtypes = [ctypes.c_void_p]
    lib.orc_prelim.argtypes = [ctypes.c_void_p, ctypes.POINTER(OrcPstats)]
    lib.orc_integrator_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.orc_pressure.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(OrcPstats)]
    lib.orc_run_steps.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                  ctypes.POINTER(OrcPstats)]
    lib.orc_time.argtypes = [ctypes.c_void_p]
    lib.orc_time.restype = ctypes.c_double
    lib.orc_energy.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                               ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    lib.orc_energy.restype = ctypes.c_int
    return lib


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        _LIB = _lib()
    return _LIB


def cfg_struct(cfg, pressure_timing=None, serial_corners=1) -> OrcCfg:
    v = cfg.values
    c = OrcCfg()
    c.Nx, c.Ny, c.Nlay = v["Nx"], v["Ny"], v["Nlay"]
    c.wall_ew, c.wall_ns = int(v["useWallEW"]), int(v["useWallNS"])
    c.ts_scheme, c.mom_scheme, c.thick_scheme = (v["timeSteppingScheme"], v["momentumScheme"],
                                                 v["thicknessScheme"])
    c.use_rl, c.ocean_surf_drag, c.wind_feedback = (int(v["useRL"]), int(v["oceanSurfDrag"]),
                                                    int(v["windFeedback"]))
    c.use_wind, c.use_fbaro, c.use_relax = int(v["useWind"]), int(v["useFbaro"]), int(v["useRelax"])
    c.use_wdia, c.use_diavisc = int(v["useWDia"]), int(v["useDiaVisc"])
    c.use_wdia_file = int(bool(cfg.files.get("wDiaFile")))
    c.tau_nrecs, c.wdia_nrecs = v["tauNrecs"], v["wDiaNrecs"]
    c.solver, c.use_full_mg, c.maxiters = v["pressureSolver"], int(v["use_fullMG"]), v["maxiters"]
    c.pressure_timing = int(v["pressureTiming"] if pressure_timing is None else pressure_timing)
    c.Lx, c.Ly, c.dt, c.tmin = v["Lx"], v["Ly"], v["dt"], v["tmin"]
    for a, b in (("A2", "A2"), ("A4", "A4"), ("A2smag", "A2smag"), ("A4smag", "A4smag"),
                 ("h0", "h0"), ("hsml", "hsml"), ("hmin_surf", "hmin_surf"), ("hbbl", "hbbl"),
                 ("hmin_bot", "hmin_bot"), ("KT00_sigma", "KT00_sigma"),
                 ("lin_drag", "linDragCoeff"), ("quad_drag", "quadDragCoeff"),
                 ("lin_drag_surf", "linDragSurf"), ("quad_drag_surf", "quadDragSurf"),
                 ("tau_period", "tauPeriod"), ("wdia_period", "wDiaPeriod"),
                 ("conv_diff", "convDiff"), ("pi_tol", "tol"), ("sor_rp", "SOR_rp"),
                 ("omega_mg", "omega_MG")):
        setattr(c, a, float(v[b]))
    c.serial_corners = int(serial_corners)
    return c


class Oracle:
    """One oracle model instance loaded from a parsed config and its input fields."""

    def __init__(self, cfg, fields, pressure_timing=None, serial_corners=1):
        if cfg.values["useTracer"]:
            raise NotImplementedError("the oracle covers the tracer-free path")
        self.cfg = cfg
        self.L, self.Nx, self.Ny = cfg.values["Nlay"], cfg.values["Nx"], cfg.values["Ny"]
        self._c = cfg_struct(cfg, pressure_timing, serial_corners)
        self._m = lib().orc_create(ctypes.byref(self._c))
        if not self._m:
            raise ValueError("orc_create rejected the configuration")
        for name in ("u", "v", "h", "uRelax", "vRelax", "hRelax", "eRelax", "uTime", "vTime",
                     "eTime", "nu_u_dia", "nu_v_dia"):
            for k in range(self.L):
                self.set(name, k, fields[name][k])
        for name in ("hhs", "hhb", "uLid", "vLid", "Fbaro_x", "Fbaro_y", "hTime", "omegaz"):
            self.set(name, 0, fields[name])
        for r in range(fields["taux"].shape[0]):
            self.set("taux", r, fields["taux"][r])
            self.set("tauy", r, fields["tauy"][r])
        nw = fields["wdia_ff"].shape[0]
        for r in range(nw):
            for k in range(self.L + 1):
                self.set("wdia_ff", r * (self.L + 1) + k, fields["wdia_ff"][r, k])
        self.set("gg", 0, fields["gg"])
        if lib().orc_init(self._m) != 0:
            raise ValueError("gFile may contain only non-negative values")

    def __del__(self):
        m = getattr(self, "_m", None)
        if m:
            lib().orc_destroy(m)
            self._m = None

    def set(self, name, k, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        rc = lib().orc_set(self._m, name.encode(), k, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        if rc != 0:
            raise KeyError(name)

    def get(self, name, k=0):
        if name == "omegaz":
            out = np.empty((self.Ny + 1, self.Nx + 1))
        elif name == "gg":
            out = np.empty(self.L)
        else:
            out = np.empty((self.Ny, self.Nx))
        rc = lib().orc_get(self._m, name.encode(), k, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        if rc != 0:
            raise KeyError(f"{name}[{k}]")
        return out

    def state(self):
        return {n: np.stack([self.get(n, k) for k in range(self.L)]) for n in ("u", "v", "h")}

    def tendency(self):
        lib().orc_tendency(self._m)
        return {n: np.stack([self.get("tend_" + n, k) for k in range(self.L)]) for n in ("u", "v", "h")}

    def prepare_and_core(self):
        lib().orc_prepare_and_core(self._m)

    def prelim(self):
        st = OrcPstats()
        rc = lib().orc_prelim(self._m, ctypes.byref(st))
        if rc < 0:
            raise NotImplementedError("pressure solver not covered by the oracle")
        return st

    def integrator_step(self, n):
        lib().orc_integrator_step(self._m, n)

    def pressure(self, update_diags=True):
        st = OrcPstats()
        rc = lib().orc_pressure(self._m, int(update_diags), ctypes.byref(st))
        if rc < 0:
            raise NotImplementedError("pressure solver not covered by the oracle")
        return st

    def run(self, n0, nsteps):
        st = OrcPstats()
        rc = lib().orc_run_steps(self._m, n0, nsteps, ctypes.byref(st))
        if rc < 0:
            raise NotImplementedError("pressure solver not covered by the oracle")
        return st

    @property
    def t(self):
        return lib().orc_time(self._m)

    def energy(self, reload=False):
        """(KE, PE, Z[Nlay]) of the current state, diagnostics.c:478-700."""
        ke, pe = ctypes.c_double(), ctypes.c_double()
        z = (ctypes.c_double * self.L)()
        lib().orc_energy(self._m, int(reload), ctypes.byref(ke), ctypes.byref(pe), z)
        return ke.value, pe.value, list(z)


def reference_exe():
    """Path of the reference's serial executable, or None when it was not built."""
    p = os.path.join(REF_DIR, "PAWSIM.exe")
    return p if os.path.exists(p) else None
