"""AWSIM input files: parameter-file parsing, data-file I/O and seeded synthetic setups.

The parameter file is the AWSIM key/value format (one ``name value`` pair per line,
``matlab_common/writeParamFile.m:8-45``); data files are raw little-endian float64
with no header (``matlab_common/writeDataFile.m:16-20``):

* 2-D cell fields: Nx x Ny, x fastest (``model_code/defs.c:140-216``);
* Omegaz: (Nx+1) x (Ny+1) on the q grid, x fastest (``model_code/state.c:440-477``);
* 3-D layer fields: layer fastest, then x, then y (``model_code/defs.c:229-314``);
* wind records: record fastest, then x, then y;
* wDia records: record fastest, then interface, then x, then y
  (``model_code/defs.c:327-426``).

:func:`read_config` mirrors ``pawsim_config_defaults/read/validate``
(``model_code/config.c:42-459``) and the grid/time set-up of
``model_code/pawsim.c:126-196``. :func:`load_fields` mirrors the defaults of
``model_code/state.c:957-1100``. The synthetic set-ups at the bottom stand in for the
benchmark configurations (no public dataset is involved); each is seeded.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

# --------------------------------------------------------------------------- config

_INT_KEYS = {
    "Nlay", "Nx", "Ny", "Nt", "startIdx", "timeSteppingScheme", "momentumScheme",
    "thicknessScheme", "tracerScheme", "tauNrecs", "wDiaNrecs", "maxiters",
}
_BOOL_KEYS = {
    "useTrad", "use_MG", "use_fullMG", "pressureTiming", "writeInitDiagnostics",
    "restart", "useWallEW", "useWallNS", "useRL", "oceanSurfDrag", "windFeedback",
    "useTracer", "useBuoyancy", "useRandomForcing",
}
_SIGNED_INT_KEYS = {"mpiNx", "mpiNy"}
_REAL_KEYS = {
    "Lx", "Ly", "dt", "tmin", "tmax", "savefrequency", "savefreqAvg", "savefreqUMom",
    "savefreqVMom", "savefreqThic", "savefreqEnergy", "savefreqTracer", "savefreqEZ",
    "KT00_sigma", "h0", "hsml", "hmin_surf", "hbbl", "hmin_bot", "A2", "A4", "A2smag",
    "A4smag", "K2", "K4", "linDragCoeff", "quadDragCoeff", "linDragSurf",
    "quadDragSurf", "tauPeriod", "wDiaPeriod", "convDiff", "omega_MG",
}
_FILE_KEYS = {
    "hInitFile", "uInitFile", "vInitFile", "bInitFile", "hbFile", "hsFile", "OmegazFile",
    "gFile", "tauxFile", "tauyFile", "uLidFile", "vLidFile", "FbaroXFile", "FbaroYFile",
    "uRelaxFile", "vRelaxFile", "hRelaxFile", "eRelaxFile", "bRelaxFile", "uTimeFile",
    "vTimeFile", "hTimeFile", "eTimeFile", "bTimeFile", "wDiaFile", "diaDiffFile",
    "diaViscUFile", "diaViscVFile", "bFluxFile",
}


class ConfigError(ValueError):
    """Raised for parameter files that the reference would also reject."""


@dataclass
class Config:
    """Parsed AWSIM parameters plus the derived flags of ``config.c:285-312``."""

    values: dict = field(default_factory=dict)
    files: dict = field(default_factory=dict)
    input_dir: str = "."

    def __getattr__(self, name):
        v = self.__dict__.get("values", {})
        if name in v:
            return v[name]
        raise AttributeError(name)


def _defaults() -> dict:
    """``pawsim_config_defaults`` (config.c:42-122)."""
    return dict(
        Nlay=0, Nx=0, Ny=0, Nt=0, startIdx=0, timeSteppingScheme=5, momentumScheme=3,
        thicknessScheme=0, tracerScheme=0, Lx=0.0, Ly=0.0, dt=0.0, tmin=-1.0, tmax=0.0,
        savefrequency=0.0, savefreqAvg=0.0, savefreqUMom=0.0, savefreqVMom=0.0,
        savefreqThic=0.0, savefreqEnergy=0.0, savefreqTracer=0.0, savefreqEZ=0.0,
        KT00_sigma=1.4, h0=0.0, hsml=0.0, hmin_surf=0.0, hbbl=0.0, hmin_bot=0.0, A2=0.0,
        A4=0.0, A2smag=0.0, A4smag=0.0, K2=0.0, K4=0.0, linDragCoeff=0.0,
        quadDragCoeff=0.0, linDragSurf=0.0, quadDragSurf=0.0, tol=1e-10, SOR_rp=1.0,
        tauPeriod=0.0, wDiaPeriod=0.0, convDiff=0.0, omega_MG=2.0 / 3.0, tauNrecs=1,
        wDiaNrecs=1, maxiters=10000, pressureSolver=0, mpiNx=0, mpiNy=0, use_MG=False,
        use_fullMG=False, pressureTiming=False, writeInitDiagnostics=False, restart=False,
        useWallEW=False, useWallNS=False, useRL=True, oceanSurfDrag=True,
        windFeedback=False, useTracer=False, useBuoyancy=False, useRandomForcing=False,
        useTrad=False,
    )


def _strtoul(s: str) -> int:
    """C ``strtoul(s, NULL, 10)`` on a token: leading digits, else 0 (wrapped to 32 bits)."""
    digits = ""
    t = s.lstrip()
    neg = t.startswith("-")
    if t[:1] in "+-":
        t = t[1:]
    for ch in t:
        if not ch.isdigit():
            break
        digits += ch
    v = int(digits) if digits else 0
    return (-v) % (1 << 32) if neg else v % (1 << 32)


def _atoi(s: str) -> int:
    t = s.lstrip()
    sign = -1 if t.startswith("-") else 1
    if t[:1] in "+-":
        t = t[1:]
    digits = ""
    for ch in t:
        if not ch.isdigit():
            break
        digits += ch
    return sign * int(digits) if digits else 0


def _strtod(s: str) -> float:
    """C ``strtod``: the longest leading float literal, else 0."""
    t = s.strip()
    for end in range(len(t), 0, -1):
        try:
            return float(t[:end])
        except ValueError:
            continue
    return 0.0


def read_config(path: str) -> Config:
    """Parse and validate an AWSIM parameter file like ``pawsim_config_read/validate``.

    Also applies ``setGridDimensions`` and ``setTimeParameters`` (pawsim.c:126-196) so
    ``dx``, ``dy``, ``Nt``, ``dt``, ``tmin``, ``tmax`` and ``savefrequency`` are final.
    """
    v = _defaults()
    files = {k: "" for k in _FILE_KEYS}
    solver_given = False
    with open(path, "r") as fh:
        toks = fh.read().split()
    if len(toks) % 2:
        raise ConfigError(f"Missing value for parameter {toks[-1]}")
    for key, val in zip(toks[0::2], toks[1::2]):
        if key in _INT_KEYS:
            v[key] = _strtoul(val)
        elif key in _BOOL_KEYS:
            v[key] = _atoi(val) != 0
        elif key in _SIGNED_INT_KEYS:
            v[key] = _atoi(val)
        elif key in _REAL_KEYS:
            v[key] = _strtod(val)
        elif key == "tol":
            v["tol"] = _strtod(val)
        elif key in ("SOR_rp", "SOR_rp_min"):
            v["SOR_rp"] = _strtod(val)
        elif key == "pressureSolver":
            v["pressureSolver"] = _strtoul(val)
            solver_given = True
        elif key in _FILE_KEYS:
            files[key] = val[:255]
    if not solver_given:
        v["pressureSolver"] = 1 if v["use_MG"] else 0
    else:
        v["use_MG"] = v["pressureSolver"] != 0
    v["useWind"] = bool(files["tauxFile"] or files["tauyFile"])
    v["useFbaro"] = bool(files["FbaroXFile"] or files["FbaroYFile"])
    v["useRelax"] = bool(files["uTimeFile"] or files["vTimeFile"] or files["hTimeFile"]
                         or files["eTimeFile"] or (v["useTracer"] and files["bTimeFile"]))
    v["useWDia"] = v["useRelax"] or bool(files["wDiaFile"])
    v["useDiaDiff"] = bool(files["bFluxFile"] or files["diaDiffFile"]) or v["convDiff"] != 0
    v["useDiaVisc"] = bool(files["diaViscUFile"] or files["diaViscVFile"]) or v["convDiff"] != 0
    _validate(v)
    slash = path.rfind("/")
    input_dir = "." if slash < 0 else path[:slash]
    cfg = Config(values=v, files=files, input_dir=input_dir)
    _grid_and_time(cfg)
    return cfg


def _validate(v: dict) -> None:
    """``pawsim_config_validate`` (config.c:320-459)."""
    if v["Nlay"] == 0 or v["Nx"] == 0 or v["Ny"] == 0:
        raise ConfigError("Nlay, Nx and Ny must all be specified and positive")
    if v["Ly"] <= 0:
        raise ConfigError("Ly must be specified and positive")
    if (v["timeSteppingScheme"] > 5 or v["momentumScheme"] > 3 or v["thicknessScheme"] > 3
            or v["tracerScheme"] > 2):
        raise ConfigError("Unknown or unsupported numerical scheme identifier")
    if v["h0"] < 0:
        raise ConfigError("h0 must be non-negative")
    neg = ("hsml", "hmin_surf", "hbbl", "hmin_bot", "linDragCoeff", "quadDragCoeff",
           "linDragSurf", "quadDragSurf", "A2", "A4", "A2smag", "A4smag", "K2", "K4", "convDiff")
    if any(v[k] < 0 for k in neg) or v["tauNrecs"] == 0 or v["wDiaNrecs"] == 0:
        raise ConfigError("Invalid wind forcing parameters")
    if v["tol"] <= 0 or v["SOR_rp"] <= 0 or v["SOR_rp"] >= 2 or v["omega_MG"] <= 0 or v["maxiters"] == 0:
        raise ConfigError("Invalid pressure solver parameters")
    if v["pressureSolver"] > 2:
        raise ConfigError("Unknown pressureSolver identifier")
    if (v["mpiNx"] == 0 or v["mpiNy"] == 0) and (v["mpiNx"] != 0 or v["mpiNy"] != 0):
        raise ConfigError("mpiNx and mpiNy must both be specified or both omitted")
    if v["mpiNx"] < 0 or v["mpiNy"] < 0:
        raise ConfigError("mpiNx and mpiNy must be non-negative")
    if v["useBuoyancy"] and not v["useTracer"]:
        raise ConfigError("useBuoyancy requires useTracer in PAWSIM")
    if v["useTrad"]:
        raise ConfigError("AWSIM useTrad time stepping is not ported in PAWSIM")
    if v["useRandomForcing"]:
        raise ConfigError("AWSIM random forcing is not ported in PAWSIM; prescribe deterministic forcing instead")
    if v["timeSteppingScheme"] < 3:
        raise ConfigError("PAWSIM only supports AB1, AB2 and AB3 time stepping so far")


def _grid_and_time(cfg: Config) -> None:
    """``setGridDimensions`` and ``setTimeParameters`` (pawsim.c:126-196)."""
    v = cfg.values
    if v["Lx"] <= 0:
        v["Lx"] = v["Ly"] * v["Nx"] / v["Ny"]
    v["dx"] = v["Lx"] / v["Nx"]
    v["dy"] = v["Ly"] / v["Ny"]
    cnt = (v["Nt"] > 0) + (v["tmax"] > 0) + (v["dt"] > 0)
    if cnt != 2:
        raise ConfigError("Must specify exactly two of {Nt, tmax, dt}")
    if v["tmin"] < 0:
        v["tmin"] = v["startIdx"] * v["savefrequency"] if v["restart"] else 0.0
    if v["Nt"] == 0:
        if v["tmax"] <= v["tmin"]:
            raise ConfigError("Integration end time must exceed integration start time")
        v["Nt"] = int(math.ceil((v["tmax"] - v["tmin"]) / v["dt"]))
    if v["dt"] == 0:
        if v["tmax"] <= v["tmin"]:
            raise ConfigError("Integration end time must exceed integration start time")
        v["dt"] = (v["tmax"] - v["tmin"]) / v["Nt"]
    if v["savefrequency"] == 0:
        v["savefrequency"] = v["dt"]
    if v["tmax"] == 0:
        v["tmax"] = v["tmin"] + v["dt"] * v["Nt"]
    if v["tmin"] >= v["tmax"]:
        raise ConfigError("Integration start time exceeds integration end time")


# ----------------------------------------------------------------------- data files

def write_data(path: str, arr: np.ndarray) -> None:
    """Write an array as raw little-endian float64 in its C order (x fastest for (Ny, Nx))."""
    np.ascontiguousarray(arr, dtype="<f8").tofile(path)


def read_data(path: str, shape) -> np.ndarray:
    """Read a raw LE float64 file into ``shape`` (C order); short files raise."""
    n = int(np.prod(shape))
    a = np.fromfile(path, dtype="<f8", count=n)
    if a.size < n:
        raise ConfigError(f"Could only read {a.size} of {n} values from {path}")
    return a.reshape(shape).astype(np.float64)


def write_param_file(path: str, params: dict) -> None:
    """One ``name value`` pair per line, as writeParamFile.m does."""
    with open(path, "w") as fh:
        for k, val in params.items():
            if isinstance(val, bool):
                val = int(val)
            if isinstance(val, float):
                fh.write(f"{k} {val!r} \n")
            else:
                fh.write(f"{k} {val} \n")


def _resolve(cfg: Config, name: str) -> str:
    """Data paths are relative to the parameter file (state.c:67-87)."""
    f = cfg.files.get(name, "")
    if not f:
        return ""
    return f if f.startswith("/") else os.path.join(cfg.input_dir, f)


def load_fields(cfg: Config) -> dict:
    """Read every input named by ``cfg`` with the defaults of ``state.c:968-1006``.

    Returns numpy arrays shaped (Ny, Nx) (x fastest) or (L, Ny, Nx) for layer fields,
    omegaz (Ny+1, Nx+1), taux/tauy (nrecs, Ny, Nx), wdia_ff (nrecs, L+1, Ny, Nx), gg (L,).
    """
    v = cfg.values
    L, Nx, Ny = v["Nlay"], v["Nx"], v["Ny"]
    nt, nw = v["tauNrecs"], v["wDiaNrecs"]
    f = {
        "u": np.zeros((L, Ny, Nx)), "v": np.zeros((L, Ny, Nx)), "h": np.zeros((L, Ny, Nx)),
        "uRelax": np.zeros((L, Ny, Nx)), "vRelax": np.zeros((L, Ny, Nx)),
        "hRelax": np.full((L, Ny, Nx), 1000.0 / L),
        "eRelax": np.stack([np.full((Ny, Nx), 1000.0 * k / L) for k in range(L)]),
        "uTime": np.full((L, Ny, Nx), -1.0), "vTime": np.full((L, Ny, Nx), -1.0),
        "eTime": np.full((L, Ny, Nx), -1.0),
        "nu_u_dia": np.zeros((L, Ny, Nx)), "nu_v_dia": np.zeros((L, Ny, Nx)),
        "gg": np.full(L, 9.81), "hhb": np.zeros((Ny, Nx)), "hhs": np.zeros((Ny, Nx)),
        "omegaz": np.zeros((Ny + 1, Nx + 1)), "uLid": np.zeros((Ny, Nx)),
        "vLid": np.zeros((Ny, Nx)), "Fbaro_x": np.zeros((Ny, Nx)),
        "Fbaro_y": np.zeros((Ny, Nx)), "hTime": np.full((Ny, Nx), -1.0),
        "taux": np.zeros((nt, Ny, Nx)), "tauy": np.zeros((nt, Ny, Nx)),
        "wdia_ff": np.zeros((nw, L + 1, Ny, Nx)),
        "b": np.zeros((L, Ny, Nx)), "bRelax": np.zeros((L, Ny, Nx)), "bTime": np.full((L, Ny, Nx), -1.0),
        "kappa_dia": np.zeros((L, Ny, Nx)), "Fsurf_b": np.zeros((Ny, Nx)),
    }

    def rd2(key, name):
        p = _resolve(cfg, key)
        if p:
            f[name] = read_data(p, (Ny, Nx))

    def rd3(key, name):
        p = _resolve(cfg, key)
        if p:
            f[name] = np.moveaxis(read_data(p, (Ny, Nx, L)), 2, 0).copy()

    rd2("hsFile", "hhs")
    rd2("hbFile", "hhb")
    p = _resolve(cfg, "OmegazFile")
    if p:
        f["omegaz"] = read_data(p, (Ny + 1, Nx + 1))
    p = _resolve(cfg, "gFile")
    if p:
        f["gg"] = read_data(p, (L,))
    for key, name in (("uInitFile", "u"), ("vInitFile", "v"), ("hInitFile", "h"),
                      ("uRelaxFile", "uRelax"), ("vRelaxFile", "vRelax"),
                      ("hRelaxFile", "hRelax"), ("eRelaxFile", "eRelax"),
                      ("uTimeFile", "uTime"), ("vTimeFile", "vTime"), ("eTimeFile", "eTime"),
                      ("diaViscUFile", "nu_u_dia"), ("diaViscVFile", "nu_v_dia")):
        rd3(key, name)
    if v["useTracer"]:
        for key, name in (("bInitFile", "b"), ("bRelaxFile", "bRelax"), ("bTimeFile", "bTime"),
                          ("diaDiffFile", "kappa_dia")):
            rd3(key, name)
        rd2("bFluxFile", "Fsurf_b")
    for key, name in (("tauxFile", "taux"), ("tauyFile", "tauy")):
        p = _resolve(cfg, key)
        if p:
            f[name] = np.moveaxis(read_data(p, (Ny, Nx, nt)), 2, 0).copy()
    for key, name in (("uLidFile", "uLid"), ("vLidFile", "vLid"), ("FbaroXFile", "Fbaro_x"),
                      ("FbaroYFile", "Fbaro_y"), ("hTimeFile", "hTime")):
        rd2(key, name)
    p = _resolve(cfg, "wDiaFile")
    if p:
        a = read_data(p, (Ny, Nx, L + 1, nw))
        f["wdia_ff"] = np.transpose(a, (3, 2, 0, 1)).copy()
    if np.any(f["gg"] < 0):
        raise ConfigError("gFile may contain only non-negative values")
    return f


# ------------------------------------------------------------- synthetic set-ups

RHO0 = 1000.0


def add_tracer(param_path, scheme=2, relax_days=100.0, K2=0.0, K4=0.0, amp=1.0, seed=7, buoyancy=False):
    """Add a tracer to an existing set-up: b = amp * (sin(2 pi y / Ly) + noise) per layer
    (bInitFile), relaxation to it on relax_days (bRelaxFile, bTimeFile; <= 0 turns relaxation
    off), tracerScheme and the K2 / K4 diffusivities; ``buoyancy`` makes it an active buoyancy
    anomaly (useBuoyancy). Returns the parameter path."""
    cfg = read_config(param_path)
    v = cfg.values
    L, Nx, Ny = v["Nlay"], v["Nx"], v["Ny"]
    rng = np.random.default_rng(seed)
    y = (np.arange(Ny) + 0.5) / Ny
    b = np.stack([amp * (np.sin(2 * np.pi * (y + 0.1 * k))[:, None] * np.ones((1, Nx))
                         + 0.1 * _smoothed_noise(rng, Ny, Nx, 1.0, 3, True, True)) for k in range(L)])
    d = os.path.dirname(param_path)
    write_data(os.path.join(d, "bInit.dat"), _layer_stack(b))
    write_data(os.path.join(d, "bRelax.dat"), _layer_stack(b))
    t = relax_days * 86400.0 if relax_days > 0 else -1.0
    write_data(os.path.join(d, "bTime.dat"), _layer_stack(np.full((L, Ny, Nx), t)))
    params = {}
    with open(param_path) as fh:
        for line in fh:
            parts = line.split()
            if len(parts) >= 2:
                params[parts[0]] = parts[1]
    params.update(useTracer=1, tracerScheme=scheme, K2=K2, K4=K4, bInitFile="bInit.dat",
                  bRelaxFile="bRelax.dat", bTimeFile="bTime.dat")
    if buoyancy:
        params.update(useBuoyancy=1)
    write_param_file(param_path, params)
    return param_path


def add_diapycnal_diffusion(param_path, kappa=1e-4, flux=1e-9, conv_diff=0.0, seed=11):
    """Give an existing tracer set-up diapycnal diffusion: a diffusivity kappa (times 1 + noise/2)
    at every interface (diaDiffFile), a surface flux flux * (1 + noise) (bFluxFile) and, when
    conv_diff is not zero, convective mixing where the local reduced gravity is negative."""
    cfg = read_config(param_path)
    v = cfg.values
    L, Nx, Ny = v["Nlay"], v["Nx"], v["Ny"]
    rng = np.random.default_rng(seed)
    kap = kappa * (1 + 0.5 * np.stack([_smoothed_noise(rng, Ny, Nx, 1.0, 3, True, True) for _ in range(L)]))
    fl = flux * (1 + _smoothed_noise(rng, Ny, Nx, 1.0, 3, True, True))
    d = os.path.dirname(param_path)
    write_data(os.path.join(d, "diaDiff.dat"), _layer_stack(kap))
    write_data(os.path.join(d, "bFlux.dat"), fl)
    params = {}
    with open(param_path) as fh:
        for line in fh:
            parts = line.split()
            if len(parts) >= 2:
                params[parts[0]] = parts[1]
    params.update(diaDiffFile="diaDiff.dat", bFluxFile="bFlux.dat")
    if conv_diff:
        params.update(convDiff=conv_diff)
    write_param_file(param_path, params)
    return param_path


def _smoothed_noise(rng, ny, nx, sigma, width, periodic_x, periodic_y):
    """Gaussian white noise box-smoothed over ``width`` cells in x and y, rescaled to ``sigma``."""
    a = rng.standard_normal((ny, nx))
    if width > 1:
        half = width // 2
        for axis, per in ((1, periodic_x), (0, periodic_y)):
            if per:
                a = sum(np.roll(a, s, axis=axis) for s in range(-half, half + 1)) / width
            else:
                pad = [(0, 0), (0, 0)]
                pad[axis] = (half, half)
                b = np.pad(a, pad, mode="reflect")
                n = a.shape[axis]
                a = sum(np.take(b, range(s, s + n), axis=axis) for s in range(width)) / width
    a -= a.mean()
    sd = a.std()
    return a * (sigma / sd) if sd > 0 else a


def _layers_from_interfaces(hb, etas):
    """Layer thicknesses from the surface (0), interior interfaces and the bottom."""
    tops = [np.zeros_like(hb)] + list(etas)
    bots = list(etas) + [hb]
    return np.stack([t - b for t, b in zip(tops, bots)])


def _write_setup(outdir, params, data):
    os.makedirs(outdir, exist_ok=True)
    for fname, arr in data.items():
        write_data(os.path.join(outdir, fname), arr)
    path = os.path.join(outdir, "params.dat")
    write_param_file(path, params)
    return path


def _layer_stack(a):
    """(L, Ny, Nx) -> AWSIM 3-D order (layer fastest, then x, then y)."""
    return np.moveaxis(a, 0, 2)


def gyre(outdir, N=128, Ny=None, Ly=2000e3, H=(1000.0, 3000.0), gg=(9.81, 0.02), f0=1e-4,
         beta=2e-11, tau0=0.1, A2=500.0, A4=0.0, r_bot=1e-7, dt=900.0, Nt=100,
         solver=0, sor_rp=1.8, tol=1e-10, noise=1.0, smooth=3, seed=0, savefrequency=None,
         extra=None):
    """Wind-driven double gyre in a closed basin with a flat bottom (the CPU-runnable case
    and, at 2048^2, the headline case). Linear drag ``r_bot`` [1/s] acts on the bottom layer
    and is passed as ``linDragCoeff = r_bot * H[-1]`` [m/s]; the wind stress is kinematic
    (``tau0 / rho0``), as in examples/gyre/setparams_gyre.m:295."""
    Nx = N
    Ny = N if Ny is None else Ny
    Lx = Ly * Nx / Ny
    dy = Ly / Ny
    L = len(H)
    rng = np.random.default_rng(seed)
    y_q = np.arange(Ny + 1) * dy
    omz = 0.5 * (f0 + beta * (y_q - Ly / 2))[:, None] * np.ones((1, Nx + 1))
    y_h = (np.arange(Ny) + 0.5) * dy
    taux = (tau0 * np.cos(2 * np.pi * y_h / Ly) / RHO0)[:, None] * np.ones((1, Nx))
    hb = np.full((Ny, Nx), -float(sum(H)))
    etas, depth = [], 0.0
    for k in range(L - 1):
        depth -= H[k]
        etas.append(depth + _smoothed_noise(rng, Ny, Nx, noise, smooth, False, False))
    h = _layers_from_interfaces(hb, etas)
    params = dict(Nlay=L, Nx=Nx, Ny=Ny, Ly=Ly, Lx=Lx, dt=dt, Nt=Nt, useWallEW=1, useWallNS=1,
                  A2=A2, A4=A4, linDragCoeff=r_bot * H[-1], use_MG=int(solver == 1),
                  pressureSolver=solver, SOR_rp=sor_rp, tol=tol,
                  savefrequency=savefrequency if savefrequency else dt * Nt,
                  hInitFile="hInit.dat", hbFile="hb.dat", OmegazFile="Omegaz.dat",
                  gFile="g.dat", tauxFile="taux.dat")
    params.update(extra or {})
    data = {"hInit.dat": _layer_stack(h), "hb.dat": hb, "Omegaz.dat": omz,
            "g.dat": np.asarray(gg[:L], dtype=float), "taux.dat": taux}
    return _write_setup(outdir, params, data)


def channel(outdir, Nx=1024, Ny=512, Lx=4000e3, Ly=2000e3, H=(500.0, 1000.0, 2500.0),
            gg=(9.81, 0.01, 0.005), f0=-1e-4, beta=1.5e-11, tau0=0.15, ridge=1500.0,
            ridge_w=200e3, A4=1e10, A2=0.0, dt=150.0, Nt=500, solver=1, tol=1e-10,
            noise=2.0, smooth=3, seed=1, savefrequency=None, extra=None):
    """Zonally periodic channel with walls at north and south and a Gaussian meridional
    ridge; eastward wind ``tau0 sin^2(pi y / Ly)``; biharmonic viscosity."""
    L = len(H)
    rng = np.random.default_rng(seed)
    dx, dy = Lx / Nx, Ly / Ny
    x_h = (np.arange(Nx) + 0.5) * dx
    y_h = (np.arange(Ny) + 0.5) * dy
    y_q = np.arange(Ny + 1) * dy
    omz = 0.5 * (f0 + beta * (y_q - Ly / 2))[:, None] * np.ones((1, Nx + 1))
    hb = -float(sum(H)) + ridge * np.exp(-((x_h - Lx / 2) / ridge_w) ** 2)[None, :] * np.ones((Ny, 1))
    taux = (tau0 * np.sin(np.pi * y_h / Ly) ** 2 / RHO0)[:, None] * np.ones((1, Nx))
    etas, depth = [], 0.0
    for k in range(L - 1):
        depth -= H[k]
        etas.append(depth + _smoothed_noise(rng, Ny, Nx, noise, smooth, True, False))
    h = _layers_from_interfaces(hb, etas)
    params = dict(Nlay=L, Nx=Nx, Ny=Ny, Ly=Ly, Lx=Lx, dt=dt, Nt=Nt, useWallEW=0, useWallNS=1,
                  A2=A2, A4=A4, use_MG=int(solver == 1), pressureSolver=solver, tol=tol,
                  savefrequency=savefrequency if savefrequency else dt * Nt,
                  hInitFile="hInit.dat", hbFile="hb.dat", OmegazFile="Omegaz.dat",
                  gFile="g.dat", tauxFile="taux.dat")
    params.update(extra or {})
    data = {"hInit.dat": _layer_stack(h), "hb.dat": hb, "Omegaz.dat": omz,
            "g.dat": np.asarray(gg[:L], dtype=float), "taux.dat": taux}
    return _write_setup(outdir, params, data)


def jets(outdir, N=256, Ly=400e3, H=(500.0, 3500.0), gg=(9.81, 0.02), f0=1e-4, beta=1.6e-11,
         u0=0.5, jet_w=100e3, A2=100.0, dt=100.0, Nt=100, solver=1, tol=1e-10, noise=0.5,
         smooth=3, seed=2, savefrequency=None, extra=None):
    """Doubly periodic zonal jet: top-layer u = u0 exp(-((y-Ly/2)/w)^2), the interface in
    thermal-wind balance with the jet's zonal-mean-free part (so it stays periodic in y),
    plus seeded interface noise."""
    Nx = Ny = N
    Lx = Ly
    L = len(H)
    rng = np.random.default_rng(seed)
    dy = Ly / Ny
    y_h = (np.arange(Ny) + 0.5) * dy
    y_q = np.arange(Ny + 1) * dy
    u1 = u0 * np.exp(-((y_h - Ly / 2) / jet_w) ** 2)
    up = u1 - u1.mean()
    # thermal wind: d(eta1)/dy = f0 * (u1 - u2) / g', with u2 = 0
    deta = f0 * up / gg[1] * dy
    eta1 = -H[0] + np.cumsum(deta) - deta.sum() / 2
    eta1 = eta1 - eta1.mean() - H[0]
    omz = 0.5 * (f0 + beta * (y_q - Ly / 2))[:, None] * np.ones((1, Nx + 1))
    hb = np.full((Ny, Nx), -float(sum(H)))
    e1 = eta1[:, None] * np.ones((1, Nx)) + _smoothed_noise(rng, Ny, Nx, noise, smooth, True, True)
    h = _layers_from_interfaces(hb, [e1])
    u = np.zeros((L, Ny, Nx))
    u[0] = u1[:, None]
    params = dict(Nlay=L, Nx=Nx, Ny=Ny, Ly=Ly, Lx=Lx, dt=dt, Nt=Nt, useWallEW=0, useWallNS=0,
                  A2=A2, use_MG=int(solver == 1), pressureSolver=solver, tol=tol,
                  savefrequency=savefrequency if savefrequency else dt * Nt,
                  hInitFile="hInit.dat", uInitFile="uInit.dat", hbFile="hb.dat",
                  OmegazFile="Omegaz.dat", gFile="g.dat")
    params.update(extra or {})
    data = {"hInit.dat": _layer_stack(h), "uInit.dat": _layer_stack(u), "hb.dat": hb,
            "Omegaz.dat": omz, "g.dat": np.asarray(gg[:L], dtype=float)}
    return _write_setup(outdir, params, data)


def full_physics(outdir, N=4096, Ly=4000e3, H=(300.0, 700.0, 1500.0, 2500.0),
                 gg=(9.81, 0.03, 0.015, 0.008), f0=1e-4, beta=2e-11, tau0=0.1, A4=1e8,
                 bathy_amp=500.0, bathy_len=100e3, sponge=200e3, relax_days=30.0,
                 wdia=1e-7, dt=50.0, Nt=100, solver=1, tol=1e-10, noise=1.0, smooth=3,
                 seed=4, savefrequency=None, extra=None):
    """Closed-basin gyre with seeded random bathymetry, a boundary sponge that restores the
    interfaces to their initial heights (eRelax/eTime), a prescribed diapycnal velocity
    across every interior interface (wDiaFile) and biharmonic viscosity."""
    Nx = Ny = N
    Lx = Ly
    L = len(H)
    rng = np.random.default_rng(seed)
    d = Ly / N
    y_h = (np.arange(Ny) + 0.5) * d
    x_h = (np.arange(Nx) + 0.5) * d
    y_q = np.arange(Ny + 1) * d
    omz = 0.5 * (f0 + beta * (y_q - Ly / 2))[:, None] * np.ones((1, Nx + 1))
    taux = (tau0 * np.cos(2 * np.pi * y_h / Ly) / RHO0)[:, None] * np.ones((1, Nx))
    # Gaussian-filtered noise with correlation length bathy_len (spectral filter)
    kx = np.fft.fftfreq(Nx, d=d)[None, :]
    ky = np.fft.fftfreq(Ny, d=d)[:, None]
    filt = np.exp(-0.5 * (2 * np.pi) ** 2 * (kx ** 2 + ky ** 2) * bathy_len ** 2)
    b = np.real(np.fft.ifft2(np.fft.fft2(rng.standard_normal((Ny, Nx))) * filt))
    b = b / max(np.abs(b).max(), 1e-30) * bathy_amp
    hb = -float(sum(H)) + b
    etas, depth = [], 0.0
    for k in range(L - 1):
        depth -= H[k]
        etas.append(depth + _smoothed_noise(rng, Ny, Nx, noise, smooth, False, False))
    h = _layers_from_interfaces(hb, etas)
    X, Y = np.meshgrid(x_h, y_h)
    dist = np.minimum(np.minimum(X, Lx - X), np.minimum(Y, Ly - Y))
    in_sponge = dist < sponge
    eta_init = np.stack([np.zeros((Ny, Nx))] + etas)     # interfaces 0..L-1 (top of layer k)
    eTime = np.where(in_sponge[None], relax_days * 86400.0, -1.0) * np.ones((L, 1, 1))
    eTime[0] = -1.0                                      # the surface is not restored
    wd = np.zeros((1, L + 1, Ny, Nx))
    wd[0, 1:L] = wdia
    params = dict(Nlay=L, Nx=Nx, Ny=Ny, Ly=Ly, Lx=Lx, dt=dt, Nt=Nt, useWallEW=1, useWallNS=1,
                  A4=A4, use_MG=int(solver == 1), pressureSolver=solver, tol=tol,
                  savefrequency=savefrequency if savefrequency else dt * Nt,
                  hInitFile="hInit.dat", hbFile="hb.dat", OmegazFile="Omegaz.dat",
                  gFile="g.dat", tauxFile="taux.dat", eRelaxFile="eRelax.dat",
                  eTimeFile="eTime.dat", wDiaFile="wDia.dat")
    params.update(extra or {})
    data = {"hInit.dat": _layer_stack(h), "hb.dat": hb, "Omegaz.dat": omz,
            "g.dat": np.asarray(gg[:L], dtype=float), "taux.dat": taux,
            "eRelax.dat": _layer_stack(eta_init), "eTime.dat": _layer_stack(eTime),
            "wDia.dat": np.transpose(wd, (2, 3, 1, 0))}
    return _write_setup(outdir, params, data)
