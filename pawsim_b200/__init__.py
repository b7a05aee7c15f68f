"""pawsim_b200 -- B200-native timestep hot path of PAWSIM behind a C ABI.

The compute path is ``libpawsim_b200.so`` (hand-written sm_100a CUDA, see
``include/pawsim_b200.h``). This module is the Python mirror of the reference's
interface for that path: :class:`Model` is created from an AWSIM parameter file and
exposes ``tendency_eval``, ``integrator_step``, ``pressure_correct``, ``prelim`` and
``step`` with the meaning of ``pawsim_tendency_eval`` (model_code/tendency.c:81-115),
``pawsim_integrator_step`` (model_code/integrator.c:138-198) and
``pawsim_pressure_correct_rigid_lid`` (model_code/pressure.c:2254-2300). There is no CPU
fallback: importing works anywhere, but creating a model needs the built library and a
CUDA device, and fails loudly otherwise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import inputs

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpawsim_b200.so")

SOLVER_SOR, SOLVER_MG, SOLVER_MG_DISTRIBUTED = 0, 1, 2


class PawsimError(RuntimeError):
    """A negative return code of the C ABI, with the library's last error text."""

    def __init__(self, code, msg):
        super().__init__(f"pawsim_b200 error {code}: {msg}")
        self.code = code


class GpuConfig(ctypes.Structure):
    """``pawsim_gpu_config`` of include/pawsim_b200.h (field order matters)."""
    _fields_ = [(n, ctypes.c_int) for n in (
        "Nx", "Ny", "Nlay", "wall_ew", "wall_ns", "ts_scheme", "mom_scheme", "thick_scheme",
        "use_rl", "ocean_surf_drag", "wind_feedback", "use_wind", "use_fbaro", "use_relax",
        "use_wdia", "use_diavisc", "use_wdia_file", "tau_nrecs", "wdia_nrecs", "solver",
        "use_full_mg", "maxiters", "pressure_timing")] + [(n, ctypes.c_double) for n in (
        "Lx", "Ly", "dt", "tmin", "A2", "A4", "A2smag", "A4smag", "h0", "hsml", "hmin_surf",
        "hbbl", "hmin_bot", "KT00_sigma", "lin_drag", "quad_drag", "lin_drag_surf",
        "quad_drag_surf", "tau_period", "wdia_period", "conv_diff", "pi_tol", "sor_rp",
        "omega_mg")] + [("mg_fp32", ctypes.c_int), ("mg_pre", ctypes.c_int),
                        ("mg_post", ctypes.c_int), ("mg_omega", ctypes.c_double),
                        ("serial_sums", ctypes.c_int), ("mg_tile", ctypes.c_int),
                        ("use_tracer", ctypes.c_int), ("tracer_scheme", ctypes.c_int),
                        ("K2", ctypes.c_double), ("K4", ctypes.c_double),
                        ("pi_guess", ctypes.c_int), ("budgets", ctypes.c_int),
                        ("use_buoyancy", ctypes.c_int), ("use_diadiff", ctypes.c_int),
                        ("mg_fp32_inner", ctypes.c_int), ("check_nonfinite", ctypes.c_int),
                        ("fail_on_maxiters", ctypes.c_int), ("mpi_corners", ctypes.c_int)]


class GpuStats(ctypes.Structure):
    _fields_ = [("iters", ctypes.c_int), ("residual_max", ctypes.c_double),
                ("residual_rms", ctypes.c_double), ("div_max", ctypes.c_double),
                ("div_rms", ctypes.c_double), ("stop_measure", ctypes.c_double),
                ("solve_ms", ctypes.c_double), ("warm_start", ctypes.c_int), ("fallback", ctypes.c_int),
                ("mg_omega", ctypes.c_double)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


EXPORTS = (
    "pawsim_gpu_create", "pawsim_gpu_destroy", "pawsim_gpu_set_field", "pawsim_gpu_get_field",
    "pawsim_gpu_init", "pawsim_gpu_tendency_eval", "pawsim_gpu_integrator_step",
    "pawsim_gpu_pressure_correct", "pawsim_gpu_prelim", "pawsim_gpu_step", "pawsim_gpu_run",
    "pawsim_gpu_run_iterations",
    "pawsim_gpu_ensemble_create", "pawsim_gpu_ensemble_run", "pawsim_gpu_ensemble_kernel_ms",
    "pawsim_gpu_ensemble_set_graphs", "pawsim_gpu_ensemble_graph_steps", "pawsim_gpu_ensemble_batched_mg",
    "pawsim_gpu_ensemble_destroy",
    "pawsim_gpu_solve_mg", "pawsim_gpu_set_stream", "pawsim_gpu_synchronize",
    "pawsim_gpu_time", "pawsim_gpu_launch_count", "pawsim_gpu_last_error",
    "pawsim_nn_conv3x3", "pawsim_nn_conv3x3_wgrad", "pawsim_nn_flip_weights",
    "pawsim_gpu_nn_setup", "pawsim_gpu_nn_train", "pawsim_gpu_nn_pairs", "pawsim_gpu_nn_net",
    "pawsim_nn_net_create", "pawsim_nn_net_destroy", "pawsim_nn_net_param_count",
    "pawsim_nn_net_get_params", "pawsim_nn_net_set_params", "pawsim_nn_net_get_grads",
    "pawsim_nn_net_forward", "pawsim_nn_net_backward", "pawsim_nn_net_adam",
    "pawsim_gpu_accumulate_averages", "pawsim_gpu_scale_averages", "pawsim_gpu_zero_averages",
    "pawsim_gpu_energy", "pawsim_gpu_save_begin", "pawsim_gpu_save_wait", "pawsim_gpu_save_release",
    "pawsim_gpu_save_planes", "pawsim_gpu_scale_budgets", "pawsim_gpu_zero_budgets",
)

_LIB = None


def load_library(path: str = LIB_PATH):
    """Load the CUDA library (no compute happens here). Raises if it was not built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise PawsimError(-2, f"{path} is missing: run `python -m pawsim_b200.build` first")
    lib = ctypes.CDLL(path)
    P = ctypes.c_void_p
    lib.pawsim_gpu_create.argtypes = [ctypes.POINTER(GpuConfig), ctypes.POINTER(P)]
    lib.pawsim_gpu_destroy.argtypes = [P]
    lib.pawsim_gpu_destroy.restype = None
    for fn in ("pawsim_gpu_set_field", "pawsim_gpu_get_field"):
        getattr(lib, fn).argtypes = [P, ctypes.c_char_p, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_double), ctypes.c_size_t]
    lib.pawsim_gpu_init.argtypes = [P]
    lib.pawsim_gpu_tendency_eval.argtypes = [P]
    lib.pawsim_gpu_integrator_step.argtypes = [P, ctypes.c_uint]
    lib.pawsim_gpu_pressure_correct.argtypes = [P, ctypes.c_int, ctypes.POINTER(GpuStats)]
    lib.pawsim_gpu_prelim.argtypes = [P, ctypes.POINTER(GpuStats)]
    lib.pawsim_gpu_step.argtypes = [P, ctypes.c_uint, ctypes.POINTER(GpuStats)]
    lib.pawsim_gpu_run.argtypes = [P, ctypes.c_uint, ctypes.c_uint, ctypes.POINTER(GpuStats)]
    lib.pawsim_gpu_run_iterations.argtypes = [P, ctypes.POINTER(ctypes.c_int), ctypes.c_size_t]
    lib.pawsim_gpu_solve_mg.argtypes = [P, ctypes.POINTER(GpuStats)]
    lib.pawsim_gpu_ensemble_create.argtypes = [ctypes.POINTER(P), ctypes.c_int, ctypes.POINTER(P)]
    lib.pawsim_gpu_ensemble_run.argtypes = [P, ctypes.c_uint, ctypes.c_uint]
    lib.pawsim_gpu_ensemble_kernel_ms.argtypes = [P]
    lib.pawsim_gpu_ensemble_kernel_ms.restype = ctypes.c_double
    lib.pawsim_gpu_ensemble_set_graphs.argtypes = [P, ctypes.c_int]
    lib.pawsim_gpu_ensemble_graph_steps.argtypes = [P]
    lib.pawsim_gpu_ensemble_batched_mg.argtypes = [P]
    lib.pawsim_gpu_ensemble_destroy.argtypes = [P]
    lib.pawsim_gpu_ensemble_destroy.restype = None
    lib.pawsim_gpu_accumulate_averages.argtypes = [P, ctypes.c_double]
    lib.pawsim_gpu_scale_averages.argtypes = [P, ctypes.c_double]
    lib.pawsim_gpu_zero_averages.argtypes = [P]
    D = ctypes.POINTER(ctypes.c_double)
    lib.pawsim_gpu_energy.argtypes = [P, ctypes.c_int, D, D, D]
    lib.pawsim_gpu_save_begin.argtypes = [P, ctypes.POINTER(ctypes.c_int)]
    lib.pawsim_gpu_save_wait.argtypes = [P, ctypes.c_int, ctypes.POINTER(D)]
    lib.pawsim_gpu_save_release.argtypes = [P, ctypes.c_int]
    lib.pawsim_gpu_save_planes.argtypes = [P]
    lib.pawsim_gpu_save_planes.restype = ctypes.c_size_t
    lib.pawsim_gpu_scale_budgets.argtypes = [P, ctypes.c_int, ctypes.c_double]
    lib.pawsim_gpu_zero_budgets.argtypes = [P, ctypes.c_int]
    lib.pawsim_gpu_set_stream.argtypes = [P, P]
    lib.pawsim_gpu_synchronize.argtypes = [P]
    lib.pawsim_gpu_time.argtypes = [P]
    lib.pawsim_gpu_time.restype = ctypes.c_double
    lib.pawsim_gpu_launch_count.argtypes = [P]
    lib.pawsim_gpu_launch_count.restype = ctypes.c_longlong
    I, F = ctypes.c_int, ctypes.POINTER(ctypes.c_float)
    lib.pawsim_nn_conv3x3.argtypes = [P, I, I, I, I, P, P, I, I, P, P, P, P]
    lib.pawsim_nn_conv3x3_wgrad.argtypes = [P, P, I, I, I, I, I, P, P, P, P]
    lib.pawsim_nn_flip_weights.argtypes = [P, I, I, P, P]
    U64, SZ = ctypes.c_ulonglong, ctypes.c_size_t
    lib.pawsim_gpu_nn_setup.argtypes = [P, I, I, I, U64]
    lib.pawsim_gpu_nn_train.argtypes = [P, I, ctypes.c_float, ctypes.POINTER(ctypes.c_double)]
    lib.pawsim_gpu_nn_pairs.argtypes = [P]
    lib.pawsim_gpu_nn_net.argtypes = [P]
    lib.pawsim_gpu_nn_net.restype = P
    lib.pawsim_nn_net_create.argtypes = [I, I, I, U64, ctypes.POINTER(P)]
    lib.pawsim_nn_net_destroy.argtypes = [P]
    lib.pawsim_nn_net_destroy.restype = None
    lib.pawsim_nn_net_param_count.argtypes = [P]
    lib.pawsim_nn_net_param_count.restype = ctypes.c_longlong
    for fn in ("pawsim_nn_net_get_params", "pawsim_nn_net_set_params", "pawsim_nn_net_get_grads"):
        getattr(lib, fn).argtypes = [P, F, SZ]
    lib.pawsim_nn_net_forward.argtypes = [P, P, I, F]
    lib.pawsim_nn_net_backward.argtypes = [P, P, P, I, ctypes.POINTER(ctypes.c_double)]
    lib.pawsim_nn_net_adam.argtypes = [P, ctypes.c_float]
    lib.pawsim_gpu_last_error.argtypes = []
    lib.pawsim_gpu_last_error.restype = ctypes.c_char_p
    _LIB = lib
    return lib


def _check(rc):
    if rc < 0:
        raise PawsimError(rc, load_library().pawsim_gpu_last_error().decode())
    return rc


def gpu_config(cfg: inputs.Config, **over) -> GpuConfig:
    """Translate a parsed AWSIM configuration into the C ABI's struct."""
    v = cfg.values
    g = GpuConfig()
    g.Nx, g.Ny, g.Nlay = v["Nx"], v["Ny"], v["Nlay"]
    g.wall_ew, g.wall_ns = int(v["useWallEW"]), int(v["useWallNS"])
    g.ts_scheme, g.mom_scheme, g.thick_scheme = (v["timeSteppingScheme"], v["momentumScheme"],
                                                 v["thicknessScheme"])
    g.use_rl, g.ocean_surf_drag, g.wind_feedback = (int(v["useRL"]), int(v["oceanSurfDrag"]),
                                                    int(v["windFeedback"]))
    g.use_wind, g.use_fbaro, g.use_relax = int(v["useWind"]), int(v["useFbaro"]), int(v["useRelax"])
    g.use_wdia, g.use_diavisc = int(v["useWDia"]), int(v["useDiaVisc"])
    g.use_wdia_file = int(bool(cfg.files.get("wDiaFile")))
    g.tau_nrecs, g.wdia_nrecs = v["tauNrecs"], v["wDiaNrecs"]
    g.solver, g.use_full_mg, g.maxiters = v["pressureSolver"], int(v["use_fullMG"]), v["maxiters"]
    g.pressure_timing = int(v["pressureTiming"])
    g.Lx, g.Ly, g.dt, g.tmin = v["Lx"], v["Ly"], v["dt"], v["tmin"]
    for a, b in (("A2", "A2"), ("A4", "A4"), ("A2smag", "A2smag"), ("A4smag", "A4smag"),
                 ("h0", "h0"), ("hsml", "hsml"), ("hmin_surf", "hmin_surf"), ("hbbl", "hbbl"),
                 ("hmin_bot", "hmin_bot"), ("KT00_sigma", "KT00_sigma"),
                 ("lin_drag", "linDragCoeff"), ("quad_drag", "quadDragCoeff"),
                 ("lin_drag_surf", "linDragSurf"), ("quad_drag_surf", "quadDragSurf"),
                 ("tau_period", "tauPeriod"), ("wdia_period", "wDiaPeriod"),
                 ("conv_diff", "convDiff"), ("pi_tol", "tol"), ("sor_rp", "SOR_rp"),
                 ("omega_mg", "omega_MG")):
        setattr(g, a, float(v[b]))
    g.mg_fp32, g.mg_pre, g.mg_post, g.mg_omega = 0, 1, 1, -1.0   # weight chosen by the solver
    g.serial_sums = -1
    g.mg_tile = 0
    g.use_tracer, g.tracer_scheme = int(v["useTracer"]), int(v["tracerScheme"])
    g.K2, g.K4 = float(v["K2"]), float(v["K4"])
    g.use_buoyancy = int(bool(v["useBuoyancy"]) and bool(v["useTracer"]))
    g.use_diadiff = int(bool(v["useDiaDiff"]) and bool(v["useTracer"]))
    # budget families of the savefreq keys (work.c:310-319)
    g.budgets = sum(bit for bit, key in ((1, "savefreqUMom"), (2, "savefreqVMom"), (4, "savefreqThic"),
                                         (8, "savefreqEnergy"), (16, "savefreqTracer")) if v[key] > 0)
    for k, val in over.items():
        setattr(g, k, val)
    return g


class Model:
    """One model resident on the GPU (the drop-in for the reference's hot path)."""

    def __init__(self, cfg: inputs.Config, fields: dict | None = None, **options):
        self.lib = load_library()
        self.cfg = cfg
        self.L, self.Nx, self.Ny = cfg.values["Nlay"], cfg.values["Nx"], cfg.values["Ny"]
        self._gc = gpu_config(cfg, **options)
        h = ctypes.c_void_p()
        _check(self.lib.pawsim_gpu_create(ctypes.byref(self._gc), ctypes.byref(h)))
        self._h = h
        if fields is None:
            fields = inputs.load_fields(cfg)
        self.upload(fields)
        _check(self.lib.pawsim_gpu_init(self._h))

    @classmethod
    def from_param_file(cls, path: str, **options) -> "Model":
        return cls(inputs.read_config(path), **options)

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            self.lib.pawsim_gpu_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------ fields
    def set(self, name: str, k: int, arr) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64)
        _check(self.lib.pawsim_gpu_set_field(self._h, name.encode(), k,
                                             a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                             a.size))

    def get(self, name: str, k: int = 0, out: np.ndarray | None = None) -> np.ndarray:
        """Copy field `name` (layer or record k) to the host; `out` (C-contiguous float64 of
        the field's shape, e.g. a view of pinned memory) receives it when given."""
        if name == "omegaz":
            shape = (self.Ny + 1, self.Nx + 1)
        elif name == "gg":
            shape = (self.L,)
        elif name == "corner_shadow":
            shape = (4 * self.L * 2 * 4, 6)
        else:
            shape = (self.Ny, self.Nx)
        if out is None:
            out = np.empty(shape)
        elif out.shape != shape or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError(f"out must be C-contiguous float64 of shape {shape}")
        _check(self.lib.pawsim_gpu_get_field(self._h, name.encode(), k,
                                             out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                             out.size))
        return out

    def upload(self, f: dict) -> None:
        L = self.L
        for name in ("u", "v", "h", "uRelax", "vRelax", "hRelax", "eRelax", "uTime", "vTime",
                     "eTime", "nu_u_dia", "nu_v_dia"):
            for k in range(L):
                self.set(name, k, f[name][k])
        for name in ("hhs", "hhb", "uLid", "vLid", "Fbaro_x", "Fbaro_y", "hTime", "omegaz"):
            self.set(name, 0, f[name])
        for r in range(f["taux"].shape[0]):
            self.set("taux", r, f["taux"][r])
            self.set("tauy", r, f["tauy"][r])
        for r in range(f["wdia_ff"].shape[0]):
            for k in range(L + 1):
                self.set("wdia_ff", r * (L + 1) + k, f["wdia_ff"][r, k])
        self.set("gg", 0, f["gg"])
        if self._gc.use_tracer:
            for name in ("b", "bRelax", "bTime", "kappa_dia"):
                for k in range(L):
                    self.set(name, k, f[name][k])
            self.set("Fsurf_b", 0, f["Fsurf_b"])

    def state(self) -> dict:
        names = ("u", "v", "h", "b") if self._gc.use_tracer else ("u", "v", "h")
        return {n: np.stack([self.get(n, k) for k in range(self.L)]) for n in names}

    # ----------------------------------------------------------------- hot path
    def tendency_eval(self) -> dict:
        _check(self.lib.pawsim_gpu_tendency_eval(self._h))
        return {n: np.stack([self.get("dt_" + n, k) for k in range(self.L)]) for n in ("u", "v", "h")}

    def integrator_step(self, n: int) -> None:
        _check(self.lib.pawsim_gpu_integrator_step(self._h, n))

    def pressure_correct(self, update_diags: bool = True) -> dict:
        st = GpuStats()
        _check(self.lib.pawsim_gpu_pressure_correct(self._h, int(update_diags), ctypes.byref(st)))
        return st.as_dict()

    def prelim(self) -> dict:
        st = GpuStats()
        _check(self.lib.pawsim_gpu_prelim(self._h, ctypes.byref(st)))
        return st.as_dict()

    def step(self, n: int) -> dict:
        st = GpuStats()
        _check(self.lib.pawsim_gpu_step(self._h, n, ctypes.byref(st)))
        return st.as_dict()

    def run(self, n0: int, nsteps: int) -> dict:
        """nsteps steps from step n0 (enqueued without host synchronisation where the solver
        allows); the last step's report."""
        st = GpuStats()
        _check(self.lib.pawsim_gpu_run(self._h, n0, nsteps, ctypes.byref(st)))
        self._last_run = nsteps
        return st.as_dict()

    def run_iterations(self) -> np.ndarray:
        """The solve iteration count of each step of the last run."""
        n = getattr(self, "_last_run", 0)
        out = np.zeros(n, dtype=np.int32)
        _check(self.lib.pawsim_gpu_run_iterations(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n))
        return out

    def solve_mg(self) -> dict:
        st = GpuStats()
        _check(self.lib.pawsim_gpu_solve_mg(self._h, ctypes.byref(st)))
        return st.as_dict()

    # ----------------------------------------------------------------- online averages
    def accumulate_averages(self, avg_fac: float = 1.0) -> None:
        """Add avg_fac * dt times the current state to the running averages."""
        _check(self.lib.pawsim_gpu_accumulate_averages(self._h, float(avg_fac)))

    def scale_averages(self, factor: float) -> None:
        _check(self.lib.pawsim_gpu_scale_averages(self._h, float(factor)))

    def zero_averages(self) -> None:
        _check(self.lib.pawsim_gpu_zero_averages(self._h))

    def scale_budgets(self, mask: int, factor: float) -> None:
        _check(self.lib.pawsim_gpu_scale_budgets(self._h, mask, factor))

    def zero_budgets(self, mask: int = 31) -> None:
        _check(self.lib.pawsim_gpu_zero_budgets(self._h, mask))

    def save_begin(self) -> int:
        """Snapshot the state of one save on the device and start its copy to host memory;
        returns the slot (the model can step on at once)."""
        slot = ctypes.c_int()
        _check(self.lib.pawsim_gpu_save_begin(self._h, ctypes.byref(slot)))
        return slot.value

    def save_wait(self, slot: int) -> np.ndarray:
        """The planes of a save (u, v, h[, b] per layer, w_dia per interface, pi), shape
        (planes, Ny, Nx), copied out of the slot."""
        ptr = ctypes.POINTER(ctypes.c_double)()
        _check(self.lib.pawsim_gpu_save_wait(self._h, slot, ctypes.byref(ptr)))
        n = self.lib.pawsim_gpu_save_planes(self._h)
        return np.ctypeslib.as_array(ptr, shape=(n, self.Ny, self.Nx)).copy()

    def save_release(self, slot: int) -> None:
        _check(self.lib.pawsim_gpu_save_release(self._h, slot))

    def energy(self, eta_from_step_start: bool = False):
        """(KE, PE, [Z_k]) of the current state: the sums of one EZdiags.dat line
        (model_code/diagnostics.c:478-700). eta_from_step_start builds the interface heights
        from the thickness at the start of the last step, as the reference does with a free
        surface and no online averages."""
        ke, pe = ctypes.c_double(), ctypes.c_double()
        z = (ctypes.c_double * self.L)()
        _check(self.lib.pawsim_gpu_energy(self._h, int(eta_from_step_start), ctypes.byref(ke),
                                          ctypes.byref(pe), z))
        return ke.value, pe.value, list(z)

    def synchronize(self) -> None:
        _check(self.lib.pawsim_gpu_synchronize(self._h))

    # ---- learned warm start (no counterpart in the reference) ----
    def nn_setup(self, collect: bool = True, use: bool = False, max_pairs: int = 256, batch: int = 8,
                 seed: int = 1) -> None:
        """Collect training pairs after each solve and/or start solves from the network's guess."""
        mode = (1 if collect else 0) | (2 if use else 0)
        _check(self.lib.pawsim_gpu_nn_setup(self._h, mode, max_pairs, batch, seed))

    def nn_train(self, epochs: int, lr: float = 1e-3) -> float:
        loss = ctypes.c_double()
        _check(self.lib.pawsim_gpu_nn_train(self._h, epochs, lr, ctypes.byref(loss)))
        return loss.value

    def nn_pairs(self) -> int:
        return self.lib.pawsim_gpu_nn_pairs(self._h)

    def nn_net(self) -> "Net":
        h = self.lib.pawsim_gpu_nn_net(self._h)
        if not h:
            raise PawsimError(-1, "warm start not configured")
        return Net(handle=h, owner=self)

    def set_stream(self, stream_ptr: int) -> None:
        _check(self.lib.pawsim_gpu_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    @property
    def t(self) -> float:
        return self.lib.pawsim_gpu_time(self._h)

    def launch_count(self) -> int:
        return self.lib.pawsim_gpu_launch_count(self._h)


class Ensemble:
    """Several Models advanced together: per step one fused-kernel launch over all members'
    tiles, then each member's rigid-lid correction on its own stream (no host synchronisation
    until the end of a run). Members keep their own state, diagnostics and run report."""

    def __init__(self, members):
        self.lib = load_library()
        self.members = list(members)
        arr = (ctypes.c_void_p * len(self.members))(*[m._h.value for m in self.members])
        h = ctypes.c_void_p()
        _check(self.lib.pawsim_gpu_ensemble_create(arr, len(self.members), ctypes.byref(h)))
        self._h = h

    def run(self, n0: int, nsteps: int) -> None:
        _check(self.lib.pawsim_gpu_ensemble_run(self._h, n0, nsteps))
        for m in self.members:
            m._last_run = nsteps

    def set_graphs(self, on: bool) -> None:
        """Replay captured whole-step graphs where every member allows it (the default)."""
        _check(self.lib.pawsim_gpu_ensemble_set_graphs(self._h, int(on)))

    def graph_steps(self) -> int:
        """Steps of the last run that ran as graph replays."""
        return int(self.lib.pawsim_gpu_ensemble_graph_steps(self._h))

    def batched_mg(self) -> bool:
        """Whether captured steps solve all members' pressure in one batched multigrid loop."""
        return bool(self.lib.pawsim_gpu_ensemble_batched_mg(self._h))

    def kernel_ms(self) -> float:
        """Mean device time of one step's batched fused-kernel launch over the last run's
        stream-mode steps (0 when every step replayed a graph)."""
        return float(self.lib.pawsim_gpu_ensemble_kernel_ms(self._h))

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            self.lib.pawsim_gpu_ensemble_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Net:
    """A warm-start network on the GPU (standalone, or the one a Model owns)."""

    def __init__(self, H: int = 0, W: int = 0, Bmax: int = 1, seed: int = 1, handle=None, owner=None):
        self.lib = load_library()
        self._owner = owner
        if handle is not None:
            self._h, self._own = ctypes.c_void_p(handle), False
        else:
            h = ctypes.c_void_p()
            _check(self.lib.pawsim_nn_net_create(H, W, Bmax, seed, ctypes.byref(h)))
            self._h, self._own = h, True

    def close(self):
        if getattr(self, "_own", False) and self._h:
            self.lib.pawsim_nn_net_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def param_count(self) -> int:
        return int(self.lib.pawsim_nn_net_param_count(self._h))

    def _vec(self, fn, a=None):
        n = self.param_count
        if a is None:
            a = np.zeros(n, dtype=np.float32)
        a = np.ascontiguousarray(a, dtype=np.float32)
        _check(fn(self._h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n))
        return a

    def get_params(self) -> np.ndarray:
        return self._vec(self.lib.pawsim_nn_net_get_params)

    def set_params(self, p) -> None:
        self._vec(self.lib.pawsim_nn_net_set_params, p)

    def get_grads(self) -> np.ndarray:
        return self._vec(self.lib.pawsim_nn_net_get_grads)

    def forward(self, in_ptr: int, B: int, H: int, W: int) -> np.ndarray:
        out = np.zeros((B, H, W), dtype=np.float32)
        _check(self.lib.pawsim_nn_net_forward(self._h, ctypes.c_void_p(in_ptr), B,
                                              out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def backward(self, in_ptr: int, target_ptr: int, B: int) -> float:
        loss = ctypes.c_double()
        _check(self.lib.pawsim_nn_net_backward(self._h, ctypes.c_void_p(in_ptr), ctypes.c_void_p(target_ptr), B,
                                               ctypes.byref(loss)))
        return loss.value

    def adam(self, lr: float) -> None:
        _check(self.lib.pawsim_nn_net_adam(self._h, lr))
