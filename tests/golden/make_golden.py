"""Regenerate the golden fixtures from the reference's own serial build.

Run in a container where the reference sources exist (oracle/Makefile builds
oracle/_ref/PAWSIM.exe from them):  python tests/golden/make_golden.py

For each small seeded set-up this writes one ``<case>.npz`` holding the input files
themselves (parameter text and raw data files, so the fixture does not depend on the
generator), and what the reference printed and wrote: the init_* tendency dumps of
``writeInitDiagnostics 1`` (model_code/diagnostics.c:914-972), U/V/H/P after each step
(diagnostics.c:874-908) and the ``PAWSIM pressure solve`` lines of ``pressureTiming 1``
(model_code/pawsim.c:100-108). The ``*_avg`` cases hold the online-average files of
``savefreqAvg`` (diagnostics.c:378-470) instead; the ``*_ez`` cases the text of
``EZdiags.dat`` (``savefreqEZ``, diagnostics.c:478-700).
"""
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from pawsim_b200 import inputs  # noqa: E402
import oracle  # noqa: E402

NSTEPS = 3
CASES = {
    "gyre_sor": (inputs.gyre, dict(N=16, dt=900.0, solver=0, tol=1e-10)),
    "gyre_mg": (inputs.gyre, dict(N=16, dt=900.0, solver=1, tol=1e-10)),
    "gyre_hk83_a4": (inputs.gyre, dict(N=20, Ny=12, dt=600.0, solver=0, A2=0.0, A4=1e9,
                                       extra=dict(momentumScheme=1, thicknessScheme=1))),
    "channel": (inputs.channel, dict(Nx=32, Ny=16, dt=150.0, solver=1)),
    "jets": (inputs.jets, dict(N=16, dt=100.0, solver=1)),
    "full": (inputs.full_physics, dict(N=16, dt=50.0, solver=1, Ly=320e3, bathy_len=20e3,
                                       sponge=40e3)),
    "gyre_dmg": (inputs.gyre, dict(N=32, Ny=24, dt=900.0, solver=2, tol=1e-10)),
    "jets_dmg": (inputs.jets, dict(N=32, dt=100.0, solver=2)),
}
# online-average cases (savefreqAvg, diagnostics.c:307-470): windows of 2.5 steps, so the
# step that crosses a window's end adds only part of itself; SOR keeps them bit-exact
AVG_NSTEPS = 8
AVG_CASES = {
    "gyre_sor_avg": (inputs.gyre, dict(N=16, Ny=12, dt=900.0, solver=0, tol=1e-10)),
    "full_sor_avg": (inputs.full_physics, dict(N=16, dt=50.0, solver=0, Ly=320e3, bathy_len=20e3,
                                               sponge=40e3)),
}
AVG_FIELDS = ["U_avg", "V_avg", "H_avg", "M_avg", "W_avg", "HU_avg", "HV_avg", "HUU_avg", "HVV_avg",
              "HUV_avg"]
# passive tracer cases (work.c:1947-2144): the three tracer schemes with K2, K4, w_dia and
# relaxation; SOR pressure keeps them bit-exact. (set-up, its arguments, add_tracer arguments)
TRC_NSTEPS = 4
TRC_CASES = {
    "jets_tracer_kt00": (inputs.jets, dict(N=16, dt=100.0, solver=0, tol=1e-10),
                         dict(scheme=2, relax_days=100.0)),
    "gyre_tracer_up3": (inputs.gyre, dict(N=16, Ny=12, dt=900.0, solver=0, tol=1e-10),
                        dict(scheme=1, relax_days=-1.0, K2=200.0, K4=1e9)),
    "gyre_tracer_al81_hk83": (inputs.gyre, dict(N=20, Ny=12, dt=600.0, solver=0, tol=1e-10,
                                                extra=dict(thicknessScheme=1)),
                              dict(scheme=0, relax_days=30.0, K2=500.0)),
    "full_tracer_kt00": (inputs.full_physics, dict(N=16, dt=50.0, solver=0, Ly=320e3, bathy_len=20e3,
                                                   sponge=40e3, extra=dict(savefreqAvg=125.0)),
                         dict(scheme=2, relax_days=30.0, K4=1e8)),
    # the tracer as buoyancy (useBuoyancy): rigid lid, free surface, and four layers with w_dia,
    # online averages (M_avg) and the energy diagnostics (g_tot = geff - b)
    "jets_buoy_kt00": (inputs.jets, dict(N=16, dt=100.0, solver=0, tol=1e-10),
                       dict(scheme=2, relax_days=100.0, K2=100.0, amp=0.002, buoyancy=True)),
    "jets_buoy_free": (inputs.jets, dict(N=16, dt=30.0, solver=0, extra=dict(useRL=0)),
                       dict(scheme=1, relax_days=-1.0, amp=0.002, buoyancy=True)),
    "full_buoy_avg": (inputs.full_physics, dict(N=16, dt=50.0, solver=0, Ly=320e3, bathy_len=20e3, sponge=40e3,
                                                extra=dict(savefreqAvg=125.0, savefreqEZ=50.0)),
                      dict(scheme=2, relax_days=30.0, amp=0.001, buoyancy=True)),
    # diapycnal diffusion of the tracer (diaDiffFile, bFluxFile): passive on a walled gyre; as
    # buoyancy with convective mixing (convDiff) where the local reduced gravity is negative,
    # which also turns on the convective viscosity of the momentum
    "gyre_diadiff": (inputs.gyre, dict(N=16, Ny=12, dt=900.0, solver=0, tol=1e-10),
                     dict(scheme=1, relax_days=30.0, diadiff=dict(kappa=1e-4, flux=1e-8))),
    "jets_diadiff_conv": (inputs.jets, dict(N=16, dt=100.0, solver=0, tol=1e-10),
                          dict(scheme=2, relax_days=100.0, amp=0.05, buoyancy=True,
                               diadiff=dict(kappa=1e-4, flux=1e-9, conv_diff=1e-2))),
}
# energy/enstrophy cases (savefreqEZ, diagnostics.c:478-700): a rigid-lid gyre with two lines
# per step, a free-surface periodic jet (eta from the thickness of the start of the step) and a
# free-surface HK83 gyre whose online averages reload the state every step
EZ_NSTEPS = 6
EZ_CASES = {
    "gyre_sor_ez": (inputs.gyre, dict(N=16, Ny=12, dt=900.0, solver=0, tol=1e-10), 0.5),
    "jets_free_ez": (inputs.jets, dict(N=16, dt=30.0, solver=0, extra=dict(useRL=0)), 1.5),
    "gyre_hk83_free_avg_ez": (inputs.gyre, dict(N=20, Ny=12, dt=300.0, solver=0,
                                                extra=dict(useRL=0, thicknessScheme=1,
                                                           savefreqAvg=750.0)), 1.0),
}
# tendency-budget cases (savefreqUMom/VMom/Thic/Energy/Tracer, work.c:1753-1937 and the
# forcing, restoring, diapycnal and pressure terms; diagnostics.c:756-866): windows of 2 steps
# (Tracer: 3), SOR pressure so the states are bit-identical
BUD_NSTEPS = 6
BUD_PREFIXES = ["UMom_", "VMom_", "Thic_", "Energy_", "Tracer_"]
BUD_CASES = {
    "gyre_sor_budget": (inputs.gyre, dict(N=16, Ny=12, dt=900.0, solver=0, tol=1e-10), None),
    "full_sor_budget": (inputs.full_physics, dict(N=16, dt=50.0, solver=0, Ly=320e3, bathy_len=20e3,
                                                  sponge=40e3), None),
    "gyre_hk83_a4_budget": (inputs.gyre, dict(N=20, Ny=12, dt=600.0, solver=0, A2=0.0, A4=1e9,
                                              extra=dict(momentumScheme=1, thicknessScheme=1)), None),
    "jets_tracer_budget": (inputs.jets, dict(N=16, dt=100.0, solver=0, tol=1e-10),
                           dict(scheme=2, relax_days=100.0, K2=100.0)),
    "gyre_quad_budget": (inputs.gyre, dict(N=20, Ny=12, dt=600.0, solver=0,
                                           extra=dict(quadDragCoeff=2e-3, quadDragSurf=1e-3, windFeedback=1,
                                                      oceanSurfDrag=0)), None),
    "jets_diadiff_budget": (inputs.jets, dict(N=16, dt=100.0, solver=0, tol=1e-10),
                            dict(scheme=2, relax_days=100.0, amp=0.05, buoyancy=True,
                                 diadiff=dict(kappa=1e-4, flux=1e-9, conv_diff=1e-2))),
    "gyre_relax_fbaro_budget": (inputs.gyre, dict(N=16, Ny=12, dt=900.0, solver=0, tol=1e-10), "relax"),
    "gyre_fractions_budget": (inputs.gyre, dict(N=20, Ny=12, dt=600.0, solver=0,
                                                extra=dict(hsml=1500.0, hmin_surf=5.0, hbbl=500.0, hmin_bot=10.0,
                                                           linDragSurf=1e-4, thicknessScheme=3)), None),
    # quadratic bottom and surface drag over boundary layers that span both layers
    "gyre_quad_fractions_budget": (inputs.gyre, dict(N=20, Ny=12, dt=600.0, solver=0,
                                                     extra=dict(quadDragCoeff=2e-3, hbbl=3500.0, hmin_bot=10.0,
                                                                quadDragSurf=1e-3, hsml=1200.0, hmin_surf=5.0,
                                                                windFeedback=1, oceanSurfDrag=1)), None),
}
# the acceptance point of the plain FP64 path: config 0 (128 x 128 x 2 double gyre, red-black
# SOR with SOR_rp 1.8, tol 1e-10) at its stable dt of 900 s, 100 steps; the fixture keeps every
# step's pressure line and the state after step 100
LONG_NSTEPS = 100
LONG_KEEP = (100,)
LONG_CASES = {
    "config0_sor_100": (inputs.gyre, dict(N=128, dt=900.0, solver=0, tol=1e-10, sor_rp=1.8)),
}
# x-periodic, y-walled channels without pressureTiming: the serial build's corner ghosts keep
# the values of each work array's previous fill (model_code/field.c:353-532); U/V/H/P (and B)
# after each step. SOR keeps the states bit-exact. (set-up, arguments, tracer arguments)
CORNER_NSTEPS = 6
CORNER_CASES = {
    "channel_corners_sor": (inputs.channel, dict(Nx=32, Ny=16, dt=150.0, solver=0), None),
    "channel_corners_hk83": (inputs.channel, dict(Nx=40, Ny=16, dt=150.0, solver=0, A2=200.0, A4=0.0,
                                                  extra=dict(momentumScheme=1, thicknessScheme=1)), None),
    "channel_corners_free": (inputs.channel, dict(Nx=32, Ny=16, dt=20.0, solver=0, A2=200.0, A4=0.0,
                                                  extra=dict(useRL=0, thicknessScheme=1)), None),
    "channel_corners_tracer": (inputs.channel, dict(Nx=32, Ny=16, dt=150.0, solver=0),
                               dict(scheme=2, relax_days=30.0, K2=100.0)),
}
LINE = re.compile(r"iters=(\d+) walltime=\S+ s residual_max=(\S+) residual_rms=(\S+) "
                  r"div_max=(\S+) div_rms=(\S+)")


def add_tracer_and_mixing(p, tkw):
    """add_tracer with the arguments of tkw; its "diadiff" entry, if any, goes to
    add_diapycnal_diffusion."""
    tkw = dict(tkw)
    dd = tkw.pop("diadiff", None)
    inputs.add_tracer(p, **tkw)
    if dd:
        inputs.add_diapycnal_diffusion(p, **dd)


def add_relax_fbaro(p, days=20.0, fbaro=1e-6, seed=5):
    """Velocity restoring (uRelax/vRelax towards a seeded field on `days`, uTime/vTime) and a
    barotropic body force (FbaroX/FbaroY) added to an existing set-up."""
    cfg = inputs.read_config(p)
    v = cfg.values
    L, Nx, Ny = v["Nlay"], v["Nx"], v["Ny"]
    rng = np.random.default_rng(seed)
    d = os.path.dirname(p)
    ur = 0.05 * rng.standard_normal((L, Ny, Nx))
    vr = 0.05 * rng.standard_normal((L, Ny, Nx))
    t = np.full((L, Ny, Nx), days * 86400.0)
    inputs.write_data(os.path.join(d, "uRelax.dat"), inputs._layer_stack(ur))
    inputs.write_data(os.path.join(d, "vRelax.dat"), inputs._layer_stack(vr))
    inputs.write_data(os.path.join(d, "uTime.dat"), inputs._layer_stack(t))
    inputs.write_data(os.path.join(d, "vTime.dat"), inputs._layer_stack(t))
    inputs.write_data(os.path.join(d, "FbaroX.dat"), fbaro * (1 + 0.1 * rng.standard_normal((Ny, Nx))))
    inputs.write_data(os.path.join(d, "FbaroY.dat"), fbaro * 0.1 * rng.standard_normal((Ny, Nx)))
    params = {}
    with open(p) as fh:
        for line in fh:
            parts = line.split()
            if len(parts) >= 2:
                params[parts[0]] = parts[1]
    params.update(uRelaxFile="uRelax.dat", vRelaxFile="vRelax.dat", uTimeFile="uTime.dat", vTimeFile="vTime.dat",
                  FbaroXFile="FbaroX.dat", FbaroYFile="FbaroY.dat")
    inputs.write_param_file(p, params)


def make(name, fn, kw, outdir):
    with tempfile.TemporaryDirectory() as d:
        kw = dict(kw)
        extra = dict(kw.pop("extra", {}) or {})
        extra.update(writeInitDiagnostics=1, pressureTiming=1)
        dt = kw["dt"]
        p = fn(os.path.join(d, "in"), Nt=NSTEPS, savefrequency=dt, extra=extra, **kw)
        cfg = inputs.read_config(p)
        out = os.path.join(d, "out")
        os.makedirs(out)
        r = subprocess.run([oracle.reference_exe(), p, out], capture_output=True, text=True, check=True)
        stats = np.array([[float(x) for x in m.groups()] for m in LINE.finditer(r.stdout)])
        L, Nx, Ny = cfg.Nlay, cfg.Nx, cfg.Ny
        rec = {"stats": stats, "param_text": np.array(open(p).read())}
        for f in sorted(os.listdir(os.path.dirname(p))):
            if f.endswith(".dat") and f != "params.dat":
                rec["in_" + f] = np.fromfile(os.path.join(os.path.dirname(p), f), dtype="<f8")
        for k in range(L):
            for tag in ("dudt", "dvdt", "dhdt"):
                rec[f"init_{tag}{k}"] = inputs.read_data(os.path.join(out, f"init_{tag}{k}_n=0.dat"), (Ny, Nx))
            for n in range(1, NSTEPS + 1):
                for v in ("U", "V", "H"):
                    rec[f"{v}{k}_{n}"] = inputs.read_data(os.path.join(out, f"{v}{k}_n={n}.dat"), (Ny, Nx))
        for n in range(1, NSTEPS + 1):
            rec[f"P_{n}"] = inputs.read_data(os.path.join(out, f"P_n={n}.dat"), (Ny, Nx))
        np.savez_compressed(os.path.join(outdir, name + ".npz"), **rec)


def make_long(name, fn, kw, outdir):
    """Inputs, every step's pressure line (iterations and the four norms) and U/V/H/P after
    the steps of LONG_KEEP."""
    with tempfile.TemporaryDirectory() as d:
        kw = dict(kw)
        extra = dict(kw.pop("extra", {}) or {})
        extra.update(pressureTiming=1)
        dt = kw["dt"]
        p = fn(os.path.join(d, "in"), Nt=LONG_NSTEPS, savefrequency=dt, extra=extra, **kw)
        cfg = inputs.read_config(p)
        out = os.path.join(d, "out")
        os.makedirs(out)
        r = subprocess.run([oracle.reference_exe(), p, out], capture_output=True, text=True, check=True)
        stats = np.array([[float(x) for x in m.groups()] for m in LINE.finditer(r.stdout)])
        rec = {"stats": stats, "param_text": np.array(open(p).read()), "keep": np.array(LONG_KEEP)}
        for f in sorted(os.listdir(os.path.dirname(p))):
            if f.endswith(".dat") and f != "params.dat":
                rec["in_" + f] = np.fromfile(os.path.join(os.path.dirname(p), f), dtype="<f8")
        for n in LONG_KEEP:
            for k in range(cfg.Nlay):
                for v in ("U", "V", "H"):
                    rec[f"{v}{k}_{n}"] = inputs.read_data(os.path.join(out, f"{v}{k}_n={n}.dat"), (cfg.Ny, cfg.Nx))
            rec[f"P_{n}"] = inputs.read_data(os.path.join(out, f"P_n={n}.dat"), (cfg.Ny, cfg.Nx))
        np.savez_compressed(os.path.join(outdir, name + ".npz"), **rec)


def make_corner(name, fn, kw, tkw, outdir):
    """Inputs and the reference's U/V/H(/B)/P after each step, pressureTiming off."""
    with tempfile.TemporaryDirectory() as d:
        kw = dict(kw)
        extra = dict(kw.pop("extra", {}) or {})
        extra.update(pressureTiming=0)
        dt = kw["dt"]
        p = fn(os.path.join(d, "in"), Nt=CORNER_NSTEPS, savefrequency=dt, extra=extra, **kw)
        if tkw is not None:
            add_tracer_and_mixing(p, tkw)
        cfg = inputs.read_config(p)
        out = os.path.join(d, "out")
        os.makedirs(out)
        subprocess.run([oracle.reference_exe(), p, out], capture_output=True, text=True, check=True)
        rec = {"param_text": np.array(open(p).read())}
        for f in sorted(os.listdir(os.path.dirname(p))):
            if f.endswith(".dat") and f != "params.dat":
                rec["in_" + f] = np.fromfile(os.path.join(os.path.dirname(p), f), dtype="<f8")
        names = ("U", "V", "H", "B") if tkw is not None else ("U", "V", "H")
        for n in range(1, CORNER_NSTEPS + 1):
            for k in range(cfg.Nlay):
                for v in names:
                    rec[f"{v}{k}_{n}"] = inputs.read_data(os.path.join(out, f"{v}{k}_n={n}.dat"), (cfg.Ny, cfg.Nx))
            if cfg.values["useRL"]:
                rec[f"P_{n}"] = inputs.read_data(os.path.join(out, f"P_n={n}.dat"), (cfg.Ny, cfg.Nx))
        np.savez_compressed(os.path.join(outdir, name + ".npz"), **rec)


def make_avg(name, fn, kw, outdir):
    """Inputs and the reference's online-average files of every completed window."""
    with tempfile.TemporaryDirectory() as d:
        kw = dict(kw)
        extra = dict(kw.pop("extra", {}) or {})
        dt = kw["dt"]
        extra.update(savefreqAvg=2.5 * dt)
        p = fn(os.path.join(d, "in"), Nt=AVG_NSTEPS, savefrequency=4 * dt, extra=extra, **kw)
        cfg = inputs.read_config(p)
        out = os.path.join(d, "out")
        os.makedirs(out)
        subprocess.run([oracle.reference_exe(), p, out], capture_output=True, text=True, check=True)
        L, Nx, Ny = cfg.Nlay, cfg.Nx, cfg.Ny
        rec = {"param_text": np.array(open(p).read())}
        for f in sorted(os.listdir(os.path.dirname(p))):
            if f.endswith(".dat") and f != "params.dat":
                rec["in_" + f] = np.fromfile(os.path.join(os.path.dirname(p), f), dtype="<f8")
        windows = sorted({int(f.split("_n=")[1][:-4]) for f in os.listdir(out) if f.startswith("U_avg0_n=")})
        rec["windows"] = np.array(windows)
        for n in windows:
            for k in range(L):
                for fld in AVG_FIELDS:
                    rec[f"{fld}{k}_{n}"] = inputs.read_data(os.path.join(out, f"{fld}{k}_n={n}.dat"), (Ny, Nx))
            rec[f"W_avg{L}_{n}"] = inputs.read_data(os.path.join(out, f"W_avg{L}_n={n}.dat"), (Ny, Nx))
            rec[f"P_avg_{n}"] = inputs.read_data(os.path.join(out, f"P_avg_n={n}.dat"), (Ny, Nx))
        np.savez_compressed(os.path.join(outdir, name + ".npz"), **rec)


def make_tracer(name, fn, kw, tkw, outdir):
    """Inputs (with the tracer files) and the reference's U/V/H/B/P after each step, plus the
    online-average files when the set-up asks for them."""
    with tempfile.TemporaryDirectory() as d:
        kw = dict(kw)
        extra = dict(kw.pop("extra", {}) or {})
        dt = kw["dt"]
        p = fn(os.path.join(d, "in"), Nt=TRC_NSTEPS, savefrequency=dt, extra=extra, **kw)
        add_tracer_and_mixing(p, tkw)
        cfg = inputs.read_config(p)
        out = os.path.join(d, "out")
        os.makedirs(out)
        subprocess.run([oracle.reference_exe(), p, out], capture_output=True, text=True, check=True)
        L, Nx, Ny = cfg.Nlay, cfg.Nx, cfg.Ny
        rec = {"param_text": np.array(open(p).read())}
        for f in sorted(os.listdir(os.path.dirname(p))):
            if f.endswith(".dat") and f != "params.dat":
                rec["in_" + f] = np.fromfile(os.path.join(os.path.dirname(p), f), dtype="<f8")
        for n in range(0, TRC_NSTEPS + 1):
            for k in range(L):
                for v in ("U", "V", "H", "B"):
                    rec[f"{v}{k}_{n}"] = inputs.read_data(os.path.join(out, f"{v}{k}_n={n}.dat"), (Ny, Nx))
            if cfg.values["useRL"]:
                rec[f"P_{n}"] = inputs.read_data(os.path.join(out, f"P_n={n}.dat"), (Ny, Nx))
        windows = sorted({int(f.split("_n=")[1][:-4]) for f in os.listdir(out) if f.startswith("B_avg0_n=")})
        rec["windows"] = np.array(windows, dtype=int)
        for n in windows:
            for k in range(L):
                rec[f"B_avg{k}_{n}"] = inputs.read_data(os.path.join(out, f"B_avg{k}_n={n}.dat"), (Ny, Nx))
                rec[f"U_avg{k}_{n}"] = inputs.read_data(os.path.join(out, f"U_avg{k}_n={n}.dat"), (Ny, Nx))
                rec[f"M_avg{k}_{n}"] = inputs.read_data(os.path.join(out, f"M_avg{k}_n={n}.dat"), (Ny, Nx))
        if os.path.exists(os.path.join(out, "EZdiags.dat")):
            rec["ez_text"] = np.array(open(os.path.join(out, "EZdiags.dat")).read())
        np.savez_compressed(os.path.join(outdir, name + ".npz"), **rec)


def make_ez(name, fn, kw, every, outdir):
    """Inputs and the reference's EZdiags.dat text (savefreqEZ = every * dt)."""
    with tempfile.TemporaryDirectory() as d:
        kw = dict(kw)
        extra = dict(kw.pop("extra", {}) or {})
        dt = kw["dt"]
        extra.update(savefreqEZ=every * dt)
        p = fn(os.path.join(d, "in"), Nt=EZ_NSTEPS, savefrequency=EZ_NSTEPS * dt, extra=extra, **kw)
        out = os.path.join(d, "out")
        os.makedirs(out)
        subprocess.run([oracle.reference_exe(), p, out], capture_output=True, text=True, check=True)
        rec = {"param_text": np.array(open(p).read())}
        for f in sorted(os.listdir(os.path.dirname(p))):
            if f.endswith(".dat") and f != "params.dat":
                rec["in_" + f] = np.fromfile(os.path.join(os.path.dirname(p), f), dtype="<f8")
        rec["ez_text"] = np.array(open(os.path.join(out, "EZdiags.dat")).read())
        np.savez_compressed(os.path.join(outdir, name + ".npz"), **rec)


def make_budget(name, fn, kw, tkw, outdir, relax=False):
    """Inputs and the reference's budget files of every completed window."""
    with tempfile.TemporaryDirectory() as d:
        kw = dict(kw)
        extra = dict(kw.pop("extra", {}) or {})
        dt = kw["dt"]
        extra.update(savefreqUMom=2 * dt, savefreqVMom=2 * dt, savefreqThic=2 * dt, savefreqEnergy=2 * dt)
        if tkw is not None:
            extra.update(savefreqTracer=3 * dt)
        p = fn(os.path.join(d, "in"), Nt=BUD_NSTEPS, savefrequency=BUD_NSTEPS * dt, extra=extra, **kw)
        if tkw is not None:
            add_tracer_and_mixing(p, tkw)
        if relax:
            add_relax_fbaro(p)
        cfg = inputs.read_config(p)
        out = os.path.join(d, "out")
        os.makedirs(out)
        subprocess.run([oracle.reference_exe(), p, out], capture_output=True, text=True, check=True)
        rec = {"param_text": np.array(open(p).read())}
        for f in sorted(os.listdir(os.path.dirname(p))):
            if f.endswith(".dat") and f != "params.dat":
                rec["in_" + f] = np.fromfile(os.path.join(os.path.dirname(p), f), dtype="<f8")
        names = sorted(f for f in os.listdir(out) if any(f.startswith(x) for x in BUD_PREFIXES))
        rec["budget_files"] = np.array(names)
        for f in names:
            rec["b_" + f[:-4]] = inputs.read_data(os.path.join(out, f), (cfg.Ny, cfg.Nx))
        np.savez_compressed(os.path.join(outdir, name + ".npz"), **rec)


if __name__ == "__main__":
    # python tests/golden/make_golden.py [case ...]   (all cases when none are named)
    oracle.build(ref=True)
    for name, (fn, kw) in CASES.items():
        if len(sys.argv) > 1 and name not in sys.argv[1:]:
            continue
        make(name, fn, kw, HERE)
        print("wrote", name)
    for name, (fn, kw) in LONG_CASES.items():
        if len(sys.argv) > 1 and name not in sys.argv[1:]:
            continue
        make_long(name, fn, kw, HERE)
        print("wrote", name)
    for name, (fn, kw, tkw) in CORNER_CASES.items():
        if len(sys.argv) > 1 and name not in sys.argv[1:]:
            continue
        make_corner(name, fn, kw, tkw, HERE)
        print("wrote", name)
    for name, (fn, kw) in AVG_CASES.items():
        if len(sys.argv) > 1 and name not in sys.argv[1:]:
            continue
        make_avg(name, fn, kw, HERE)
        print("wrote", name)
    for name, (fn, kw, tkw) in TRC_CASES.items():
        if len(sys.argv) > 1 and name not in sys.argv[1:]:
            continue
        make_tracer(name, fn, kw, tkw, HERE)
        print("wrote", name)
    for name, (fn, kw, every) in EZ_CASES.items():
        if len(sys.argv) > 1 and name not in sys.argv[1:]:
            continue
        make_ez(name, fn, kw, every, HERE)
        print("wrote", name)
    for name, (fn, kw, tkw) in BUD_CASES.items():
        if len(sys.argv) > 1 and name not in sys.argv[1:]:
            continue
        if tkw == "relax":
            make_budget(name, fn, kw, None, HERE, relax=True)
        else:
            make_budget(name, fn, kw, tkw, HERE)
        print("wrote", name)
