"""The oracle against the reference binary (built here from its sources) on the optional
physics the GPU kernel supports: UP3/KT00 thickness, Smagorinsky A2/A4, quadratic drag,
surface/bottom layer fractions -- U/V/H after each of 4 steps, bit for bit."""
import os
import subprocess

import numpy as np
import pytest

from conftest import make_setup

CASES = {
    "up3": ("gyre", dict(N=24, Ny=16, dt=600.0, solver=0, extra=dict(thicknessScheme=2, momentumScheme=0))),
    "kt00_jets": ("jets", dict(N=24, dt=100.0, solver=1, extra=dict(thicknessScheme=3))),
    "smag_a4": ("channel", dict(Nx=32, Ny=16, dt=150.0, solver=0, extra=dict(A4smag=1.0, A4=1e9))),
    "smag_a2": ("gyre", dict(N=24, Ny=16, dt=600.0, solver=0, extra=dict(A2smag=2.0))),
    "quad_surf": ("gyre", dict(N=24, Ny=16, dt=600.0, solver=0, extra=dict(quadDragSurf=1e-3, windFeedback=1))),
    "fractions": ("gyre", dict(N=24, Ny=16, dt=600.0, solver=0,
                               extra=dict(hsml=1500.0, hbbl=500.0, linDragSurf=1e-4))),
    "quad_hbbl": ("gyre", dict(N=24, Ny=16, dt=600.0, solver=0, extra=dict(quadDragCoeff=2e-3, hbbl=500.0, hmin_bot=10.0))),
    "quad_hbbl_deep": ("gyre", dict(N=24, Ny=16, dt=600.0, solver=0,
                                    extra=dict(quadDragCoeff=2e-3, hbbl=3500.0, hmin_bot=10.0))),
    "quad_surf_hsml": ("gyre", dict(N=24, Ny=16, dt=600.0, solver=0,
                                    extra=dict(quadDragSurf=1e-3, windFeedback=1, oceanSurfDrag=1, hsml=1200.0,
                                               hmin_surf=5.0))),
    "quad_both_fractions_jets": ("jets", dict(N=24, dt=100.0, solver=0,
                                              extra=dict(quadDragCoeff=2e-3, hbbl=3800.0, quadDragSurf=1e-3,
                                                         hsml=700.0, thicknessScheme=1))),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_physics_matches_reference(tmp_path, oracle_mod, name):
    exe = oracle_mod.reference_exe()
    if exe is None:
        pytest.skip("reference binary not built (no reference sources here)")
    from pawsim_b200 import inputs
    kind, kw = CASES[name]
    kw = dict(kw)
    extra = dict(kw.pop("extra"))
    extra["pressureTiming"] = 1
    p, cfg, f = make_setup(tmp_path, kind, Nt=4, savefrequency=kw["dt"], extra=extra, **kw)
    out = tmp_path / "out"
    out.mkdir()
    subprocess.run([exe, p, str(out)], check=True, capture_output=True)
    o = oracle_mod.Oracle(cfg, f)
    o.prelim()
    for n in range(1, 5):
        o.integrator_step(n)
        o.pressure(True)
        s = o.state()
        for k in range(cfg.Nlay):
            for v, fn in (("u", "U"), ("v", "V"), ("h", "H")):
                ref = inputs.read_data(os.path.join(out, f"{fn}{k}_n={n}.dat"), (cfg.Ny, cfg.Nx))
                assert np.array_equal(s[v][k], ref), (name, n, v, k)
