"""Tendency budgets on the GPU (savefreqUMom, savefreqVMom, savefreqThic, savefreqEnergy,
savefreqTracer: the terms of model_code/work.c:1753-1937, forcing.c:243-389,
restoring.c:190-214, diapycnal.c:243-284 and pressure.c:2182-2245, written by
diagnostics.c:756-866).

The drop-in executable accumulates every enabled family on the device during the step
(the budget build of the fused tendency kernel, the tracer kernel and the projection) and
writes each window under the reference's names. On the committed fixtures (windows of two
steps, three for the tracer; SOR pressure, so the states are bit-identical) every budget
file must equal the reference binary's bit for bit: walled gyre with wind and drag, the
four-layer full-physics set-up (bathymetry, sponge restoring, w_dia, A4), HK83 momentum and
thickness with A4, a periodic jet with a KT00 tracer, quadratic bottom and surface drag with
wind feedback, surface/bottom layer fractions with linear surface drag and KT00 thickness, and
a buoyant tracer with diapycnal diffusion and convective mixing (diaDiff and diaVisc terms),
and velocity restoring with a barotropic body force (relaxation and baroForcing terms)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, value_equal
from golden_util import load_case

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(ROOT, "pawsim_b200", "bin", "PAWSIM_B200.exe")
CASES = ["gyre_sor_budget", "full_sor_budget", "gyre_hk83_a4_budget", "jets_tracer_budget", "gyre_quad_budget",
         "gyre_fractions_budget", "jets_diadiff_budget", "gyre_relax_fbaro_budget",
         "gyre_quad_fractions_budget"]


@pytest.mark.parametrize("name", CASES)
def test_driver_budgets_match_reference(tmp_path, name):
    from pawsim_b200 import inputs
    cfg, _, z = load_case(name, tmp_path)
    out = tmp_path / "out"
    out.mkdir()
    param = os.path.join(str(tmp_path), name, "params.dat")
    r = subprocess.run([DRIVER, param, str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    want = [str(f) for f in z["budget_files"]]
    got = sorted(f for f in os.listdir(out) if f.split("_")[0] in ("UMom", "VMom", "Thic", "Energy", "Tracer"))
    assert got == sorted(want)
    bad = []
    for f in want:
        a = inputs.read_data(str(out / f), (cfg.Ny, cfg.Nx))
        b = z["b_" + f[:-4]]
        if not value_equal(a, b):
            bad.append((f, float(np.nanmax(np.abs(a - b))), float(np.abs(b).max())))
    assert not bad, bad[:10]


def test_budget_api_scale_and_zero(tmp_path):
    """Through the Python API: the u-momentum budget accumulates over steps, scale multiplies
    every sum of the chosen families only, zero resets them."""
    import pawsim_b200 as lib
    from conftest import make_setup
    _, cfg, f = make_setup(tmp_path, "gyre", N=32, solver=0, dt=900.0,
                           extra=dict(savefreqUMom=1800.0, savefreqThic=1800.0))
    m = lib.Model(cfg, f)
    assert m._gc.budgets == 1 | 4
    m.prelim()
    m.step(1)                       # from rest: the PV flux of the first step is zero
    m.step(2)
    q1 = m.get("UMom_PVadvection", 0)
    assert np.abs(q1).max() > 0
    m.step(3)
    q2 = m.get("UMom_PVadvection", 0)
    th = m.get("Thic_advection", 1)
    assert not value_equal(q1, q2)
    m.scale_budgets(1, 0.5)
    assert value_equal(m.get("UMom_PVadvection", 0), q2 * 0.5)
    assert value_equal(m.get("Thic_advection", 1), th)
    m.zero_budgets(1)
    assert not m.get("UMom_PVadvection", 0).any()
    assert value_equal(m.get("Thic_advection", 1), th)
    with pytest.raises(lib.PawsimError):
        m.get("VMom_PVadvection", 0)     # family off: no such field
    m.close()
