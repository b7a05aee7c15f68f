"""The passive tracer on the GPU (model_code/work.c:1947-2144 and the AB update of
integrator.c), against the reference binary's own outputs on the committed fixtures: the
three tracer schemes (AL81, UP3, KT00) with Laplacian and biharmonic diffusion, diapycnal
advection by w_dia, relaxation to bRelax, walled and doubly periodic grids, AL81 and HK83
face thickness. SOR pressure keeps the runs bit-exact, so every B file (and U, V, H, P)
must equal the reference's bit for bit, through the drop-in executable and through the
Python API; B_avg (savefreqAvg) likewise. With useBuoyancy the tracer is a buoyancy anomaly
(Bernoulli pressure, -hz db/dx in the momentum, g' in the tracer's diapycnal jumps): rigid
lid, free surface, and four layers with w_dia whose M_avg and EZdiags.dat (g_tot = geff - b)
must also match. Diapycnal diffusion (diaDiffFile, bFluxFile): passive on a walled gyre, and
as buoyancy with convective mixing (convDiff) where the local reduced gravity is negative,
which also drives the convective viscosity of the momentum."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, value_equal
from golden_util import load_case

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(ROOT, "pawsim_b200", "bin", "PAWSIM_B200.exe")
CASES = ["jets_tracer_kt00", "gyre_tracer_up3", "gyre_tracer_al81_hk83", "full_tracer_kt00",
         "jets_buoy_kt00", "jets_buoy_free", "full_buoy_avg", "gyre_diadiff", "jets_diadiff_conv"]
NSTEPS = 4


@pytest.mark.parametrize("name", CASES)
def test_driver_tracer_matches_reference(tmp_path, name):
    from pawsim_b200 import inputs
    cfg, _, z = load_case(name, tmp_path)
    out = tmp_path / "out"
    out.mkdir()
    param = os.path.join(str(tmp_path), name, "params.dat")
    r = subprocess.run([DRIVER, param, str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    shape = (cfg.Ny, cfg.Nx)
    for n in range(0, NSTEPS + 1):
        for k in range(cfg.Nlay):
            for v in ("B", "U", "V", "H"):
                got = inputs.read_data(str(out / f"{v}{k}_n={n}.dat"), shape)
                ref = z[f"{v}{k}_{n}"]
                assert value_equal(got, ref), (n, v, k, np.abs(got - ref).max())
        if cfg.values["useRL"]:
            assert value_equal(inputs.read_data(str(out / f"P_n={n}.dat"), shape), z[f"P_{n}"]), n
    for n in [int(w) for w in z["windows"]]:
        for k in range(cfg.Nlay):
            for v in ("B_avg", "U_avg", "M_avg"):
                if f"{v}{k}_{n}" not in z.files:
                    continue
                got = inputs.read_data(str(out / f"{v}{k}_n={n}.dat"), shape)
                assert value_equal(got, z[f"{v}{k}_{n}"]), (n, v, k)
    if "ez_text" in z.files:
        assert (out / "EZdiags.dat").read_text() == str(z["ez_text"])


@pytest.mark.parametrize("name", ["jets_tracer_kt00", "gyre_tracer_up3"])
def test_api_tracer_steps(tmp_path, name):
    import pawsim_b200 as lib
    cfg, f, z = load_case(name, tmp_path)
    m = lib.Model(cfg, f)
    m.prelim()
    assert value_equal(m.get("b", 0), z["B0_0"])
    for n in range(1, NSTEPS + 1):
        m.step(n)
        s = m.state()
        for k in range(cfg.Nlay):
            assert value_equal(s["b"][k], z[f"B{k}_{n}"]), (n, k)
    m.close()
