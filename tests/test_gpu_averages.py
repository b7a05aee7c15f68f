"""Online time averages (savefreqAvg, model_code/diagnostics.c:307-470) on the GPU.

The drop-in executable accumulates the running sums on the device after every step and
writes each completed window under AWSIM's names. On the committed fixtures (windows of
2.5 steps, so the step that crosses a window's end adds only its share; SOR pressure, so the
states are bit-identical) every average file must equal the reference binary's bit for bit:
u, v, h, the Montgomery potential plus pi, w_dia on every interface, the face-thickness
fluxes and their squares, the q-point product and pi."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, value_equal
from golden_util import load_case

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(ROOT, "pawsim_b200", "bin", "PAWSIM_B200.exe")
FIELDS = ["U_avg", "V_avg", "H_avg", "M_avg", "W_avg", "HU_avg", "HV_avg", "HUU_avg", "HVV_avg", "HUV_avg"]


@pytest.mark.parametrize("name", ["gyre_sor_avg", "full_sor_avg"])
def test_driver_averages_match_reference(tmp_path, name):
    from pawsim_b200 import inputs
    cfg, _, z = load_case(name, tmp_path)
    out = tmp_path / "out"
    out.mkdir()
    param = os.path.join(str(tmp_path), name, "params.dat")
    r = subprocess.run([DRIVER, param, str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    shape = (cfg.Ny, cfg.Nx)
    windows = [int(n) for n in z["windows"]]
    assert len(windows) == 3
    for n in windows:
        for k in range(cfg.Nlay):
            for f in FIELDS:
                got = inputs.read_data(str(out / f"{f}{k}_n={n}.dat"), shape)
                assert value_equal(got, z[f"{f}{k}_{n}"]), (n, f, k, np.abs(got - z[f"{f}{k}_{n}"]).max())
        got = inputs.read_data(str(out / f"W_avg{cfg.Nlay}_n={n}.dat"), shape)
        assert value_equal(got, z[f"W_avg{cfg.Nlay}_{n}"]), n
        got = inputs.read_data(str(out / f"P_avg_n={n}.dat"), shape)
        assert value_equal(got, z[f"P_avg_{n}"]), n
    assert not os.path.exists(out / f"U_avg0_n={windows[-1] + 1}.dat")


def test_average_api_sums_scale_and_reset(tmp_path):
    """Through the Python API: two accumulations with weight 1 give dt*u1 + dt*u2 (in that
    order), scale multiplies every sum, zero resets them."""
    import pawsim_b200 as lib
    from conftest import make_setup
    _, cfg, f = make_setup(tmp_path, "gyre", N=32, solver=0, dt=900.0)
    m = lib.Model(cfg, f)
    m.prelim()
    m.step(1)
    u1 = m.get("u", 1)
    m.accumulate_averages(1.0)
    m.step(2)
    u2 = m.get("u", 1)
    m.accumulate_averages(1.0)
    dt = cfg.dt
    want = (0.0 + dt * u1) + dt * u2
    assert value_equal(m.get("U_avg", 1), want)
    m.scale_averages(0.5)
    assert value_equal(m.get("U_avg", 1), want * 0.5)
    p = m.get("P_avg", 0)
    assert np.isfinite(p).all()
    m.zero_averages()
    assert not m.get("HUV_avg", 0).any()
    assert not m.get("W_avg", cfg.Nlay).any()
    m.close()
