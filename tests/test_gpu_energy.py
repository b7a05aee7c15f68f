"""Energy and enstrophy diagnostics on the GPU (savefreqEZ, model_code/diagnostics.c:478-700).

1. The drop-in executable on the committed ``*_ez`` fixtures writes EZdiags.dat with the same
   text as the reference binary, byte for byte: rigid lid with two lines per step (walls, AL81),
   a doubly periodic free surface (interface heights from the thickness of the start of the
   step) and a free-surface HK83 gyre whose online averages reload the state every step.
2. Through the Python API on larger grids, against the oracle stepping the same inputs: bit
   for bit with the serial summation order, and to a relative 1e-12 with the tree sums."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, make_setup
from golden_util import load_case
from test_oracle_energy import EZ_CASES

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(ROOT, "pawsim_b200", "bin", "PAWSIM_B200.exe")


@pytest.mark.parametrize("name", EZ_CASES)
def test_driver_ez_file_matches_reference(tmp_path, name):
    cfg, _, z = load_case(name, tmp_path)
    out = tmp_path / "out"
    out.mkdir()
    param = os.path.join(str(tmp_path), name, "params.dat")
    r = subprocess.run([DRIVER, param, str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    got = (out / "EZdiags.dat").read_text()
    want = str(z["ez_text"])
    assert got.splitlines() == want.splitlines()
    assert got == want


CASES = [
    ("gyre", dict(N=128, Ny=96, dt=900.0, solver=0, tol=1e-10)),
    ("gyre", dict(N=96, dt=40.0, solver=0, extra=dict(useRL=0, thicknessScheme=1))),
    ("jets", dict(N=128, dt=5.0, solver=0, extra=dict(useRL=0))),
    ("full", dict(N=64, dt=50.0, solver=0, Ly=1280e3, bathy_len=80e3, sponge=160e3)),
]


@pytest.mark.parametrize("serial", [1, 0])
@pytest.mark.parametrize("kind,kw", CASES)
def test_api_energy_matches_oracle(tmp_path, oracle_mod, kind, kw, serial):
    import pawsim_b200 as lib
    _, cfg, f = make_setup(tmp_path, kind, Nt=3, **kw)
    rl = bool(cfg.values["useRL"])
    m = lib.Model(cfg, f, serial_sums=serial)
    o = oracle_mod.Oracle(cfg, f)
    m.prelim()
    o.prelim()
    for n in range(1, 4):
        m.step(n)
        o.integrator_step(n)
        if rl:
            o.pressure(True)
        got = m.energy(eta_from_step_start=not rl)
        want = o.energy(False)
        if serial:
            assert got[0] == want[0] and got[1] == want[1], (n, got, want)
            assert got[2] == want[2], (n, got, want)
        else:
            np.testing.assert_allclose(got[:2], want[:2], rtol=1e-12, atol=0)
            np.testing.assert_allclose(got[2], want[2], rtol=1e-12, atol=0)
    # the current thickness (what the averages reload) gives the oracle's reloaded sums
    got = m.energy(eta_from_step_start=False)
    want = o.energy(True)
    if serial:
        assert got[0] == want[0] and got[1] == want[1] and got[2] == want[2]
    m.close()


def test_energy_needs_a_step_for_the_start_thickness(tmp_path):
    import pawsim_b200 as lib
    _, cfg, f = make_setup(tmp_path, "jets", N=32, dt=10.0, solver=0, extra=dict(useRL=0))
    m = lib.Model(cfg, f)
    m.prelim()
    with pytest.raises(lib.PawsimError):
        m.energy(eta_from_step_start=True)
    ke, pe, z = m.energy()
    assert np.isfinite([ke, pe] + z).all() and ke > 0
    m.step(1)
    m.energy(eta_from_step_start=True)
    m.close()
