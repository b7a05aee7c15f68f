"""Pins the CPU oracle to the reference.

1. Against the committed fixtures (tests/golden/, made by make_golden.py from the reference's
   serial build): init_* tendencies, U/V/H/P after each of 3 steps, and the iteration counts
   and norms of every pressure solve -- bit for bit.
2. Against the reference binary itself when oracle/_ref has been built here: a 32x32 gyre run
   for 6 steps, compared file by file.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import make_setup
from golden_util import CASES, load_case


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_golden(tmp_path, oracle_mod, name):
    cfg, f, z = load_case(name, tmp_path)
    o = oracle_mod.Oracle(cfg, f)
    st = o.prelim()
    stats = z["stats"]
    assert st.iters == int(stats[0, 0])
    for k in range(cfg.Nlay):
        for tag, fld in (("dudt", "dt_u"), ("dvdt", "dt_v"), ("dhdt", "dt_h")):
            assert np.array_equal(o.get(fld, k), z[f"init_{tag}{k}"]), (tag, k)
    for n in range(1, 4):
        o.integrator_step(n)
        st = o.pressure(True)
        assert st.iters == int(stats[n, 0]), n
        got = np.array([st.residual_max, st.residual_rms, st.div_max, st.div_rms])
        # the reference prints %0.6e; compare at that precision
        np.testing.assert_allclose(got, stats[n, 1:], rtol=6e-7, atol=0)
        s = o.state()
        for k in range(cfg.Nlay):
            for v, fn in (("u", "U"), ("v", "V"), ("h", "H")):
                assert np.array_equal(s[v][k], z[f"{fn}{k}_{n}"]), (n, v, k)
        assert np.array_equal(o.get("pi"), z[f"P_{n}"]), n


def test_oracle_matches_reference_binary(tmp_path, oracle_mod):
    exe = oracle_mod.reference_exe()
    if exe is None:
        pytest.skip("reference binary not built (no reference sources here)")
    from pawsim_b200 import inputs
    p, cfg, f = make_setup(tmp_path, "gyre", N=32, dt=900.0, solver=0, Nt=6,
                           savefrequency=900.0)
    out = tmp_path / "out"
    out.mkdir()
    subprocess.run([exe, p, str(out)], check=True, capture_output=True)
    o = oracle_mod.Oracle(cfg, f)
    o.prelim()
    for n in range(1, 7):
        o.integrator_step(n)
        o.pressure(True)
        s = o.state()
        for k in range(cfg.Nlay):
            for v, fn in (("u", "U"), ("v", "V"), ("h", "H")):
                ref = inputs.read_data(os.path.join(out, f"{fn}{k}_n={n}.dat"), (cfg.Ny, cfg.Nx))
                assert np.array_equal(s[v][k], ref), (n, v, k)


def test_planted_error_is_detected(tmp_path, oracle_mod):
    """A 1e-9 m change of one thickness must show up in the compared state (the comparison
    is not vacuous)."""
    cfg, f, z = load_case("gyre_sor", tmp_path)
    f["h"][0, 5, 5] += 1e-9
    o = oracle_mod.Oracle(cfg, f)
    o.prelim()
    o.integrator_step(1)
    o.pressure(True)
    assert not np.array_equal(o.state()["u"][0], z["U0_1"])


CORNER_CASES = ["channel_corners_sor", "channel_corners_hk83", "channel_corners_free"]


@pytest.mark.parametrize("name", CORNER_CASES)
def test_oracle_serial_corners_match_reference(tmp_path, oracle_mod, name):
    """x-periodic, y-walled channels with pressureTiming off: with the serial build's fill order
    (periodic columns first, then the wall rows) the oracle's corner ghosts keep each work
    array's previous fill and every step is bit-identical to the reference's serial build;
    the MPI build's order (current corners) is not."""
    cfg, f, z = load_case(name, tmp_path)
    assert not cfg.values["useWallEW"] and cfg.values["useWallNS"] and not cfg.values["pressureTiming"]
    for serial in (1, 0):
        o = oracle_mod.Oracle(cfg, f, serial_corners=serial)
        o.prelim()
        same = True
        for n in range(1, 7):
            o.integrator_step(n)
            o.pressure(True)
            s = o.state()
            for k in range(cfg.Nlay):
                for v, fn in (("u", "U"), ("v", "V"), ("h", "H")):
                    eq = np.array_equal(s[v][k], z[f"{fn}{k}_{n}"])
                    if serial:
                        assert eq, (name, n, v, k, np.abs(s[v][k] - z[f"{fn}{k}_{n}"]).max())
                    same = same and eq
        if not serial:
            assert not same, "the fixture does not see the corner ghosts"


def test_oracle_config0_100_steps(tmp_path, oracle_mod):
    """The plain FP64 path's acceptance point: config 0 (128 x 128 x 2 double gyre, SOR with
    SOR_rp 1.8, tol 1e-10, dt 900 s) for 100 steps. Every step's iteration count and pressure
    norms and the state after step 100 equal the reference's serial build."""
    cfg, f, z = load_case("config0_sor_100", tmp_path)
    stats = z["stats"]
    o = oracle_mod.Oracle(cfg, f)
    st = o.prelim()
    assert st.iters == int(stats[0, 0])
    for n in range(1, 101):
        o.integrator_step(n)
        st = o.pressure(True)
        assert st.iters == int(stats[n, 0]), n
        got = np.array([st.residual_max, st.residual_rms, st.div_max, st.div_rms])
        np.testing.assert_allclose(got, stats[n, 1:], rtol=6e-7, atol=0, err_msg=f"step {n}")
    s = o.state()
    for k in range(cfg.Nlay):
        for v, fn in (("u", "U"), ("v", "V"), ("h", "H")):
            assert np.array_equal(s[v][k], z[f"{fn}{k}_100"]), (v, k)
    assert np.array_equal(o.get("pi"), z["P_100"])
