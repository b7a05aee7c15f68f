"""The drop-in host driver end to end on the GPU: PAWSIM_B200.exe <input_file> <output_dir>
on the committed fixtures' inputs must write the reference's output files (U/V/H/W for
every layer and interface, P, n = 0..3 on the dt save schedule) and print its pressure
lines. SOR cases are bit-identical to the reference's files and iteration counts; multigrid
cases agree within the solver tolerance."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, rel_l2, value_equal
from golden_util import CASES, load_case

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(ROOT, "pawsim_b200", "bin", "PAWSIM_B200.exe")
LINE = re.compile(r"PAWSIM pressure solve: phase=(\w+) n=(\d+) solver=(\w+) iters=(\d+)")


@pytest.mark.parametrize("name", CASES)
def test_driver_writes_reference_outputs(tmp_path, name):
    from pawsim_b200 import inputs
    cfg, _, z = load_case(name, tmp_path)
    out = tmp_path / "out"
    out.mkdir()
    param = os.path.join(str(tmp_path), name, "params.dat")
    r = subprocess.run([DRIVER, param, str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert f"PAWSIM parsed {cfg.Nx} x {cfg.Ny} x {cfg.Nlay} AWSIM input" in r.stdout
    solves = LINE.findall(r.stdout)
    assert [s[0] for s in solves] == ["prelim", "step", "step", "step"]
    assert "PAWSIM pressure summary:" in r.stdout
    sor = cfg.values["pressureSolver"] == 0
    stats = z["stats"]
    shape = (cfg.Ny, cfg.Nx)
    for n in range(0, 4):
        for k in range(cfg.Nlay + 1):
            assert os.path.exists(out / f"W{k}_n={n}.dat")
        if n == 0:
            continue
        if sor:
            assert int(solves[n][3]) == int(stats[n, 0]), n
        for k in range(cfg.Nlay):
            for fn in ("U", "V", "H"):
                got = inputs.read_data(str(out / f"{fn}{k}_n={n}.dat"), shape)
                ref = z[f"{fn}{k}_{n}"]
                if sor:
                    assert value_equal(got, ref), (n, fn, k)
                else:
                    assert rel_l2(got, ref) < 1e-6, (n, fn, k, rel_l2(got, ref))
        got = inputs.read_data(str(out / f"P_n={n}.dat"), shape)
        if sor:
            assert value_equal(got, z[f"P_{n}"]), n
        else:
            # the gathered multigrid leaves pi's constant free: compare modulo the mean
            ref = z[f"P_{n}"]
            assert rel_l2(got - got.mean(), ref - ref.mean()) < 1e-5, n
    assert not os.path.exists(out / "U0_n=4.dat")


def test_driver_restart_continues_the_run(tmp_path):
    """restart 1 / startIdx 2 picks up U/V/H of save 2 from the output directory and
    continues; with SOR the continued states equal those of the uninterrupted run."""
    from pawsim_b200 import inputs
    cfg, _, z = load_case("gyre_sor", tmp_path)
    param = os.path.join(str(tmp_path), "gyre_sor", "params.dat")
    full = tmp_path / "full"
    full.mkdir()
    assert subprocess.run([DRIVER, param, str(full)], capture_output=True, timeout=600).returncode == 0
    rs = tmp_path / "rs"
    rs.mkdir()
    for f in os.listdir(full):
        if f.endswith("_n=2.dat"):
            os.link(full / f, rs / f)
    text = open(param).read() + "\nrestart 1\nstartIdx 2\n"
    p2 = os.path.join(str(tmp_path), "gyre_sor", "params_rs.dat")
    with open(p2, "w") as fh:
        fh.write(text.replace("Nt ", "Ntold "))   # keep dt, set the end by tmax
    dt = cfg.dt
    with open(p2, "a") as fh:
        fh.write(f"tmax {4 * dt!r}\n")
    r = subprocess.run([DRIVER, p2, str(rs)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert os.path.exists(rs / "U0_n=4.dat")
