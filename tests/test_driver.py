"""The drop-in host driver (PAWSIM_B200.exe) on the CPU: command line and parameter-file
validation, which run before any GPU work. Each malformed input must be rejected with exit
status 1 and the reference's message, and the reference binary (when built here) must agree.
"""
import os
import subprocess

import pytest

from conftest import ROOT, make_setup

DRIVER = os.path.join(ROOT, "pawsim_b200", "bin", "PAWSIM_B200.exe")
REF = os.path.join(ROOT, "oracle", "_ref", "PAWSIM.exe")

pytestmark = pytest.mark.skipif(not os.path.exists(DRIVER), reason="driver not built")


def _run(exe, *args):
    return subprocess.run([exe, *args], capture_output=True, text=True, timeout=120)


def test_usage():
    r = _run(DRIVER)
    assert r.returncode == 1 and "Usage:" in r.stderr


def _edit(path, drop=(), add=None):
    lines = [l for l in open(path).read().splitlines() if l.split() and l.split()[0] not in drop]
    for k, v in (add or {}).items():
        lines = [l for l in lines if l.split()[0] != k] + [f"{k} {v}"]
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


CASES = [
    (dict(drop=("Ny",)), "Nlay, Nx and Ny must all be specified and positive"),
    (dict(add={"Ly": "-1"}), "Ly must be specified and positive"),
    (dict(add={"momentumScheme": "7"}), "Unknown or unsupported numerical scheme identifier"),
    (dict(add={"SOR_rp": "2.5"}), "Invalid pressure solver parameters"),
    (dict(add={"pressureSolver": "3"}), "Unknown pressureSolver identifier"),
    (dict(add={"A2": "-5"}), "Invalid wind forcing parameters"),
    (dict(add={"mpiNx": "2"}), "mpiNx and mpiNy must both be specified or both omitted"),
    (dict(add={"useTrad": "1"}), "AWSIM useTrad time stepping is not ported in PAWSIM"),
    (dict(add={"timeSteppingScheme": "2"}), "PAWSIM only supports AB1, AB2 and AB3 time stepping so far"),
    (dict(add={"tmax": "99999"}), "Must specify exactly two of {Nt, tmax, dt}"),
]


@pytest.mark.parametrize("edit,msg", CASES, ids=[c[1][:24] for c in CASES])
def test_rejects_like_the_reference(tmp_path, edit, msg):
    p, _, _ = make_setup(tmp_path, "gyre", N=16, dt=900.0, Nt=2)
    _edit(p, **edit)
    out = tmp_path / "out"
    out.mkdir()
    r = _run(DRIVER, p, str(out))
    assert r.returncode == 1
    assert msg in r.stderr, r.stderr
    assert not os.listdir(out)
    if os.path.exists(REF):
        rr = _run(REF, p, str(out))
        assert rr.returncode == 1 and msg in rr.stderr, rr.stderr
