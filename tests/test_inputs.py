"""AWSIM parameter parsing and data I/O (model_code/config.c:42-459, pawsim.c:126-196,
state.c:957-1100, defs.c:140-426)."""
import os

import numpy as np
import pytest

from pawsim_b200 import inputs


def write(tmp, text):
    p = os.path.join(str(tmp), "params.dat")
    with open(p, "w") as fh:
        fh.write(text)
    return p


BASE = "Nlay 2\nNx 8\nNy 4\nLy 4000\ndt 10\nNt 5\n"


def test_defaults_and_grid(tmp_path):
    c = inputs.read_config(write(tmp_path, BASE))
    v = c.values
    assert v["timeSteppingScheme"] == 5 and v["momentumScheme"] == 3 and v["thicknessScheme"] == 0
    assert v["tol"] == 1e-10 and v["SOR_rp"] == 1.0 and v["maxiters"] == 10000
    assert v["omega_MG"] == 2.0 / 3.0 and v["useRL"] and v["oceanSurfDrag"]
    assert v["Lx"] == 8000.0 and v["dx"] == 1000.0 and v["dy"] == 1000.0
    assert v["tmax"] == 50.0 and v["savefrequency"] == 10.0 and v["tmin"] == 0.0


def test_solver_switches(tmp_path):
    assert inputs.read_config(write(tmp_path, BASE + "use_MG 1\n")).values["pressureSolver"] == 1
    assert inputs.read_config(write(tmp_path, BASE + "use_MG 0\n")).values["pressureSolver"] == 0
    c = inputs.read_config(write(tmp_path, BASE + "use_MG 0\npressureSolver 2\n"))
    assert c.values["pressureSolver"] == 2 and c.values["use_MG"]
    c = inputs.read_config(write(tmp_path, BASE + "use_MG 1\npressureSolver 0\n"))
    assert c.values["pressureSolver"] == 0 and not c.values["use_MG"]
    assert inputs.read_config(write(tmp_path, BASE + "SOR_rp_min 1.5\n")).values["SOR_rp"] == 1.5


def test_flags_from_files(tmp_path):
    c = inputs.read_config(write(tmp_path, BASE + "tauxFile t.dat\neTimeFile e.dat\n"))
    v = c.values
    assert v["useWind"] and v["useRelax"] and v["useWDia"] and not v["useFbaro"]
    c = inputs.read_config(write(tmp_path, BASE + "convDiff 1e-3\n"))
    assert c.values["useDiaVisc"] and c.values["useDiaDiff"]


@pytest.mark.parametrize("extra,msg", [
    ("Nt 0\ntmax 0\n", "two of"),
    ("momentumScheme 7\n", "scheme"),
    ("tol 0\n", "pressure solver"),
    ("pressureSolver 3\n", "pressureSolver"),
    ("useRandomForcing 1\n", "random"),
    ("useBuoyancy 1\n", "useBuoyancy"),
    ("A2 -1\n", "Invalid"),
])
def test_rejections(tmp_path, extra, msg):
    with pytest.raises(inputs.ConfigError, match=msg):
        inputs.read_config(write(tmp_path, BASE + extra))


def test_time_from_tmax(tmp_path):
    c = inputs.read_config(write(tmp_path, "Nlay 1\nNx 8\nNy 8\nLy 1\ndt 3\ntmax 10\n"))
    assert c.values["Nt"] == 4


def test_layer_order_round_trip(tmp_path):
    """3-D AWSIM files are layer-fastest, then x, then y."""
    L, Nx, Ny = 3, 5, 4
    h = np.arange(L * Nx * Ny, dtype=float).reshape(L, Ny, Nx)
    inputs.write_data(os.path.join(str(tmp_path), "h.dat"), np.moveaxis(h, 0, 2))
    raw = np.fromfile(os.path.join(str(tmp_path), "h.dat"), dtype="<f8")
    assert raw[0] == h[0, 0, 0] and raw[1] == h[1, 0, 0] and raw[L] == h[0, 0, 1]
    p = write(tmp_path, f"Nlay {L}\nNx {Nx}\nNy {Ny}\nLy 1\ndt 1\nNt 1\nhInitFile h.dat\n")
    f = inputs.load_fields(inputs.read_config(p))
    assert np.array_equal(f["h"], h)
    assert f["eRelax"][2, 0, 0] == 1000.0 * 2 / 3 and f["uTime"][0, 0, 0] == -1


def test_short_file_is_an_error(tmp_path):
    np.zeros(3).tofile(os.path.join(str(tmp_path), "hb.dat"))
    p = write(tmp_path, BASE + "hbFile hb.dat\n")
    with pytest.raises(inputs.ConfigError, match="Could only read"):
        inputs.load_fields(inputs.read_config(p))
