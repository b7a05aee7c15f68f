"""The plain FP64 GPU path at the acceptance points, against the reference's serial build.

1. Config 0 (128 x 128 x 2 wind-driven double gyre, red-black SOR with SOR_rp 1.8, tol 1e-10,
   dt 900 s, the stable step of that grid) for 100 steps: the criterion is u, v, h within relative
   L2 1e-11 of the reference after 100 steps; the GPU meets it bit for bit. Every step's
   iteration count and its four pressure norms (residual max/RMS, divergence max/RMS, printed by
   the reference with %0.6e) agree as well.
2. x-periodic, y-walled channels with pressureTiming off, where the serial build's corner
   ghosts keep each work array's previous fill: the GPU reproduces them (mpi_corners 0, the
   default) and matches every step bit for bit, including a free surface and a KT00 tracer;
   with mpi_corners 1 (current corners, the MPI build's exchange order) it does not.
"""
import numpy as np
import pytest

from conftest import rel_l2, value_equal
from golden_util import load_case

pytestmark = pytest.mark.gpu


def test_config0_100_steps_match_reference(tmp_path):
    import pawsim_b200
    cfg, f, z = load_case("config0_sor_100", tmp_path)
    stats = z["stats"]
    m = pawsim_b200.Model(cfg, f)
    st = m.prelim()
    assert st["iters"] == int(stats[0, 0])
    for n in range(1, 101):
        st = m.step(n)
        assert st["iters"] == int(stats[n, 0]), (n, st["iters"], stats[n, 0])
        got = np.array([st["residual_max"], st["residual_rms"], st["div_max"], st["div_rms"]])
        np.testing.assert_allclose(got, stats[n, 1:], rtol=6e-7, atol=0, err_msg=f"step {n}")
    s = m.state()
    for k in range(cfg.Nlay):
        for v, fn in (("u", "U"), ("v", "V"), ("h", "H")):
            ref = z[f"{fn}{k}_100"]
            assert rel_l2(s[v][k], ref) <= 1e-11, (v, k, rel_l2(s[v][k], ref))
            assert value_equal(s[v][k], ref), (v, k, np.abs(s[v][k] - ref).max())
    assert value_equal(m.get("pi"), z["P_100"])
    m.close()


@pytest.mark.parametrize("name", ["channel_corners_sor", "channel_corners_hk83", "channel_corners_free",
                                  "channel_corners_tracer"])
def test_channel_serial_corners_match_reference(tmp_path, name):
    """The serial build's corner ghosts on x-periodic, y-walled grids (pressureTiming off): with
    them (mpi_corners 0, the default) every step is bit-identical to the reference; the current
    corners of the MPI build's exchange order (mpi_corners 1) differ."""
    import pawsim_b200
    cfg, f, z = load_case(name, tmp_path)
    names = (("u", "U"), ("v", "V"), ("h", "H")) + ((("b", "B"),) if cfg.values["useTracer"] else ())
    for mpi in (0, 1):
        m = pawsim_b200.Model(cfg, f, mpi_corners=mpi)
        m.prelim()
        same = True
        for n in range(1, 7):
            m.step(n)
            s = m.state()
            for k in range(cfg.Nlay):
                for v, fn in names:
                    eq = value_equal(s[v][k], z[f"{fn}{k}_{n}"])
                    if not mpi:
                        assert eq, (name, n, v, k, rel_l2(s[v][k], z[f"{fn}{k}_{n}"]))
                    same = same and eq
            if cfg.values["useRL"] and not mpi:
                assert value_equal(m.get("pi"), z[f"P_{n}"]), (name, n)
        if mpi:
            assert not same, "the current-corner option must differ from the serial build here"
        m.close()
