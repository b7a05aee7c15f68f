"""The optional physics of the tendency against the oracle, bit for bit, through the C ABI:
UP3 and KT00 thickness (3-cell tile halo, also in the pressure right-hand side),
Smagorinsky A2 and A4, quadratic bottom and surface drag (with wind feedback), and the
hsml / hbbl layer fractions of wind, linear and quadratic drag. Each case is checked as a tendency
after the preliminary correction and over 5 SOR steps (state, pi and iteration count); the
oracle itself is bit-identical to the reference binary on these options
(tests/test_oracle_physics.py)."""
import numpy as np
import pytest

from conftest import make_setup, value_equal

pytestmark = pytest.mark.gpu

CASES = {
    "up3": ("gyre", dict(N=40, Ny=24, dt=600.0, solver=0, extra=dict(thicknessScheme=2, momentumScheme=0))),
    "kt00": ("gyre", dict(N=40, Ny=24, dt=600.0, solver=0, extra=dict(thicknessScheme=3, KT00_sigma=1.4))),
    "kt00_jets": ("jets", dict(N=32, dt=100.0, solver=0, extra=dict(thicknessScheme=3))),
    "up3_channel": ("channel", dict(Nx=64, Ny=32, dt=150.0, solver=0, extra=dict(thicknessScheme=2, pressureTiming=1))),
    "smag_a2": ("gyre", dict(N=40, Ny=24, dt=600.0, solver=0, extra=dict(A2smag=2.0))),
    "smag_a4": ("channel", dict(Nx=64, Ny=32, dt=150.0, solver=0, extra=dict(A4smag=1.0, A4=1e9, pressureTiming=1))),
    "smag_both_hk83": ("gyre", dict(N=40, Ny=24, dt=600.0, solver=0, A4=1e9,
                                    extra=dict(A2smag=1.5, A4smag=0.5, momentumScheme=1, thicknessScheme=1))),
    "quad": ("gyre", dict(N=40, Ny=24, dt=600.0, solver=0, extra=dict(quadDragCoeff=2e-3))),
    "quad_surf": ("gyre", dict(N=40, Ny=24, dt=600.0, solver=0,
                               extra=dict(quadDragSurf=1e-3, windFeedback=1, oceanSurfDrag=0))),
    "fractions": ("gyre", dict(N=40, Ny=24, dt=600.0, solver=0,
                               extra=dict(hsml=1500.0, hmin_surf=5.0, hbbl=500.0, hmin_bot=10.0, linDragSurf=1e-4))),
    "fractions_kt00_quad": ("gyre", dict(N=40, Ny=24, dt=600.0, solver=0,
                                         extra=dict(hsml=800.0, thicknessScheme=3, quadDragCoeff=1e-3))),
    # quadratic drag whose boundary layer spans several layers (forcing.c:95-143, 181-223)
    "quad_hbbl": ("gyre", dict(N=40, Ny=24, dt=600.0, solver=0,
                               extra=dict(quadDragCoeff=2e-3, hbbl=3500.0, hmin_bot=10.0))),
    "quad_surf_hsml": ("gyre", dict(N=40, Ny=24, dt=600.0, solver=0,
                                    extra=dict(quadDragSurf=1e-3, windFeedback=1, oceanSurfDrag=1, hsml=1200.0,
                                               hmin_surf=5.0))),
    "quad_both_fractions_jets": ("jets", dict(N=32, dt=100.0, solver=0,
                                              extra=dict(quadDragCoeff=2e-3, hbbl=3800.0, quadDragSurf=1e-3,
                                                         hsml=700.0, thicknessScheme=1))),
}


@pytest.fixture(scope="module")
def lib():
    import pawsim_b200
    return pawsim_b200


@pytest.mark.parametrize("name", sorted(CASES))
def test_physics_bitwise(tmp_path, oracle_mod, lib, name):
    kind, kw = CASES[name]
    _, cfg, f = make_setup(tmp_path, kind, **kw)
    o = oracle_mod.Oracle(cfg, f)
    m = lib.Model(cfg, f)
    ref = o.tendency()
    got = m.tendency_eval()
    for var in ("u", "v", "h"):
        for k in range(cfg.Nlay):
            a, b = got[var][k], ref[var][k]
            assert value_equal(a, b), ("tendency", var, k, np.abs(a - b).max(), np.argwhere(a != b)[:4])
    so, sg = o.prelim(), m.prelim()
    assert so.iters == sg["iters"]
    for n in range(1, 6):
        o.integrator_step(n)
        so = o.pressure(True)
        sg = m.step(n)
        assert so.iters == sg["iters"], n
        s_o, s_g = o.state(), m.state()
        for var in ("u", "v", "h"):
            assert value_equal(s_g[var], s_o[var]), (n, var, np.abs(s_g[var] - s_o[var]).max())
        assert value_equal(m.get("pi"), o.get("pi")), n

