"""Failure reporting through the C ABI, with the failures made on the host side: a NaN planted
in an uploaded thickness, and a pressure solve limited to one iteration (maxiters 1).

The reference prints "WARNING: PAWSIM pressure solve reached maxiters" and runs on, to NaN when
the state blows up (model_code/pawsim.c:488-491). That stays the default here; the options
check_nonfinite (PAWSIM_GPU_ENONFINITE) and fail_on_maxiters (PAWSIM_GPU_ENOTCONVERGED) turn the
two cases into return codes. No GPU fault is involved: the fused kernel only raises a flag that
the host reads.
"""
import numpy as np
import pytest

from conftest import make_setup

pytestmark = pytest.mark.gpu

ENOTCONVERGED, ENONFINITE = -3, -4


def _nan_fields(f):
    f = dict(f)
    h = f["h"].copy()
    h[0, 5, 7] = np.nan
    f["h"] = h
    return f


@pytest.mark.parametrize("solver", [0, 1], ids=["sor", "mg"])
def test_nonfinite_state_reported(tmp_path, solver):
    import pawsim_b200
    _, cfg, f = make_setup(tmp_path, "gyre", N=32, solver=solver, dt=900.0)
    bad = _nan_fields(f)
    # off (the reference's behaviour): the steps complete and the NaN spreads
    m = pawsim_b200.Model(cfg, bad)
    m.prelim()
    for n in (1, 2):
        m.step(n)
    assert np.isnan(m.state()["h"]).any()
    m.close()
    # every step: the first step reports it, with the step completed
    m = pawsim_b200.Model(cfg, bad, check_nonfinite=1)
    m.prelim()
    with pytest.raises(pawsim_b200.PawsimError) as e:
        m.step(1)
    assert e.value.code == ENONFINITE
    assert "non-finite" in str(e.value)
    m.close()
    # every third step: steps 1 and 2 return normally, step 3 reports it
    m = pawsim_b200.Model(cfg, bad, check_nonfinite=3)
    m.prelim()
    m.step(1)
    m.step(2)
    with pytest.raises(pawsim_b200.PawsimError) as e:
        m.step(3)
    assert e.value.code == ENONFINITE
    m.close()
    # a finite state never raises it
    m = pawsim_b200.Model(cfg, f, check_nonfinite=1)
    m.prelim()
    for n in range(1, 5):
        m.step(n)
        m.integrator_step(n + 4)
    m.close()


@pytest.mark.parametrize("solver", [0, 1, 2], ids=["sor", "mg", "dmg"])
def test_maxiters_reported(tmp_path, solver):
    import pawsim_b200
    _, cfg, f = make_setup(tmp_path, "gyre", N=32, solver=solver, dt=900.0, tol=1e-13,
                           extra=dict(maxiters=1))
    # off: the solve stops after one iteration and the step succeeds (the reference warns)
    m = pawsim_b200.Model(cfg, f)
    m.prelim()
    st = m.step(1)
    assert st["iters"] == 1
    m.close()
    m = pawsim_b200.Model(cfg, f, fail_on_maxiters=1)
    m.prelim()
    with pytest.raises(pawsim_b200.PawsimError) as e:
        m.step(1)
    assert e.value.code == ENOTCONVERGED
    assert "maxiters" in str(e.value)
    # the step completed: the model advanced by one dt
    assert m.t == pytest.approx(cfg.values["tmin"] + cfg.values["dt"])
    m.close()
