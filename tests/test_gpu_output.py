"""Asynchronous state output (the saves of model_code/diagnostics.c:874-908 written by a
background thread while the model steps on).

1. The drop-in executable writes the same files, byte for byte, with the background writer
   (default) and with PAWSIM_GPU_SYNC_OUTPUT=1, saving every step of a rigid-lid gyre with a
   tracer and of a free-surface jet.
2. Through the API: a save snapshots the state at the moment of the call, whatever the model
   does afterwards; two slots are in flight at once; a released slot is refilled in order."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, make_setup, value_equal

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(ROOT, "pawsim_b200", "bin", "PAWSIM_B200.exe")


@pytest.mark.parametrize("kind,kw,tracer", [
    ("gyre", dict(N=128, dt=900.0, solver=1), True),
    ("jets", dict(N=96, dt=5.0, solver=0, extra=dict(useRL=0)), False),
])
def test_driver_async_and_sync_output_identical(tmp_path, kind, kw, tracer):
    from pawsim_b200 import inputs
    p, cfg, _ = make_setup(tmp_path, kind, Nt=12, savefrequency=kw["dt"], **kw)
    if tracer:
        inputs.add_tracer(p, scheme=2, relax_days=30.0, K2=100.0)
    outs = {}
    for mode in ("0", "1"):
        out = tmp_path / f"out{mode}"
        out.mkdir()
        env = dict(os.environ, PAWSIM_GPU_SYNC_OUTPUT=mode)
        r = subprocess.run([DRIVER, p, str(out)], capture_output=True, text=True, timeout=600, env=env)
        assert r.returncode == 0, r.stderr
        outs[mode] = out
    names = sorted(os.listdir(outs["0"]))
    assert names == sorted(os.listdir(outs["1"]))
    assert len(names) >= 13 * (3 * cfg.Nlay + cfg.Nlay + 1)
    for n in names:
        assert (outs["0"] / n).read_bytes() == (outs["1"] / n).read_bytes(), n


def test_api_save_snapshots_the_state_at_the_call(tmp_path):
    import pawsim_b200 as lib
    _, cfg, f = make_setup(tmp_path, "gyre", N=96, dt=900.0, solver=1)
    m = lib.Model(cfg, f)
    m.prelim()
    L = cfg.Nlay
    nplanes = 3 * L + (L + 1) + 1
    want = []
    slots = []
    for n in (1, 2):
        m.step(n)
        s = m.state()
        want.append(np.concatenate([np.stack([s["u"][k], s["v"][k], s["h"][k]]) for k in range(L)]
                                   + [np.stack([m.get("wdia", k) for k in range(L + 1)]), m.get("pi")[None]]))
        slots.append(m.save_begin())
    assert sorted(slots) == [0, 1]
    m.step(3)                       # the model moves on while both copies are in flight
    for s_, w in zip(slots, want):
        got = m.save_wait(s_)
        assert got.shape == (nplanes, cfg.Ny, cfg.Nx)
        assert value_equal(got, w)
    m.save_release(slots[0])
    slot = m.save_begin()           # the released slot is the next one filled
    assert slot == slots[0]
    s = m.state()
    got = m.save_wait(slot)
    assert value_equal(got[0], s["u"][0]) and value_equal(got[2], s["h"][0])
    m.save_release(slot)
    m.save_release(slots[1])
    m.close()
