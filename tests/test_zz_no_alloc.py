"""The non-allocating right-hand-side entry point against the model's own pressure path.

Callers that cannot allocate device memory (code running under an allocator it does not own,
or hosts that forbid device allocation after start-up) build the rigid-lid right-hand side
with pawsim_pressure_rhs_noalloc from device arrays they already hold. This test feeds it the
thickness-corrected state of two consecutive steps and compares each result with the pi_rhs
that pawsim_gpu_pressure_correct builds for the same state (same tolerance as the other
floating-point parity tests; both sum in the reference's serial order at this size, so the
values are expected to agree exactly). The file sorts last so that a run stopping at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from conftest import make_setup

pytestmark = pytest.mark.gpu


def _entry(lib):
    fn = lib.pawsim_pressure_rhs_noalloc
    P = ctypes.c_void_p
    fn.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                   ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                   ctypes.c_int, ctypes.c_int, P, P]
    fn.restype = ctypes.c_int
    return fn


def test_noalloc_rhs_matches_pressure_correct(tmp_path):
    import torch

    import pawsim_b200

    lib = pawsim_b200.load_library()
    fn = _entry(lib)
    _, cfg, f = make_setup(tmp_path, "gyre", N=48, Ny=40, solver=0, dt=900.0)
    m = pawsim_b200.Model(cfg, f)
    m.prelim()
    Hc = m.get("Hc")
    L, Nx, Ny = cfg.Nlay, cfg.Nx, cfg.Ny
    dev = torch.device("cuda", 0)
    for n in (1, 2):
        m.integrator_step(n)
        s = m.state()
        # the column correction pawsim_gpu_pressure_correct applies before its RHS
        h = s["h"].copy()
        tot = np.zeros_like(Hc)
        for k in range(L):
            tot = tot + h[k]
        fac = 1 - (tot - Hc) / tot
        for k in range(L):
            h[k] = h[k] * fac
        u = torch.from_numpy(np.ascontiguousarray(s["u"])).to(dev)
        v = torch.from_numpy(np.ascontiguousarray(s["v"])).to(dev)
        hh = torch.from_numpy(np.ascontiguousarray(h)).to(dev)
        rhs = torch.full((Ny, Nx), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        rc = fn(u.data_ptr(), v.data_ptr(), hh.data_ptr(), Nx, Ny, L, Nx, m.cfg.dx, m.cfg.dy,
                cfg.dt, int(cfg.useWallEW), int(cfg.useWallNS), cfg.thicknessScheme, -1,
                rhs.data_ptr(), None)
        assert rc == 0, lib.pawsim_gpu_last_error()
        torch.cuda.synchronize()
        got = rhs.cpu().numpy()
        m.pressure_correct(True)
        want = m.get("pi_rhs")
        scale = np.abs(want).max()
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12 * scale)


def test_noalloc_rejects_oversized_grid():
    import pawsim_b200

    lib = pawsim_b200.load_library()
    fn = _entry(lib)
    rc = fn(None, None, None, 64, 40000, 2, 64, 1.0, 1.0, 1.0, 1, 1, 0, -1, None, None)
    assert rc < 0
    big = ctypes.c_double(0.0)
    p = ctypes.addressof(big)
    rc = fn(p, p, p, 64, 40000, 2, 64, 1.0, 1.0, 1.0, 1, 1, 0, -1, p, None)
    assert rc == -5
