"""The non-allocating right-hand-side entry point against the model's own pressure path.

Callers that cannot allocate device memory (code running under an allocator it does not own,
or hosts that forbid device allocation after start-up) build the rigid-lid right-hand side
with pawsim_pressure_rhs_noalloc from device arrays they already hold. These tests feed it the
thickness-corrected state that pawsim_gpu_pressure_correct works on and compare the result
with that call's pi_rhs. Both run the same kernels and the same summation order for the
mean (the reference's serial order on small grids, the fixed pairwise tree on large ones, or
the one forced by serial_sum), so the values must agree bit for bit. The tree order keeps its
per-row partial sums in the entry point's static scratch array, so a grid above 65536 cells
and the largest accepted grid (32760 rows) exercise that array; 32761 rows must be refused.
The file sorts last so that a run stopping at the first failure has already run every other
test.
"""
import ctypes

import numpy as np
import pytest

from conftest import make_setup

pytestmark = pytest.mark.gpu

EUNSUPPORTED = -5


def _entry(lib):
    fn = lib.pawsim_pressure_rhs_noalloc
    P = ctypes.c_void_p
    fn.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                   ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                   ctypes.c_int, ctypes.c_int, P, P]
    fn.restype = ctypes.c_int
    return fn


def _corrected_thickness(h, Hc):
    """The column correction pawsim_gpu_pressure_correct applies before its RHS
    (model_code/pressure.c:525-561), in the same operation order."""
    h = h.copy()
    tot = np.zeros_like(Hc)
    for k in range(h.shape[0]):
        tot = tot + h[k]
    fac = 1 - (tot - Hc) / tot
    for k in range(h.shape[0]):
        h[k] = h[k] * fac
    return h


def _noalloc_rhs(fn, lib, m, cfg, s, serial_sum):
    import torch

    dev = torch.device("cuda", 0)
    L, Nx, Ny = cfg.Nlay, cfg.Nx, cfg.Ny
    h = _corrected_thickness(s["h"], m.get("Hc"))
    u = torch.from_numpy(np.ascontiguousarray(s["u"])).to(dev)
    v = torch.from_numpy(np.ascontiguousarray(s["v"])).to(dev)
    hh = torch.from_numpy(np.ascontiguousarray(h)).to(dev)
    # the output starts as NaN so that a cell the call did not write cannot pass
    rhs = torch.full((Ny, Nx), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    rc = fn(u.data_ptr(), v.data_ptr(), hh.data_ptr(), Nx, Ny, L, Nx, m.cfg.dx, m.cfg.dy,
            cfg.dt, int(cfg.useWallEW), int(cfg.useWallNS), cfg.thicknessScheme, serial_sum,
            rhs.data_ptr(), None)
    assert rc == 0, lib.pawsim_gpu_last_error()
    torch.cuda.synchronize()
    return rhs.cpu().numpy()


def test_noalloc_rhs_matches_pressure_correct(tmp_path):
    """Two consecutive steps of a 48 x 40 gyre (serial order of the mean)."""
    import pawsim_b200

    lib = pawsim_b200.load_library()
    fn = _entry(lib)
    _, cfg, f = make_setup(tmp_path, "gyre", N=48, Ny=40, solver=0, dt=900.0)
    m = pawsim_b200.Model(cfg, f)
    m.prelim()
    for n in (1, 2):
        m.integrator_step(n)
        got = _noalloc_rhs(fn, lib, m, cfg, m.state(), -1)
        m.pressure_correct(True)
        want = m.get("pi_rhs")
        assert np.array_equal(got, want), (n, np.abs(got - want).max())
    m.close()


@pytest.mark.parametrize("serial_sum", [0, 1, -1])
def test_noalloc_rhs_tree_and_serial_orders(tmp_path, serial_sum):
    """A 288 x 256 gyre (73728 cells, above the serial-order threshold): the tree order's
    partials live in the static scratch; serial_sum 1 forces the serial order on both sides."""
    import pawsim_b200

    lib = pawsim_b200.load_library()
    fn = _entry(lib)
    _, cfg, f = make_setup(tmp_path, "gyre", N=288, Ny=256, solver=1, dt=300.0)
    m = pawsim_b200.Model(cfg, f, serial_sums=1 if serial_sum == 1 else -1)
    m.prelim()
    for n in (1, 2):
        m.integrator_step(n)
        got = _noalloc_rhs(fn, lib, m, cfg, m.state(), serial_sum)
        m.pressure_correct(True)
        want = m.get("pi_rhs")
        assert np.array_equal(got, want), (n, serial_sum, np.abs(got - want).max())
    m.close()


def test_noalloc_rhs_largest_grid(tmp_path):
    """8 x 32760 cells, the most rows the static scratch holds, with random velocities: the
    entry point succeeds twice in a row and matches the model's RHS."""
    import pawsim_b200

    lib = pawsim_b200.load_library()
    fn = _entry(lib)
    _, cfg, f = make_setup(tmp_path, "gyre", N=8, Ny=32760, solver=0, dt=60.0,
                           extra=dict(maxiters=1))
    m = pawsim_b200.Model(cfg, f)
    rng = np.random.default_rng(3)
    for call in range(2):
        for k in range(cfg.Nlay):
            m.set("u", k, rng.standard_normal((cfg.Ny, cfg.Nx)) * 0.1)
            m.set("v", k, rng.standard_normal((cfg.Ny, cfg.Nx)) * 0.1)
        got = _noalloc_rhs(fn, lib, m, cfg, m.state(), -1)
        m.pressure_correct(False)
        want = m.get("pi_rhs")
        assert np.abs(want).max() > 0
        assert np.array_equal(got, want), (call, np.abs(got - want).max())
    m.close()


def test_noalloc_rejects_oversized_grid():
    import pawsim_b200

    lib = pawsim_b200.load_library()
    fn = _entry(lib)
    rc = fn(None, None, None, 64, 40000, 2, 64, 1.0, 1.0, 1.0, 1, 1, 0, -1, None, None)
    assert rc < 0
    big = ctypes.c_double(0.0)
    p = ctypes.addressof(big)
    # refused before any launch, so the host address is never handed to a kernel
    for ny in (32761, 40000):
        rc = fn(p, p, p, 8, ny, 2, 8, 1.0, 1.0, 1.0, 1, 1, 0, -1, p, None)
        assert rc == EUNSUPPORTED, (ny, rc)
