"""GPU parity against the CPU oracle, through the C ABI.

Tendencies and SOR steps are compared bit for bit (IEEE equality, so +0 and -0 compare
equal): the GPU kernels keep the reference's expression order and are built without
multiply-add contraction. Multigrid steps are compared at the solver's tolerance because
the GPU smoother is red-black where the reference's is lexicographic.
"""
import numpy as np
import pytest

from conftest import make_setup, rel_l2, value_equal

pytestmark = pytest.mark.gpu

CASES = [
    ("gyre", dict(N=32, solver=0, tol=1e-10, dt=900.0)),
    ("gyre", dict(N=40, Ny=24, solver=0, A4=1e9, A2=0.0, extra=dict(momentumScheme=0))),
    ("gyre", dict(N=32, solver=0, extra=dict(momentumScheme=1, thicknessScheme=1))),
    ("gyre", dict(N=24, solver=0, extra=dict(momentumScheme=2))),
    ("channel", dict(Nx=64, Ny=32, dt=150.0, solver=0, extra=dict(pressureTiming=1))),
    ("jets", dict(N=32, dt=100.0, solver=0)),
    ("full", dict(N=32, dt=50.0, solver=0, Ly=400e3, bathy_len=20e3, sponge=40e3)),
]


@pytest.fixture(scope="module")
def lib():
    import pawsim_b200
    return pawsim_b200


@pytest.mark.parametrize("kind,kw", CASES, ids=[f"{c[0]}-{i}" for i, c in enumerate(CASES)])
def test_tendency_bitwise(tmp_path, oracle_mod, lib, kind, kw):
    _, cfg, f = make_setup(tmp_path, kind, **kw)
    o = oracle_mod.Oracle(cfg, f)
    m = lib.Model(cfg, f)
    ref = o.tendency()
    got = m.tendency_eval()
    for var in ("u", "v", "h"):
        for k in range(cfg.Nlay):
            a, b = got[var][k], ref[var][k]
            assert value_equal(a, b), (var, k, np.abs(a - b).max(), np.argwhere(a != b)[:5])


@pytest.mark.parametrize("kind,kw", CASES[:1] + CASES[4:7], ids=["gyre", "channel", "jets", "full"])
def test_sor_steps_bitwise(tmp_path, oracle_mod, lib, kind, kw):
    _, cfg, f = make_setup(tmp_path, kind, **kw)
    o = oracle_mod.Oracle(cfg, f)
    m = lib.Model(cfg, f)
    so = o.prelim()
    sg = m.prelim()
    assert so.iters == sg["iters"]
    for n in range(1, 7):
        o.integrator_step(n)
        so = o.pressure(True)
        sg = m.step(n)
        assert so.iters == sg["iters"], n
        s_o, s_g = o.state(), m.state()
        for var in ("u", "v", "h"):
            assert value_equal(s_g[var], s_o[var]), (n, var, np.abs(s_g[var] - s_o[var]).max())
        assert value_equal(m.get("pi"), o.get("pi")), n


def test_mg_steps_tolerance(tmp_path, oracle_mod, lib):
    _, cfg, f = make_setup(tmp_path, "gyre", N=64, solver=1, tol=1e-13, dt=900.0)
    o = oracle_mod.Oracle(cfg, f)
    m = lib.Model(cfg, f)
    o.prelim()
    m.prelim()
    for n in range(1, 11):
        o.integrator_step(n)
        o.pressure(True)
        st = m.step(n)
        assert st["iters"] < 60
    s_o, s_g = o.state(), m.state()
    for var in ("u", "v", "h"):
        assert rel_l2(s_g[var], s_o[var]) < 1e-9, var


@pytest.mark.parametrize("fp32", [0, 1], ids=["fp64", "fp32-defect"])
@pytest.mark.parametrize("kind,kw", [
    ("gyre", dict(N=128, solver=1, tol=1e-13, dt=900.0)),
    ("channel", dict(Nx=128, Ny=64, solver=1, tol=1e-13, dt=150.0)),
    ("jets", dict(N=64, solver=1, tol=1e-13, dt=100.0)),
], ids=["gyre128", "channel128x64", "jets64"])
def test_mg_tiled_levels_tolerance(tmp_path, oracle_mod, lib, fp32, kind, kw):
    """Grids large enough for the tiled multigrid levels (above the one-CTA coarse block),
    in FP64 and in FP32 V-cycles inside FP64 defect correction: 6 steps against the oracle's
    serial multigrid at tol 1e-13."""
    _, cfg, f = make_setup(tmp_path, kind, **kw)
    o = oracle_mod.Oracle(cfg, f)
    m = lib.Model(cfg, f, mg_fp32=fp32)
    o.prelim()
    m.prelim()
    for n in range(1, 7):
        o.integrator_step(n)
        o.pressure(True)
        st = m.step(n)
        assert 1 <= st["iters"] < 80, st
        assert st["stop_measure"] <= 1e-13
    s_o, s_g = o.state(), m.state()
    for var in ("u", "v", "h"):
        assert rel_l2(s_g[var], s_o[var]) < 1e-9, (var, rel_l2(s_g[var], s_o[var]))


@pytest.mark.gpu
@pytest.mark.parametrize("inner", [2, 4])
@pytest.mark.parametrize("kind,kw", [
    ("gyre", dict(N=16, solver=1, tol=1e-13, dt=900.0)),
    ("gyre", dict(N=128, solver=1, tol=1e-13, dt=900.0)),
    ("jets", dict(N=64, solver=1, tol=1e-13, dt=100.0)),
], ids=["gyre16", "gyre128", "jets64"])
def test_mg_fp32_inner_cycles_tolerance(tmp_path, oracle_mod, lib, inner, kind, kw):
    """Several FP32 V-cycles per FP64 defect-correction step (each continuing from the
    correction the previous one left; on the 16 x 16 grid the whole hierarchy is the one-CTA
    coarse block): the solves still stop on the reference's test and the states stay within
    1e-9 of the oracle's serial multigrid at tol 1e-13 over 6 steps."""
    _, cfg, f = make_setup(tmp_path, kind, **kw)
    o = oracle_mod.Oracle(cfg, f)
    m = lib.Model(cfg, f, mg_fp32=1, mg_fp32_inner=inner)
    o.prelim()
    m.prelim()
    for n in range(1, 7):
        o.integrator_step(n)
        o.pressure(True)
        st = m.step(n)
        assert 1 <= st["iters"] < 80, st
        assert st["stop_measure"] <= 1e-13
    s_o, s_g = o.state(), m.state()
    for var in ("u", "v", "h"):
        assert rel_l2(s_g[var], s_o[var]) < 1e-9, (var, rel_l2(s_g[var], s_o[var]))


@pytest.mark.gpu
@pytest.mark.parametrize("solver", [1, 2], ids=["mg", "dmg"])
def test_extrapolated_first_guess_tolerance(tmp_path, oracle_mod, lib, solver):
    """pi_guess = 1 starts each multigrid solve (from the third on) at 2 pi(n-1) - pi(n-2):
    the stopping test is the reference's, so the states stay within 1e-9 of the oracle's
    serial solver at tol 1e-13 over 8 steps."""
    _, cfg, f = make_setup(tmp_path, "gyre", N=64, solver=solver, tol=1e-13, dt=900.0)
    o = oracle_mod.Oracle(cfg, f)
    m = lib.Model(cfg, f, pi_guess=1)
    o.prelim()
    m.prelim()
    for n in range(1, 9):
        o.integrator_step(n)
        o.pressure(True)
        st = m.step(n)
        assert 1 <= st["iters"] < 200, st
    s_o, s_g = o.state(), m.state()
    for var in ("u", "v", "h"):
        assert rel_l2(s_g[var], s_o[var]) < 1e-9, (var, rel_l2(s_g[var], s_o[var]))


@pytest.mark.gpu
@pytest.mark.parametrize("fp32", [0, 1], ids=["fp64", "fp32"])
@pytest.mark.parametrize("kind,kw", [
    ("gyre", dict(N=256, solver=1, tol=1e-12, dt=450.0)),
    ("channel", dict(Nx=256, Ny=128, solver=1, tol=1e-12, dt=150.0)),
    ("jets", dict(N=256, solver=1, tol=1e-12, dt=100.0)),
    ("gyre", dict(N=1024, solver=1, tol=1e-11, dt=120.0)),
], ids=["gyre256", "channel256x128", "jets256", "gyre1024"])
def test_mg_tile_shapes_identical(tmp_path, lib, fp32, kind, kw):
    """Every shape of the fused multigrid level kernels (four tile shapes, the streamed
    strips) and the autotuned choice give bit-identical states and iteration counts: the
    shape changes only the speed. At 1024^2 the strips cover several segments per column."""
    _, cfg, f = make_setup(tmp_path, kind, **kw)
    runs = []
    for tile in (0, 1, 2, 3, 4, 5):
        m = lib.Model(cfg, f, mg_fp32=fp32, mg_tile=tile)
        m.prelim()
        iters = [m.step(n)["iters"] for n in range(1, 5)]
        runs.append((tile, iters, m.state()))
    _, iters0, s0 = runs[1]
    for tile, iters, s in runs:
        assert iters == iters0, (tile, iters, iters0)
        for var in ("u", "v", "h"):
            assert np.array_equal(s[var], s0[var]), (tile, var)


@pytest.mark.gpu
@pytest.mark.parametrize("kind,kw", [
    ("gyre", dict(N=128, solver=2, tol=1e-13, dt=900.0)),
    ("jets", dict(N=64, solver=2, tol=1e-13, dt=100.0)),
    ("channel", dict(Nx=128, Ny=64, solver=2, tol=1e-13, dt=150.0)),
], ids=["gyre128", "jets64", "channel128x64"])
def test_dmg_tolerance(tmp_path, oracle_mod, lib, kind, kw):
    """pressureSolver 2 (distributed multigrid, serial semantics) against the oracle's
    restatement of the reference's: same hierarchy, transfers, coarse SOR tail and stopping
    test; the GPU sweeps red-black instead of in place, so states agree to the tolerance."""
    _, cfg, f = make_setup(tmp_path, kind, **kw)
    o = oracle_mod.Oracle(cfg, f)
    m = lib.Model(cfg, f)
    o.prelim()
    m.prelim()
    for n in range(1, 7):
        o.integrator_step(n)
        so = o.pressure(True)
        st = m.step(n)
        assert st["fallback"] == 0
        assert 1 <= st["iters"] < 200, st
        assert abs(st["iters"] - so.iters) <= max(4, so.iters // 2), (st["iters"], so.iters)
        assert st["stop_measure"] <= 1e-13
    s_o, s_g = o.state(), m.state()
    for var in ("u", "v", "h"):
        assert rel_l2(s_g[var], s_o[var]) < 1e-9, (var, rel_l2(s_g[var], s_o[var]))


@pytest.mark.gpu
def test_dmg_falls_back_to_gathered_mg(tmp_path, oracle_mod, lib):
    """A grid whose first 2:1 coarsening is not clean (odd side) runs the gathered multigrid,
    as the reference does, and says so in the report."""
    _, cfg, f = make_setup(tmp_path, "gyre", N=18, Ny=9, solver=2, tol=1e-12, dt=900.0)
    o = oracle_mod.Oracle(cfg, f)
    m = lib.Model(cfg, f)
    o.prelim()
    m.prelim()
    for n in range(1, 4):
        o.integrator_step(n)
        o.pressure(True)
        st = m.step(n)
        assert st["fallback"] == 1
    s_o, s_g = o.state(), m.state()
    for var in ("u", "v", "h"):
        assert rel_l2(s_g[var], s_o[var]) < 1e-8, var


@pytest.mark.gpu
@pytest.mark.parametrize("kind,kw", [
    ("gyre", dict(N=256, solver=1, tol=1e-12, dt=450.0)),
    ("jets", dict(N=128, solver=1, tol=1e-12, dt=100.0)),
], ids=["gyre256", "jets128"])
def test_mg_omega_choice(tmp_path, oracle_mod, lib, kind, kw):
    """The automatic red-black weight: the start-up solve uses 1.0, the first time-step
    solve tries every candidate from the same pressure and keeps the one with the fewest
    V-cycles (so two models choose the same); the choice never needs more V-cycles than
    1.0 on that solve, and the state still agrees with the oracle to the solver tolerance."""
    _, cfg, f = make_setup(tmp_path, kind, **kw)
    runs = {}
    for omega in (1.0, -1.0, -1.0):
        m = lib.Model(cfg, f, mg_omega=omega)
        m.prelim()
        reps = [m.step(n) for n in range(1, 5)]
        runs.setdefault(omega, []).append((reps, m.state()))
    fixed = runs[1.0][0][0]
    (auto_a, sa), (auto_b, sb) = runs[-1.0]
    assert fixed[0]["mg_omega"] == 1.0
    chosen = auto_a[0]["mg_omega"]
    assert chosen in (1.0, 1.05, 1.1, 1.15, 1.2, 1.3)
    assert all(r["mg_omega"] == chosen for r in auto_a + auto_b)
    assert [r["iters"] for r in auto_a] == [r["iters"] for r in auto_b]
    for var in ("u", "v", "h"):
        assert np.array_equal(sa[var], sb[var])
    assert auto_a[0]["iters"] <= fixed[0]["iters"]
    o = oracle_mod.Oracle(cfg, f)
    o.prelim()
    for n in range(1, 5):
        o.integrator_step(n)
        o.pressure(True)
    so = o.state()
    for var in ("u", "v", "h"):
        assert rel_l2(sa[var], so[var]) < 1e-9, (var, rel_l2(sa[var], so[var]))


@pytest.mark.parametrize("fp32", [0, 1], ids=["fp64", "fp32-defect"])
@pytest.mark.parametrize("kind,kw", [
    ("gyre", dict(N=16, solver=1, tol=1e-13, dt=900.0)),
    ("gyre", dict(N=128, solver=1, tol=1e-13, dt=900.0)),
    ("channel", dict(Nx=128, Ny=64, solver=1, tol=1e-13, dt=150.0)),
    ("jets", dict(N=64, solver=1, tol=1e-13, dt=100.0)),
    ("gyre", dict(N=48, Ny=40, solver=1, tol=1e-13, dt=900.0)),
], ids=["gyre16", "gyre128", "channel128x64", "jets64", "gyre48x40"])
def test_full_mg_tolerance(tmp_path, oracle_mod, lib, fp32, kind, kw):
    """use_fullMG 1 (multigrid.c:1236-1270): the rhs restricted to every level, the nested
    iteration from the 1 x 1 level up (each level's V-cycles to the tolerance), then the finest
    level's iteration, on the whole coarse block (16 x 16), tiled levels (128 x 128, 128 x 64,
    64 x 64) and uneven coarsening (48 x 40). The oracle runs the reference's full_MG; the states
    stay within 1e-9 of it over 6 steps at tol 1e-13, and each solve meets the stopping test.
    V-cycle counts are not compared: the red-black smoother with its tuned weight needs about
    half the cycles of the reference's lexicographic sweep (10-11 against 24-25 here)."""
    extra = dict(kw.pop("extra", {}))
    extra["use_fullMG"] = 1
    _, cfg, f = make_setup(tmp_path, kind, extra=extra, **kw)
    assert cfg.values["use_fullMG"]
    o = oracle_mod.Oracle(cfg, f)
    m = lib.Model(cfg, f, mg_fp32=fp32)
    o.prelim()
    m.prelim()
    for n in range(1, 7):
        o.integrator_step(n)
        so = o.pressure(True)
        st = m.step(n)
        assert 1 <= st["iters"] < 80, st
        assert st["stop_measure"] <= 1e-13
        assert so.iters >= 1
    s_o, s_g = o.state(), m.state()
    for var in ("u", "v", "h"):
        assert rel_l2(s_g[var], s_o[var]) < 1e-9, (var, rel_l2(s_g[var], s_o[var]))


@pytest.mark.parametrize("fp32", [0, 1], ids=["fp64", "fp32-defect"])
@pytest.mark.parametrize("kind,kw", [
    ("gyre", dict(N=128, solver=1, tol=1e-12, dt=900.0)),
    ("gyre", dict(N=48, Ny=40, solver=0, tol=1e-10, dt=900.0)),
    ("channel", dict(Nx=128, Ny=64, solver=1, tol=1e-12, dt=150.0)),
], ids=["gyre128-mg", "gyre48x40-sor", "channel-mg"])
def test_run_without_host_syncs_matches_steps(tmp_path, lib, fp32, kind, kw):
    """pawsim_gpu_run enqueues the steps whose correction needs no host report back to back
    (device-side iteration counts, the FP32 solve's final copy decided on the device): the
    states and every step's iteration count equal those of pawsim_gpu_step called step by
    step."""
    _, cfg, f = make_setup(tmp_path, kind, **kw)
    a = lib.Model(cfg, f, mg_fp32=fp32)
    b = lib.Model(cfg, f, mg_fp32=fp32)
    a.prelim()
    b.prelim()
    want = [a.step(n)["iters"] for n in range(1, 13)]
    st = b.run(1, 12)
    got = list(b.run_iterations())
    assert got == want, (got, want)
    assert st["iters"] == want[-1]
    for var in ("u", "v", "h"):
        assert value_equal(a.state()[var], b.state()[var]), var
    assert value_equal(a.get("pi"), b.get("pi"))
