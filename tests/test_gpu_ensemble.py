"""The batched ensemble against its members run alone.

An ensemble advances members of different grid sizes with one fused-kernel launch per step
over all members' tiles and each member's rigid-lid correction on its own stream. Every tile
computes what the member's own launch computes and every correction is the member's own, so
after the same steps each member's state, pressure and per-step iteration counts must equal,
bit for bit, those of the same model advanced alone with Model.run.
"""
import numpy as np
import pytest

from conftest import make_setup

pytestmark = pytest.mark.gpu

EUNSUPPORTED = -5


def _jets(tmp_path, tag, N, seed, solver=1, **extra):
    # dx = 4 km on every member, as the 256^2 / 512^2 jets ensemble (dt = 600 s stays stable)
    _, cfg, f = make_setup(tmp_path / tag, "jets", N=N, Ly=N * 4e3, dt=600.0, seed=seed, solver=solver,
                           **extra)
    return cfg, f


def _state(m):
    s = m.state()
    return {k: np.array(s[k]) for k in ("u", "v", "h")} | {"pi": np.array(m.get("pi"))}


def _check_members(members, alone, iters):
    """State and pressure bitwise, the per-step iteration counts, the model time."""
    for i, (a, b) in enumerate(zip(members, alone)):
        sa, sb = _state(a), _state(b)
        for k in sa:
            assert np.array_equal(sa[k], sb[k]), (i, k, np.abs(sa[k] - sb[k]).max())
        assert np.array_equal(iters[i], b.run_iterations()), (i, iters[i], b.run_iterations())
        assert a.t == b.t


@pytest.mark.parametrize("solver,graphs", [(0, True), (1, True), (1, False)])
def test_uneven_jets_members_equal_alone(tmp_path, solver, graphs):
    """Three 64^2 and two 128^2 jets members with distinct noise seeds; multigrid (the first
    solves tune it synchronously, then whole steps replay captured graphs, or run on streams
    with graphs off) and red-black SOR (streams)."""
    import pawsim_b200

    specs = [(64, 11), (128, 12), (64, 13), (128, 14), (64, 15)]
    setups = [_jets(tmp_path, f"m{i}", N, seed, solver=solver) for i, (N, seed) in enumerate(specs)]
    steps = 12
    alone = []
    for cfg, f in setups:
        m = pawsim_b200.Model(cfg, f)
        m.prelim()
        m.run(1, steps)
        alone.append(m)
    members = []
    for cfg, f in setups:
        m = pawsim_b200.Model(cfg, f)
        m.prelim()
        members.append(m)
    ens = pawsim_b200.Ensemble(members)
    ens.set_graphs(graphs)
    ens.run(1, 5)
    it1 = [m.run_iterations() for m in members]
    ens.run(6, steps - 5)
    it2 = [m.run_iterations() for m in members]
    # the multigrid members replay graphs from the first step whose loops are built; the
    # cooperative SOR launch stays on streams
    if graphs and solver == 1:
        assert ens.graph_steps() == steps - 5
        assert ens.batched_mg()   # one batched multigrid loop for the 64^2 and 128^2 groups
    else:
        assert ens.graph_steps() == 0
    ens.close()
    _check_members(members, alone, [np.concatenate([a, b]) for a, b in zip(it1, it2)])
    # closed, the members step on alone exactly like their twins
    for a, b in zip(members[:2], alone[:2]):
        a.run(steps + 1, 3)
        b.run(steps + 1, 3)
    _check_members(members[:2], alone[:2], [m.run_iterations() for m in members[:2]])
    for m in members + alone:
        m.close()


def test_walled_gyres_of_two_sizes(tmp_path):
    """Closed-basin gyres (wall faces, wind, linear drag) of 48 x 40 and 96 x 64 with SOR."""
    import pawsim_b200

    shapes = [(48, 40), (96, 64), (48, 40)]
    setups = []
    for i, (nx, ny) in enumerate(shapes):
        _, cfg, f = make_setup(tmp_path / f"g{i}", "gyre", N=nx, Ny=ny, solver=0, dt=900.0)
        setups.append((cfg, f))
    steps = 6
    alone = []
    for cfg, f in setups:
        m = pawsim_b200.Model(cfg, f)
        m.prelim()
        m.run(1, steps)
        alone.append(m)
    members = []
    for cfg, f in setups:
        m = pawsim_b200.Model(cfg, f)
        m.prelim()
        members.append(m)
    ens = pawsim_b200.Ensemble(members)
    ens.run(1, steps)
    _check_members(members, alone, [m.run_iterations() for m in members])
    ens.close()
    # after the ensemble is closed a member steps on alone exactly like its twin
    members[1].run(steps + 1, 2)
    alone[1].run(steps + 1, 2)
    sa, sb = _state(members[1]), _state(alone[1])
    for k in sa:
        assert np.array_equal(sa[k], sb[k]), k
    for m in members + alone:
        m.close()


def test_walled_multigrid_members(tmp_path):
    """Closed-basin gyres with the multigrid (wall faces in every level kernel), two sizes, whole
    steps as graph replays with the batched multigrid loop; the per-member iteration counts
    differ between members and each member stops at its own test."""
    import pawsim_b200

    shapes = [(64, 64), (128, 64), (64, 64), (128, 128)]
    setups = []
    for i, (nx, ny) in enumerate(shapes):
        _, cfg, f = make_setup(tmp_path / f"w{i}", "gyre", N=nx, Ny=ny, solver=1, dt=900.0 * 64 / nx,
                               seed=i)
        setups.append((cfg, f))
    steps = 10
    alone = []
    for cfg, f in setups:
        m = pawsim_b200.Model(cfg, f)
        m.prelim()
        m.run(1, steps)
        alone.append(m)
    members = []
    for cfg, f in setups:
        m = pawsim_b200.Model(cfg, f)
        m.prelim()
        members.append(m)
    ens = pawsim_b200.Ensemble(members)
    ens.run(1, 4)
    it1 = [m.run_iterations() for m in members]
    ens.run(5, steps - 4)
    it2 = [m.run_iterations() for m in members]
    assert ens.graph_steps() == steps - 4 and ens.batched_mg()
    ens.close()
    _check_members(members, alone, [np.concatenate([a, b]) for a, b in zip(it1, it2)])
    for m in members + alone:
        m.close()


def test_ensemble_refuses_mixed_members(tmp_path):
    import pawsim_b200

    cfg_a, fa = _jets(tmp_path, "a", 64, 1)
    _, cfg_b, fb = make_setup(tmp_path / "b", "channel", Nx=64, Ny=32, solver=1, dt=600.0)
    a = pawsim_b200.Model(cfg_a, fa)
    b = pawsim_b200.Model(cfg_b, fb)
    assert cfg_a.values["Nlay"] != cfg_b.values["Nlay"]
    with pytest.raises(pawsim_b200.PawsimError) as e:
        pawsim_b200.Ensemble([a, b])
    assert e.value.code == EUNSUPPORTED
    with pytest.raises(pawsim_b200.PawsimError):
        pawsim_b200.Ensemble([a, a])
    a.close()
    b.close()
