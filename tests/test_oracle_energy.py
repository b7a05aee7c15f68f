"""Pins the oracle's energy and enstrophy diagnostics (model_code/diagnostics.c:478-700) to
the reference: on each committed ``*_ez`` fixture the oracle steps the same inputs and every
line of the reference's EZdiags.dat -- KE, PE, KE+PE and the enstrophy of each layer -- must
equal the oracle's sums bit for bit (the file prints 51 significant digits, which read back
to the exact double)."""
import numpy as np
import pytest

from golden_util import load_case

EZ_CASES = ["gyre_sor_ez", "jets_free_ez", "gyre_hk83_free_avg_ez"]


def parse_ez(text):
    """[(t, KE, PE, KE+PE, [Z_k])] from the text of EZdiags.dat."""
    rows = []
    for line in text.splitlines():
        v = [float(x) for x in line.split()]
        rows.append((v[0], v[1], v[2], v[3], v[4:]))
    return rows


def oracle_lines(oracle_mod, cfg, f, nsteps):
    """The EZdiags.dat lines that the oracle's run of nsteps writes (pawsim.c:434-438, 471-509)."""
    o = oracle_mod.Oracle(cfg, f)
    o.prelim()
    every = cfg.values["savefreqEZ"]
    n_ez = int(round(cfg.tmin / every)) + 1
    t_next = cfg.tmin + every
    reload = cfg.values["savefreqAvg"] > 0
    lines = []
    for n in range(1, nsteps + 1):
        o.integrator_step(n)
        if cfg.values["useRL"]:
            o.pressure(True)
        if o.t >= t_next:
            ke, pe, z = o.energy(reload)
            while o.t >= t_next:
                lines.append((t_next, ke, pe, ke + pe, z))
                n_ez += 1
                t_next = n_ez * every
    return lines


@pytest.mark.parametrize("name", EZ_CASES)
def test_oracle_energy_matches_reference(tmp_path, oracle_mod, name):
    cfg, f, z = load_case(name, tmp_path)
    want = parse_ez(str(z["ez_text"]))
    got = oracle_lines(oracle_mod, cfg, f, cfg.Nt)
    assert len(got) == len(want) > 0
    for g, w in zip(got, want):
        assert g[0] == pytest.approx(w[0], rel=1e-6)   # printed as %le
        assert g[1:4] == w[1:4], (g, w)
        assert g[4] == w[4], (g, w)


def test_oracle_energy_eta_source_matters(tmp_path, oracle_mod):
    """Under a free surface the interface heights come from the thickness of the start of the
    step; rebuilding them from the current thickness changes PE, so the fixture pins which."""
    cfg, f, z = load_case("jets_free_ez", tmp_path)
    o = oracle_mod.Oracle(cfg, f)
    o.prelim()
    o.integrator_step(1)
    ke0, pe0, z0 = o.energy(False)
    ke1, pe1, z1 = o.energy(True)
    assert ke0 == ke1 and z0 == z1
    assert pe0 != pe1
    assert np.isfinite([ke0, pe0] + z0).all()
