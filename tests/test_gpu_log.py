"""Block point statistics and QWalk log output from real engine runs: the
variances follow the reference's definitions, and the reference's gosling
analyser reads the engine's DMC log."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
from mainline_b200 import engine, systems

pytestmark = pytest.mark.gpu

GOSLING = os.path.join(ROOT, "oracle", "_ref", "gosling")


def test_vmc_block_point_statistics():
    deck = os.path.join(GOLDEN, "n2_pseudo.qw")
    nw, ns = 256, 10
    E = engine.Engine(deck, engine.FP64, max_walkers=nw)
    E.set_walkers(systems.random_configs(systems.read_deck(deck), nw, seed=3))
    E.vmc_block(10, 0.3, seed=1)
    s = E.vmc_block(ns, 0.3, seed=2)
    n = nw * ns
    assert s["npoints"] == n and s["weight"] == 1.0 and s["var_weight"] == 0.0
    # all weights are 1 in VMC: the point variance is the weighted one times n/(n-1)
    assert np.isclose(s["var_energy"], s["energy_var"] * n / (n - 1), rtol=1e-8)
    for k in ("var_kinetic", "var_potential", "var_nonlocal"):
        assert np.isfinite(s[k]) and s[k] > 0


def test_dmc_log_read_by_gosling(tmp_path):
    deck = os.path.join(GOLDEN, "n2_pseudo.qw")
    nw = 512
    E = engine.Engine(deck, engine.MIXED, max_walkers=nw)
    E.set_walkers(systems.random_configs(systems.read_deck(deck), nw, seed=4))
    E.vmc_block(10, 0.3, seed=5)
    E.dmc_init(timestep=0.01, nstep=10, seed=6)
    log = str(tmp_path / "run.log")
    engine.log_header(log, "DMC", "dmc", 0.01)
    energies = []
    for _ in range(4):
        s = E.dmc_block()
        assert s["npoints"] == nw * 10 and s["var_weight"] > 0 and s["var_energy"] > 0
        engine.log_block(log, "dmc", s)
        energies.append(s["energy"])
    if not os.path.exists(GOSLING):
        pytest.skip("reference gosling not built")
    out = subprocess.run([GOSLING, "-no_equil", log], capture_output=True, text=True, timeout=60, check=True).stdout
    assert "4 total blocks" in out
    m = re.search(r"total_energy0\s+(\S+)", out)
    assert m and min(energies) - 1e-6 <= float(m.group(1)) <= max(energies) + 1e-6


def test_store_configs_round_trip(tmp_path):
    """The resident DMC walkers written as a QWalk configuration file read
    back as the same positions, weights and signs."""
    deck = os.path.join(GOLDEN, "n2_pseudo.qw")
    nw = 256
    E = engine.Engine(deck, engine.FP64, max_walkers=nw)
    E.set_walkers(systems.random_configs(systems.read_deck(deck), nw, seed=8))
    E.vmc_block(5, 0.3, seed=9)
    E.dmc_init(timestep=0.01, nstep=10, seed=10)
    E.dmc_block()
    p = str(tmp_path / "run.config")
    E.store_configs(p, dmc=True)
    R, w, sg = engine.read_configs(p)
    assert np.allclose(R, E.get_walkers(), rtol=1e-14, atol=1e-14)
    assert np.allclose(w, E.walker_scalars()[1], rtol=1e-14)
    assert set(np.unique(sg)) <= {-1.0, 1.0}
    E2 = engine.Engine(deck, engine.FP64, max_walkers=nw)
    E2.set_walkers(R)
    assert np.all(np.isfinite(E2.eval().energy))
