"""Error handling through the C-ABI on a GPU: calls out of order and
unsupported requests return their status class with a message, and the
context stays usable afterwards."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from mainline_b200 import engine, systems

pytestmark = pytest.mark.gpu


def test_calls_out_of_order_and_recovery():
    deck = os.path.join(GOLDEN, "n2_pseudo.qw")
    d = systems.read_deck(deck)
    E = engine.Engine(deck, engine.FP64, max_walkers=64)
    with pytest.raises(engine.QwgError, match="no walkers"):
        E.eval()
    E.set_walkers(systems.random_configs(d, 64, seed=1))
    with pytest.raises(engine.QwgError, match="qwg_dmc_init first"):
        E.dmc_block()
    with pytest.raises(engine.QwgError, match="no block has run"):
        E.walker_scalars()
    with pytest.raises(engine.QwgError, match="qwg_dmc_init first"):
        E.time_kernels(2)
    with pytest.raises(engine.QwgError, match="bad walker count"):
        E.set_walkers(systems.random_configs(d, 65, seed=1))
    with pytest.raises(engine.QwgError, match="tmoves must be"):
        E.dmc_init(timestep=0.01, nstep=5, tmoves=3)
    # the context still works after every refusal
    E.dmc_init(timestep=0.01, nstep=5, seed=2)
    s = E.dmc_block()
    assert np.isfinite(s["energy"])
    E.dmc_block_async()
    with pytest.raises(engine.QwgError, match="not collected"):
        E.dmc_block_async()
    assert np.isfinite(E.dmc_block_wait()["energy"])


def test_tmoves_need_a_pseudopotential():
    deck = os.path.join(GOLDEN, "n2_allelectron.qw")
    d = systems.read_deck(deck)
    E = engine.Engine(deck, engine.FP64, max_walkers=32)
    E.set_walkers(systems.random_configs(d, 32, seed=3))
    with pytest.raises(engine.QwgError, match="pseudopotential"):
        E.dmc_init(timestep=0.01, nstep=5, tmoves=2)
    with pytest.raises(engine.QwgError):
        E.tmove_select(2, 0.1)
    E.dmc_init(timestep=0.01, nstep=5, seed=4)
    assert np.isfinite(E.dmc_block()["energy"])


def test_create_reports_a_missing_deck(tmp_path):
    with pytest.raises(engine.QwgError):
        engine.Engine(str(tmp_path / "missing.qw"), engine.FP64, max_walkers=8)
