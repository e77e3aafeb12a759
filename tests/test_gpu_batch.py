"""Batched uneven systems on one GPU: several decks of different sizes
(electron counts, atoms, basis sizes, walker counts) advanced together, one
DMC block of every system per CUDA graph launch.  Each system's statistics
must equal those of the same system run alone with the same seeds: walker
state, trial energy and the counter-based RNG stream are per system."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from mainline_b200 import engine, systems

pytestmark = pytest.mark.gpu


def _setup(deck, nw, seed):
    E = engine.Engine(deck.path, engine.MIXED, max_walkers=nw)
    E.set_walkers(systems.random_configs(deck, nw, seed=seed))
    E.vmc_block(10, 0.3, seed=seed + 1)
    E.dmc_init(timestep=0.01, nstep=5, seed=seed + 2)
    return E


def test_batch_blocks_match_standalone(tmp_path):
    decks = systems.write_batch(str(tmp_path), nsys=4, seed=31)
    decks = [(d, min(nw, 1024)) for d, nw in decks]
    alone = []
    for i, (d, nw) in enumerate(decks):
        E = _setup(d, nw, 100 + 10 * i)
        alone.append([E.dmc_block()["energy"] for _ in range(2)])
        E.close()
    engines = [_setup(d, nw, 100 + 10 * i) for i, (d, nw) in enumerate(decks)]
    B = engine.Batch(engines)
    got = [[] for _ in engines]
    for _ in range(2):
        for k, s in enumerate(B.block()):
            assert np.isfinite(s["energy"]) and s["nonfinite"] == 0
            got[k].append(s["energy"])
    B.close()
    for k in range(len(engines)):
        assert np.allclose(got[k], alone[k], rtol=1e-12, atol=0), (k, got[k], alone[k])


def test_autotune_returns_valid_walkers_per_cta():
    deck = os.path.join(GOLDEN, "mol43.qw")
    d = systems.read_deck(deck)
    E = engine.Engine(deck, engine.MIXED, max_walkers=512)
    E.set_walkers(systems.random_configs(d, 512, seed=2))
    wpc = E.autotune()
    assert wpc in (1, 2, 4)
    ev = E.eval()
    assert np.all(np.isfinite(ev.energy))
