"""Host-side behaviour of the job server without a GPU: footprint estimates,
queueing and the budget check at submission (no context is created until a
progress call admits a job)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from mainline_b200 import engine, systems


def test_footprint_grows_with_walkers_and_precision():
    deck = os.path.join(GOLDEN, "n2_pseudo.qw")
    a, b = engine.footprint(deck, engine.MIXED, 1024), engine.footprint(deck, engine.MIXED, 2048)
    c = engine.footprint(deck, engine.FP64, 1024)
    assert 0 < a < b and c > a
    big = engine.footprint(os.path.join(GOLDEN, "cell32.qw"), engine.MIXED, 1024)
    assert big > 10 * a


def test_submit_queues_and_rejects_oversized_jobs():
    deck = os.path.join(GOLDEN, "n2_pseudo.qw")
    R = systems.random_configs(systems.read_deck(deck), 64, seed=1)
    need = engine.footprint(deck, engine.MIXED, 64)
    srv = engine.Server(need + 1)
    jid = srv.submit(deck, R, engine.MIXED, 2, dict(nstep=2))
    assert jid == 0 and srv.status()["queued"] == 1
    R2 = systems.random_configs(systems.read_deck(deck), 4096, seed=1)
    with pytest.raises(engine.QwgError, match="budget"):
        srv.submit(deck, R2, engine.MIXED, 2, dict(nstep=2))
    with pytest.raises(engine.QwgError):
        srv.submit(os.path.join(GOLDEN, "missing.qw"), R, engine.MIXED, 2, dict(nstep=2))
    srv.close()
