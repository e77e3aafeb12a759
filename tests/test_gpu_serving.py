"""The continuous-batching job server on one GPU: a job's results are the
same alone and in a mix of concurrent jobs (including an HBM-resident
large system), and admission never exceeds the device-memory budget."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from mainline_b200 import engine, systems

pytestmark = pytest.mark.gpu


def _drive(srv):
    events = []
    while True:
        events += srv.progress()
        st = srv.status()
        if st["queued"] == 0 and st["active"] == 0:
            return events, st


def _job(srv, name, nw, blocks, seed):
    deck = os.path.join(GOLDEN, name + ".qw")
    R = systems.random_configs(systems.read_deck(deck), nw, seed=seed)
    return srv.submit(deck, R, engine.MIXED, blocks, dict(timestep=0.01, nstep=3, seed=seed + 1),
                      vmc_blocks=1, vmc_steps=3, vmc_seed=seed + 2)


def test_job_same_alone_and_in_mix():
    budget = 8 << 30
    srv = engine.Server(budget)
    a = _job(srv, "n2_pseudo", 256, 3, 5)
    alone, _ = _drive(srv)
    srv.close()
    srv = engine.Server(budget)
    _job(srv, "mol43", 128, 2, 9)
    a2 = _job(srv, "n2_pseudo", 256, 3, 5)
    _job(srv, "mol72", 64, 2, 13)
    mix, st = _drive(srv)
    srv.close()
    assert st["finished"] == 3 and st["failed"] == 0
    ea = [e["energy"] for e in sorted((e for e in alone if e["job"] == a), key=lambda e: e["block"])]
    em = [e["energy"] for e in sorted((e for e in mix if e["job"] == a2), key=lambda e: e["block"])]
    assert len(ea) == len(em) == 3
    assert np.allclose(ea, em, rtol=1e-12, atol=0), (ea, em)
    assert all(e["latency_ms"] > 0 and np.isfinite(e["energy"]) for e in mix)


def test_admission_respects_budget():
    fp = [engine.footprint(os.path.join(GOLDEN, n + ".qw"), engine.MIXED, 256) for n in ("n2_pseudo", "mol43")]
    budget = max(fp) + 1024  # one job at a time
    srv = engine.Server(budget)
    for k in range(3):
        _job(srv, ("n2_pseudo", "mol43")[k % 2], 256, 2, 20 + k)
    max_active = 0
    while True:
        srv.progress()
        st = srv.status()
        max_active = max(max_active, st["active"])
        assert st["bytes_in_use"] <= budget
        if st["queued"] == 0 and st["active"] == 0:
            break
    srv.close()
    assert max_active == 1 and st["finished"] == 3
