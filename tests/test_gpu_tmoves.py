"""T-moves (Casula's moves from the negative nonlocal matrix elements): the
engine's selection over many copies of one configuration follows the
probabilities tau |v_xx| / (1 + tau sum |v_xx|) of the reference's
Dmc_method::doTmove, with v_xx and the target points from the oracle; DMC
with T-moves runs."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
import qworacle
from mainline_b200 import engine, systems

pytestmark = pytest.mark.gpu

DECK = os.path.join(GOLDEN, "n2_pseudo.qw")
W = 16384
TAU = 0.3


@pytest.fixture(scope="module")
def case():
    g = np.load(os.path.join(GOLDEN, "n2_pseudo.npz"))
    R, rot = g["R"][0], g["rot"][0]
    terms = qworacle.System(DECK).tmove_terms(R, rot)
    return R, rot, terms


def _engine(R, rot):
    E = engine.Engine(DECK, engine.FP64, max_walkers=W)
    E.set_walkers(np.broadcast_to(R, (W,) + R.shape).copy())
    return E, np.broadcast_to(rot, (W, 3, 3)).copy()


def _match(terms, e, x):
    """Index of the oracle term of electron e whose target is x."""
    best = min(((np.max(np.abs(t[1] - x)), k) for k, t in enumerate(terms) if t[0] == e), default=(1.0, -1))
    return best[1] if best[0] < 1e-9 else -1


def test_size_consistent_selection(case):
    R, rot, terms = case
    E, rots = _engine(R, rot)
    moved, pos = E.tmove_select(2, TAU, seed=7, rot=rots)
    N = R.shape[0]
    for e in range(N):
        neg = [(k, t[2]) for k, t in enumerate(terms) if t[0] == e and t[2] < 0]
        s = 1.0 + TAU * sum(-v for _, v in neg)
        p_move = 1.0 - 1.0 / s
        f = moved[:, e].mean()
        assert abs(f - p_move) < 5 * np.sqrt(max(p_move * (1 - p_move), 1e-12) / W) + 1e-12, (e, f, p_move)
        # every target is one of the electron's negative-term points, with
        # the per-point frequencies of tau |v| / s
        counts = {}
        for w in np.flatnonzero(moved[:, e]):
            k = _match(terms, e, pos[w, e])
            assert k >= 0 and terms[k][2] < 0
            counts[k] = counts.get(k, 0) + 1
        for k, v in neg:
            p = TAU * (-v) / s
            assert abs(counts.get(k, 0) / W - p) < 5 * np.sqrt(p * (1 - p) / W) + 1e-12


def test_one_move_per_walker_selection(case):
    R, rot, terms = case
    E, rots = _engine(R, rot)
    moved, pos = E.tmove_select(1, TAU, seed=11, rot=rots)
    assert moved.sum(axis=1).max() <= 1
    s = 1.0 + TAU * sum(-t[2] for t in terms if t[2] < 0)
    f = 1.0 - moved.any(axis=1).mean()
    p0 = 1.0 / s
    assert abs(f - p0) < 5 * np.sqrt(p0 * (1 - p0) / W)
    for w in np.flatnonzero(moved.any(axis=1))[:500]:
        e = int(np.flatnonzero(moved[w])[0])
        k = _match(terms, e, pos[w, e])
        assert k >= 0 and terms[k][2] < 0


@pytest.mark.parametrize("mode", [1, 2])
def test_dmc_with_tmoves_runs(mode):
    d = systems.read_deck(DECK)
    E = engine.Engine(DECK, engine.MIXED, max_walkers=1024)
    E.set_walkers(systems.random_configs(d, 1024, seed=3))
    E.vmc_block(10, 0.3, seed=4)
    E.dmc_init(timestep=0.01, nstep=10, seed=5, tmoves=mode)
    # from a random-orbital trial function the trial energy lags the first
    # blocks and the mean weight climbs: third-block means of 2.7-3.2 over six
    # seeds, with and without T-moves; the cap per walker is 7
    for _ in range(3):
        s = E.dmc_block()
        assert np.isfinite(s["energy"]) and s["nonfinite"] == 0 and 0.3 < s["weight"] < 5.0
    R = E.get_walkers()
    E2 = engine.Engine(DECK, engine.FP64, max_walkers=1024)
    E2.set_walkers(R)
    assert np.all(np.isfinite(E2.eval().energy))
