"""Population control through the C-ABI: the one-CTA kernel (populations
up to 8192 walkers: bitonic sort in shared memory) and the device-wide
pipeline (larger populations: stable 8-bit radix passes over all CTAs,
parallel pairing, one-CTA gather map) implement the same match_walkers
pairing (Dmc_method.cpp:961-995) and copy order (:1099-1107).  Forcing the
device-wide pipeline on a small population (QWG_BRANCH_DEVICE_WIDE=1) must
reproduce the one-CTA walk: the sort orders are identical (ascending weight,
ties by walker index) and only the weight sum behind E_T may round
differently."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from mainline_b200 import engine, systems

pytestmark = pytest.mark.gpu


def _dmc(deck, R0, device_wide, blocks=2, nstep=20):
    old = os.environ.get("QWG_BRANCH_DEVICE_WIDE")
    os.environ["QWG_BRANCH_DEVICE_WIDE"] = "1" if device_wide else "0"
    try:
        E = engine.Engine(deck, engine.FP64, max_walkers=len(R0))
    finally:
        if old is None:
            del os.environ["QWG_BRANCH_DEVICE_WIDE"]
        else:
            os.environ["QWG_BRANCH_DEVICE_WIDE"] = old
    E.set_walkers(R0)
    E.vmc_block(5, 0.3, seed=4)
    E.dmc_init(timestep=0.01, nstep=nstep, seed=5)
    st = [E.dmc_block() for _ in range(blocks)]
    R = E.get_walkers()
    _, w = E.walker_scalars()
    E.close()
    return st, R, w


def test_device_wide_population_control_matches_one_cta():
    deck = os.path.join(GOLDEN, "n2_pseudo.qw")
    R0 = systems.random_configs(systems.read_deck(deck), 4096, seed=21)
    st1, R1, w1 = _dmc(deck, R0, False)
    st2, R2, w2 = _dmc(deck, R0, True)
    dev = float(np.max(np.abs(R1 - R2)))
    print(f"BRANCH one-CTA vs device-wide: max position difference {dev:.1e}, energies "
          f"{st1[-1]['energy']:.6f} / {st2[-1]['energy']:.6f}")
    assert dev < 1e-9
    assert np.allclose(w1, w2, rtol=1e-12, atol=0)
    for a, b in zip(st1, st2):
        assert abs(a["energy"] - b["energy"]) < 1e-9 * max(1.0, abs(a["energy"]))


def test_large_population_stays_constant_and_finite():
    deck = os.path.join(GOLDEN, "h4pp.qw")
    R0 = systems.random_configs(systems.read_deck(deck), 20000, seed=22)  # above 8192, not a power of two
    st, R, w = _dmc(deck, R0, False, blocks=3, nstep=10)
    assert R.shape[0] == 20000 and np.all(np.isfinite(R))
    assert np.all(np.isfinite(w)) and np.all(w > 0) and np.all(w <= 7.0)
    for s in st:
        assert np.isfinite(s["energy"]) and 0.5 < s["weight"] < 2.0
