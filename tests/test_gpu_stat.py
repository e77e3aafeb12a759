"""Statistical parity: block-averaged VMC and DMC energies of the engine
against the reference's own runs on the same deck, FP64 and mixed precision.

The deck (tests/golden/h4pp.qw) is a four-atom hydrogen pseudo-atom chain
with RHF orbitals and a Slater-Jastrow trial function (local-energy variance
~0.18 Ha^2), so a few million walker-steps pin the energy to a fraction of
a mHa.  tests/golden/stat_ref.json holds the reference qwalk's energies,
written by tests/golden/make_stat.py (8 independent processes, reblocked).

* VMC (tau 0.5, Split_sampler depth 2): the expectation over |psi|^2 is
  fixed by the wave function and the local energy; the test pins the
  Metropolis sampler (Vmc_method.cpp:351-558, Split_sample.cpp:302-540).
* DMC at tau 0.05 (Dmc_method.cpp:328-567): the fixed-node energy carries a
  time-step error of several mHa at this tau, so the drift-diffusion Green's
  function, the node restriction, the effective time step, the weights with
  their cut-offs (:780-824) and the branching (:961-995) all have to match
  the reference's for the energies to agree.  The DMC-VMC gap is ~75 mHa.

The bound is 4 combined standard errors (both sides reblocked)."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from statutil import reblock
from mainline_b200 import engine, systems

pytestmark = pytest.mark.gpu

DECK = os.path.join(GOLDEN, "h4pp.qw")
REF = json.load(open(os.path.join(GOLDEN, "stat_ref.json")))
NW = 4096


def _walkers(seed):
    d = systems.read_deck(DECK)
    return systems.random_configs(d, NW, seed=seed)


def _check(label, mean, err, ref):
    comb = float(np.hypot(err, ref["error"]))
    dev = mean - ref["energy"]
    print(f"STAT {label}: engine {mean:.5f} +- {err * 1e3:.3f} mHa, reference {ref['energy']:.5f} +- "
          f"{ref['error'] * 1e3:.3f} mHa, difference {dev * 1e3:+.3f} mHa = {dev / comb:+.2f} sigma")
    assert comb < 1e-3, "error bars too wide to pin the energy"
    assert abs(dev) < 4 * comb


@pytest.mark.parametrize("precision", [engine.FP64, engine.MIXED], ids=["fp64", "mixed"])
def test_vmc_energy_matches_reference(precision):
    r = REF["vmc"]
    E = engine.Engine(DECK, precision, max_walkers=NW)
    E.set_walkers(_walkers(11))
    for b in range(10):
        E.vmc_block(r["steps_per_block"], r["timestep"], seed=100 + b)
    en = [E.vmc_block(r["steps_per_block"], r["timestep"], seed=1000 + b)["energy"] for b in range(200)]
    E.close()
    mean, err = reblock(en)
    _check("VMC " + ("fp64" if precision == engine.FP64 else "mixed"), mean, err, r)


@pytest.mark.parametrize("precision", [engine.FP64, engine.MIXED], ids=["fp64", "mixed"])
def test_dmc_energy_matches_reference(precision):
    r = REF["dmc_tau0.05"]
    E = engine.Engine(DECK, precision, max_walkers=NW)
    E.set_walkers(_walkers(12))
    for b in range(10):
        E.vmc_block(20, 0.5, seed=200 + b)
    E.dmc_init(timestep=r["timestep"], nstep=r["steps_per_block"], seed=77)
    for _ in range(r["equilibration_blocks"]):
        E.dmc_block()
    st = [E.dmc_block() for _ in range(300)]
    E.close()
    en = [s["energy"] for s in st]
    assert all(0.9 < s["acceptance"] <= 1.0 for s in st)
    mean, err = reblock(en)
    _check("DMC tau=0.05 " + ("fp64" if precision == engine.FP64 else "mixed"), mean, err, r)


def test_dmc_energy_large_population_matches_reference():
    """16384 walkers: population control on the device-wide sort."""
    r = REF["dmc_tau0.05"]
    d = systems.read_deck(DECK)
    E = engine.Engine(DECK, engine.FP64, max_walkers=16384)
    E.set_walkers(systems.random_configs(d, 16384, seed=14))
    for b in range(10):
        E.vmc_block(20, 0.5, seed=400 + b)
    E.dmc_init(timestep=r["timestep"], nstep=r["steps_per_block"], seed=78)
    for _ in range(r["equilibration_blocks"]):
        E.dmc_block()
    en = [E.dmc_block()["energy"] for _ in range(120)]
    E.close()
    mean, err = reblock(en)
    _check("DMC tau=0.05 fp64, 16384 walkers", mean, err, r)


def test_dmc_mixed_within_0p1_mHa_of_fp64():
    """Mixed minus FP64 DMC energy with common random numbers: both start
    from the same walkers with the same seed, so the walks coincide until a
    decision (an acceptance, or the order of two nearly equal weights in the
    branching) falls inside the precision difference; while they coincide,
    the per-block difference measures the precision bias directly.  Once a
    walk has parted, blocks differ by their statistical noise, so the bound
    is 0.1 mHa plus three standard errors of the mean difference."""
    r = REF["dmc_tau0.05"]
    R0 = _walkers(13)
    en = {}
    for prec in (engine.FP64, engine.MIXED):
        E = engine.Engine(DECK, prec, max_walkers=NW)
        E.set_walkers(R0)
        for b in range(5):
            E.vmc_block(20, 0.5, seed=300 + b)
        E.dmc_init(timestep=r["timestep"], nstep=20, seed=91)
        en[prec] = np.array([E.dmc_block()["energy"] for _ in range(30)])
        E.close()
    d = (en[engine.MIXED] - en[engine.FP64]) * 1e3
    mean, sem = float(np.mean(d)), float(np.std(d, ddof=1) / np.sqrt(len(d)))
    print(f"MIXED_MINUS_FP64 DMC tau=0.05: {mean:+.5f} +- {sem:.5f} mHa over {len(d)} blocks; per block "
          + " ".join(f"{x:+.4f}" for x in d))
    assert sem < 1.0
    assert abs(mean) < 0.1 + 3 * sem
