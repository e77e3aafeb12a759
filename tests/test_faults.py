"""Faulty inputs, injected on the host: non-finite numbers in the tables,
truncated or missing orbital files, and a singular orbital set (an orbital
that is zero everywhere).  The deck
reader (qwg_inspect_deck, no GPU) refuses the first kinds with
QWG_ERR_INPUT and a message; a wave function whose determinant vanishes
everywhere reaches the device, evaluates to log|psi| = -1e201 (an exact zero
determinant) and gets QWG_ERR_NUMERIC from qwg_dmc_init (the reference's
guard is the re-inversion of a singular determinant,
wavefunction/Slat_wf.h:716-753), with the GPU context still usable."""
import os
import re
import shutil

import numpy as np
import pytest

from conftest import GOLDEN
from mainline_b200 import engine, systems


def _copy(tmp_path, name="n2_pseudo"):
    for ext in (".qw", ".orb"):
        shutil.copy(os.path.join(GOLDEN, name + ext), tmp_path / (name + ext))
    return tmp_path / (name + ".qw"), tmp_path / (name + ".orb")


def _refused(deck, pattern):
    with pytest.raises(engine.QwgError, match=pattern):
        engine.inspect_deck(str(deck))


def test_nan_orbital_coefficient(tmp_path):
    deck, orb = _copy(tmp_path)
    txt = orb.read_text()
    head, tail = txt.split("COEFFICIENTS\n", 1)
    vals = tail.split()
    vals[5] = "nan"
    orb.write_text(head + "COEFFICIENTS\n" + " ".join(vals) + "\n")
    _refused(deck, "non-finite")


def test_infinite_pseudopotential_coefficient(tmp_path):
    deck, _ = _copy(tmp_path)
    txt = deck.read_text()
    # the first Gaussian term of the first channel: "2 <exponent> <coefficient>"
    txt = re.sub(r"(OLDQMC \{\s+\S+ \S+\s+\S+ \S+ \S+\s+2 \S+) \S+", r"\1 inf", txt, count=1)
    deck.write_text(txt)
    _refused(deck, "non-finite")


def test_nan_jastrow_coefficient(tmp_path):
    deck, _ = _copy(tmp_path)
    txt = deck.read_text()
    txt = re.sub(r"(COEFFICIENTS \{ N) (\S+)", r"\1 NaN", txt, count=1)
    deck.write_text(txt)
    _refused(deck, "non-finite")


def test_truncated_orbital_file(tmp_path):
    deck, orb = _copy(tmp_path)
    lines = orb.read_text().splitlines()
    orb.write_text("\n".join(lines[:-40]) + "\n")
    _refused(deck, "too few coefficients")


def test_missing_orbital_file(tmp_path):
    deck, orb = _copy(tmp_path)
    orb.unlink()
    _refused(deck, "cannot open ORBFILE")


def _singular_deck(tmp_path):
    """Spin-up orbital 2 made identically zero: its ORB records point at one
    extra coefficient label whose value is 0, so every Slater matrix has a
    zero column (an exactly singular orbital set)."""
    deck, orb = _copy(tmp_path)
    txt = orb.read_text()
    head, tail = txt.split("COEFFICIENTS\n", 1)
    recs = [ln.split() for ln in head.splitlines() if ln.strip()]
    zero = max(int(r[3]) for r in recs) + 1
    out = [" ".join([r[0], r[1], r[2], str(zero) if r[0] == "2" else r[3]]) for r in recs]
    orb.write_text("\n".join(out) + "\nCOEFFICIENTS\n" + tail.rstrip("\n") + "\n0.0\n")
    return deck


@pytest.mark.gpu
def test_singular_orbitals_give_numeric_error(tmp_path):
    deck = _singular_deck(tmp_path)
    d = systems.read_deck(str(deck))
    E = engine.Engine(str(deck), engine.FP64, max_walkers=32)
    E.set_walkers(systems.random_configs(d, 32, seed=1))
    ev = E.eval()
    # log|psi| of an exact zero determinant: -1e201 (what the inversion
    # returns for a zero pivot, as the reference's ludcmp gives up on it)
    assert np.all(ev.logpsi < -1e200)
    with pytest.raises(engine.QwgError, match="finite local energy"):
        E.dmc_init(timestep=0.01, nstep=5, seed=1)
    E.close()
    # the device is fine: a healthy context on it runs
    good = os.path.join(GOLDEN, "n2_pseudo.qw")
    F = engine.Engine(good, engine.FP64, max_walkers=32)
    F.set_walkers(systems.random_configs(systems.read_deck(good), 32, seed=2))
    F.dmc_init(timestep=0.01, nstep=5, seed=3)
    assert np.isfinite(F.dmc_block()["energy"])
    F.close()
