"""GPU parity of the complex-orbital kernels (twisted boundary conditions)
against the golden vectors written by the reference.

diamond8_k: complex orbitals (CORBITALS) at the k-point (0.5, 0.25, 0), so
every image center carries the factor e^{i pi k.n} and the wave function is
complex (Slat_wf<dcomplex>); "sign" is then the phase arg psi.
diamond8_l: real orbitals at the integer k-point (1, 1, 1) (antiperiodic
boundary conditions): image factors cos(pi k.n) = +-1, and the sign of a wrap
enters the pseudopotential points.

Tolerances as for the real kernels: FP64 within 1e-10 relative (Laplacians
1e-9); phases compared as unit complex numbers."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from mainline_b200 import engine, systems

pytestmark = pytest.mark.gpu

NAMES = ["diamond8_k", "diamond8_l", "diamond8_kc"]
FP64_TOL = 1e-10


def _rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b) / np.maximum(1.0, np.abs(b))))


def _phase_err(a, b):
    return float(np.max(np.abs(np.exp(1j * np.asarray(a)) - np.exp(1j * np.asarray(b)))))


@pytest.fixture(scope="module", params=NAMES)
def golden(request):
    g = dict(np.load(os.path.join(GOLDEN, request.param + ".npz")))
    return request.param, os.path.join(GOLDEN, request.param + ".qw"), g


def _check_sign(name, got, ref):
    if name in ("diamond8_k", "diamond8_kc"):
        assert _phase_err(got, ref) < 1e-9
    else:
        assert np.array_equal(got, ref)


def test_complex_kernels_selected(golden):
    name, deck, g = golden
    E = engine.Engine(deck, engine.FP64, max_walkers=4)
    assert E.info.complex_orbitals == 1


def test_eval_fp64_matches_reference(golden):
    name, deck, g = golden
    E = engine.Engine(deck, engine.FP64, max_walkers=len(g["R"]))
    E.set_walkers(g["R"])
    ev = E.eval(g["rot"])
    _check_sign(name, ev.sign, g["sign"])
    assert _rel(ev.logpsi, g["logpsi"]) < FP64_TOL
    assert _rel(ev.grad, g["grad"]) < FP64_TOL
    assert _rel(ev.lap, g["lap"]) < 1e-9
    assert _rel(ev.kinetic, g["kinetic"]) < 1e-9
    assert _rel(ev.potential, g["potential"]) < FP64_TOL
    assert _rel(ev.nonlocal_, g["nonlocal"]) < FP64_TOL


def test_ratio_fp64_matches_reference(golden):
    name, deck, g = golden
    E = engine.Engine(deck, engine.FP64, max_walkers=len(g["R"]))
    E.set_walkers(g["R"])
    for m in range(g["move_e"].shape[1]):
        dl, sg, gr, lp = E.ratio(g["move_e"][:, m], g["move_pos"][:, m])
        assert _rel(dl, g["move_dlogpsi"][:, m]) < FP64_TOL
        _check_sign(name, sg, g["move_sign"][:, m])
        assert _rel(gr, g["move_grad"][:, m]) < FP64_TOL
        assert _rel(lp, g["move_lap"][:, m]) < 1e-9


def test_mixed_precision_error_per_configuration(golden):
    name, deck, g = golden
    E = engine.Engine(deck, engine.MIXED, max_walkers=len(g["R"]))
    E.set_walkers(g["R"])
    ev = E.eval(g["rot"])
    el_ref = g["kinetic"] + g["potential"] + g["nonlocal"]
    err = np.abs(ev.energy - el_ref)
    dlp = np.abs(ev.logpsi - g["logpsi"])
    print(f"MIXED_ERROR {name}: |dE_L| median {np.median(err):.2e} max {err.max():.2e} Ha; "
          f"|d ln psi| median {np.median(dlp):.2e}")
    nelec = g["R"].shape[1]
    assert np.median(err) / nelec < 4e-6
    assert np.median(dlp) / nelec < 2e-7


def _strip_pseudo(src, dst_dir):
    import shutil
    text = open(src).read()
    out, i = [], 0
    while True:
        j = text.find("PSEUDO", i)
        if j < 0:
            out.append(text[i:])
            break
        out.append(text[i:j])
        k, depth = text.index("{", j), 0
        while True:
            depth += {"{": 1, "}": -1}.get(text[k], 0)
            k += 1
            if depth == 0:
                break
        i = k
    dst = os.path.join(dst_dir, os.path.basename(src))
    with open(dst, "w") as fh:
        fh.write("".join(out))
    shutil.copy(os.path.splitext(src)[0] + ".orb", dst_dir)
    return dst


@pytest.mark.parametrize("prec", [engine.FP64, engine.MIXED])
@pytest.mark.parametrize("name", NAMES)
def test_moves_track_state(name, prec, tmp_path):
    """After a VMC block of single-electron moves (complex Sherman-Morrison
    updates, electrons wrapped across the twisted boundaries), the local
    energy from the updated state equals a fresh evaluation at the final
    positions (bare Coulomb copy, so no quadrature rotation enters)."""
    deck = os.path.join(GOLDEN, name + ".qw")
    d = systems.read_deck(deck)
    bare = _strip_pseudo(deck, str(tmp_path))
    nw = 64
    E = engine.Engine(bare, prec, max_walkers=nw)
    E.set_walkers(systems.random_configs(d, nw, seed=31))
    s = E.vmc_block(4, 0.3, seed=32)
    assert s["nonfinite"] == 0 and 0.2 < s["acceptance"] <= 1.0
    e_moves = E.last_energies()
    E2 = engine.Engine(bare, engine.FP64, max_walkers=nw)
    E2.set_walkers(E.get_walkers())
    tol = 1e-8 if prec == engine.FP64 else 1e-3
    assert _rel(e_moves, E2.eval().energy) < tol


@pytest.mark.parametrize("name", NAMES)
def test_dmc_blocks_run(name):
    deck = os.path.join(GOLDEN, name + ".qw")
    d = systems.read_deck(deck)
    nw = 256
    E = engine.Engine(deck, engine.MIXED, max_walkers=nw)
    E.set_walkers(systems.random_configs(d, nw, seed=41))
    E.vmc_block(10, 0.3, seed=42)
    E.dmc_init(timestep=0.01, nstep=10, seed=43)
    for _ in range(2):
        st = E.dmc_block()
        assert np.isfinite(st["energy"]) and st["nonfinite"] == 0
        assert 0.2 < st["weight"] < 5.0


@pytest.mark.parametrize("deck_name", ["n2_pseudo", "diamond8"])
def test_complex_kernels_reproduce_real_orbitals(deck_name, tmp_path):
    """The same real orbitals read as CORBITALS (a molecule and a Gamma-point
    cell) run on the complex-orbital kernels and give the real kernels'
    values: phase 0 or pi, equal energies and ratios."""
    import shutil
    src = os.path.join(GOLDEN, deck_name + ".qw")
    shutil.copy(os.path.join(GOLDEN, deck_name + ".orb"), tmp_path)
    cdeck = tmp_path / (deck_name + ".qw")
    cdeck.write_text(open(src).read().replace("ORBITALS { BLAS_MO", "CORBITALS { BLAS_MO"))
    g = dict(np.load(os.path.join(GOLDEN, deck_name + ".npz")))
    nw = min(64, len(g["R"]))
    R, rot = g["R"][:nw], g["rot"][:nw]
    A = engine.Engine(src, engine.FP64, max_walkers=nw)
    B = engine.Engine(str(cdeck), engine.FP64, max_walkers=nw)
    assert A.info.complex_orbitals == 0 and B.info.complex_orbitals == 1
    A.set_walkers(R)
    B.set_walkers(R)
    ea, eb = A.eval(rot), B.eval(rot)
    assert _phase_err(eb.sign, np.where(ea.sign < 0, np.pi, 0.0)) < 1e-12
    for k in ("logpsi", "grad", "potential", "nonlocal_"):
        assert _rel(getattr(eb, k), getattr(ea, k)) < 1e-11, k
    for k in ("lap", "kinetic"):
        assert _rel(getattr(eb, k), getattr(ea, k)) < 1e-9, k
    dla, sga, gra, lpa = A.ratio(g["move_e"][:nw, 0], g["move_pos"][:nw, 0])
    dlb, sgb, grb, lpb = B.ratio(g["move_e"][:nw, 0], g["move_pos"][:nw, 0])
    assert _rel(dlb, dla) < 1e-11 and _rel(grb, gra) < 1e-11 and _rel(lpb, lpa) < 1e-9
    assert _phase_err(sgb, np.where(sga < 0, np.pi, 0.0)) < 1e-12
