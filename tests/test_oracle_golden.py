"""Pin the numpy oracle against golden vectors written by the reference
itself (tests/golden/make_golden.py ran the reference harness)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
import qworacle

NAMES = ["n2_allelectron", "n2_pseudo", "diamond8", "mol43", "mol72", "cell32", "diamond8_k", "diamond8_l", "n2_fg",
         "diamond8_f", "n2_slater", "n2_cutoff", "diamond8_kc", "n2_jas", "n2_aip26", "n2_aip32", "n2_ppspin"]


def _rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b) / np.maximum(1.0, np.abs(b))))


@pytest.fixture(scope="module", params=NAMES)
def case(request):
    g = dict(np.load(os.path.join(GOLDEN, request.param + ".npz")))
    # the restatement is slow in numpy for the periodic and the large decks
    keep = {"diamond8": 8, "mol72": 4, "cell32": 2, "diamond8_k": 6, "diamond8_l": 6, "n2_fg": 32,
            "diamond8_f": 6, "n2_cutoff": 32, "diamond8_kc": 4, "n2_jas": 16, "n2_aip26": 8,
            "n2_aip32": 8, "n2_ppspin": 16}.get(request.param)
    if keep:
        g = {k: v[:keep] for k, v in g.items()}
    return request.param, qworacle.System(os.path.join(GOLDEN, request.param + ".qw")), g


def _same_sign(S, got, ref):
    """Signs, or phases (complex orbitals) compared as unit complex numbers."""
    if S.cplx:
        return float(np.max(np.abs(np.exp(1j * got) - np.exp(1j * ref)))) < 1e-10
    return np.array_equal(got, ref)


def test_evaluate_matches_reference(case):
    name, S, g = case
    ev = S.evaluate(g["R"])
    assert _same_sign(S, ev["sign"], g["sign"])
    assert _rel(ev["logpsi"], g["logpsi"]) < 1e-12
    assert _rel(ev["grad"], g["grad"]) < 1e-10
    # Laplacians near the nuclei are large (|lap| up to ~1e4): relative bound
    assert np.max(np.abs(ev["lap"] - g["lap"]) / np.maximum(1.0, np.abs(g["lap"]))) < 1e-9
    assert _rel(ev["kinetic"], g["kinetic"]) < 1e-9
    assert _rel(ev["potential"], g["potential"]) < 1e-12


def test_moves_match_reference(case):
    name, S, g = case
    for m in range(g["move_e"].shape[1]):
        dl, sg, gr, lp = S.move_ratio(g["R"], g["move_e"][:, m], g["move_pos"][:, m])
        assert _rel(dl, g["move_dlogpsi"][:, m]) < 1e-11
        assert _same_sign(S, sg, g["move_sign"][:, m])
        assert _rel(gr, g["move_grad"][:, m]) < 1e-10
        assert _rel(lp, g["move_lap"][:, m]) < 1e-9


def test_nonlocal_matches_reference(case):
    name, S, g = case
    if not S.pp:
        pytest.skip("all-electron deck")
    if S.periodic:
        pytest.skip("periodic V_NL in numpy takes minutes per configuration; the GPU engine is pinned to the "
                    "golden V_NL directly (checked once by hand: 6.8e-14 relative)")
    if S.nelec > 64:
        pytest.skip("numpy V_NL above 64 electrons takes minutes per configuration; the GPU engine is pinned to "
                    "the golden V_NL of this deck directly")
    n = 4 if S.nelec > 32 else 32  # numpy V_NL costs ~16 s per configuration at 43 electrons
    nl = S.nonlocal_pp(g["R"][:n], g["rot"][:n])
    assert _rel(nl, g["nonlocal"][:n]) < 1e-11
