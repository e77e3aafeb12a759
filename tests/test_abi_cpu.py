"""CPU-side checks of the C-ABI library: it loads without a GPU, exports every
symbol include/*.h declares, and its host table builder (deck parser +
spline fit) reproduces the oracle's tables."""
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
import qworacle
from mainline_b200 import engine

HEADERS = [os.path.join(ROOT, "include", h) for h in sorted(os.listdir(os.path.join(ROOT, "include")))
           if h.endswith(".h")]


def _declared():
    txt = "".join(open(h).read() for h in HEADERS)
    return sorted(set(re.findall(r"\b(qwg_[a-z_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(engine.LIB_PATH):
        from mainline_b200 import build
        build.build()
    return engine.load_library()


def test_exports_every_declared_symbol(lib):
    names = _declared()
    assert set(names) == set(engine.EXPORTS)
    for n in names:
        assert hasattr(lib, n), n


def test_version(lib):
    assert b"sm_100a" in lib.qwg_version()


@pytest.mark.parametrize("name", ["n2_allelectron", "n2_pseudo"])
def test_inspect_deck(lib, name):
    info = engine.inspect_deck(os.path.join(GOLDEN, name + ".qw"))
    assert (info.nelec, info.nup, info.ndown, info.natoms, info.nbasis) == (14, 7, 7, 2, 80)
    assert info.nshell == 36
    assert info.has_pseudo == (name == "n2_pseudo")


def test_spline_tables_match_oracle(lib):
    deck = os.path.join(GOLDEN, "n2_pseudo.qw")
    S = qworacle.System(deck)
    shells = [(b, k) for b in S.center_basis[0] for k in range(len(b.syms))]
    for sh, (b, k) in enumerate(shells):
        coef, spacing, cut = engine.inspect_spline(deck, sh)
        ref = b.coeffs[k]
        assert spacing == b.spacing
        assert cut == b.threshold
        # rounding-level differences (tridiagonal solve order)
        np.testing.assert_allclose(coef[:len(ref)], ref, rtol=1e-7, atol=1e-12 * np.abs(ref).max())


def test_bad_deck_reports_error(lib, tmp_path):
    p = tmp_path / "bad.qw"
    p.write_text("SYSTEM { MOLECULE NSPIN { 1 0 } ATOM { H 1 COOR 0 0 0 } }\nTRIALFUNC { JASTROW2 }\n")
    with pytest.raises(engine.QwgError, match="SLATER-JASTROW or SLATER"):
        engine.inspect_deck(str(p))


@pytest.mark.parametrize("edit,msg", [
    (lambda t: t.replace("DETWT { 1.0 }", "DETWT { 0.9 0.1 }"), "every determinant"),
    (lambda t: t.replace("ORBITALS { BLAS_MO", "CORBITALS { BLAS_MO").replace("DETWT { 1.0 }", "DETWT { 0.9 0.1 }"),
     "real orbitals at the Gamma point"),
])
def test_unsupported_wavefunctions_are_rejected(lib, tmp_path, edit, msg):
    """Malformed determinant expansions and expansions of complex orbitals
    (outside this engine) are rejected with a clear message, not run wrongly."""
    import shutil
    src = os.path.join(GOLDEN, "n2_pseudo.qw")
    shutil.copy(os.path.join(GOLDEN, "n2_pseudo.orb"), tmp_path)
    text = open(src).read()
    assert "DETWT { 1.0 }" in text and "ORBITALS { BLAS_MO" in text
    p = tmp_path / "x.qw"
    p.write_text(edit(text))
    with pytest.raises(engine.QwgError, match=msg):
        engine.inspect_deck(str(p))


def test_complex_orbitals_are_recognised(lib, tmp_path):
    """CORBITALS (complex coefficients, "(re,im)" or plain reals) and a nonzero
    KPOINT select the complex-orbital kernels."""
    import shutil
    src = os.path.join(GOLDEN, "n2_pseudo.qw")
    shutil.copy(os.path.join(GOLDEN, "n2_pseudo.orb"), tmp_path)
    p = tmp_path / "c.qw"
    p.write_text(open(src).read().replace("ORBITALS { BLAS_MO", "CORBITALS { BLAS_MO"))
    assert engine.inspect_deck(str(p)).complex_orbitals == 1
    assert engine.inspect_deck(src).complex_orbitals == 0
    assert engine.inspect_deck(os.path.join(GOLDEN, "diamond8_k.qw")).complex_orbitals == 1
    assert engine.inspect_deck(os.path.join(GOLDEN, "diamond8_l.qw")).complex_orbitals == 1
    assert engine.inspect_deck(os.path.join(GOLDEN, "diamond8.qw")).complex_orbitals == 0
