"""Walker configuration files without a GPU: the engine's writer and reader
round-trip, read files the reference qwalk wrote (STORECONFIG), and the
reference qwalk restarts VMC and DMC runs from files the engine wrote
(READCONFIG)."""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
from mainline_b200 import engine, systems

QWALK = os.path.join(ROOT, "oracle", "_ref", "qwalk-Linux")
needs_ref = pytest.mark.skipif(not os.path.exists(QWALK), reason="reference qwalk not built (make -C oracle)")


def _parse(path):
    """Independent reader: the numbers after each 'nElec N ndim 3'."""
    toks = open(path).read().split()
    out = []
    for i, t in enumerate(toks):
        if t == "nElec":
            n = int(toks[i + 1])
            out.append(np.array([float(x) for x in toks[i + 4:i + 4 + 3 * n]]).reshape(n, 3))
    return np.array(out)


def test_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    R = rng.normal(size=(5, 14, 3)) * 3
    w = rng.uniform(0.2, 3.0, size=5)
    sg = np.array([1.0, -1.0, 1.0, 1.0, -1.0])
    p = str(tmp_path / "run.config")
    engine.write_configs(p, R, w, sg)
    R2, w2, s2 = engine.read_configs(p)
    assert np.allclose(R2, R, rtol=1e-14, atol=1e-14) and np.allclose(w2, w, rtol=1e-14)
    assert np.array_equal(s2, sg)
    engine.write_configs(p, R)  # VMC layout; the DMC file becomes the backup
    assert os.path.exists(p + ".backup")
    R3, w3, s3 = engine.read_configs(p)
    assert np.allclose(R3, R, rtol=1e-14) and np.all(w3 == 1.0) and np.all(s3 == 1.0)
    assert "DMC" not in open(p).read()


def test_rejects_malformed(tmp_path):
    p = tmp_path / "bad.config"
    p.write_text(" walker { \nnElec 2 ndim 3\n0 0 0\n1 1\n } \n")
    with pytest.raises(engine.QwgError):
        engine.read_configs(str(p))


def _deck(tmp_path, method):
    for f in ("n2_pseudo.qw", "n2_pseudo.orb"):
        shutil.copy(os.path.join(GOLDEN, f), tmp_path)
    deck = tmp_path / "n2_pseudo.qw"
    with open(deck, "a") as fh:
        fh.write(method + "\n")
    return deck


@needs_ref
def test_reads_reference_configs(tmp_path):
    deck = _deck(tmp_path, "METHOD { VMC NCONFIG 6 NBLOCK 1 NSTEP 3 TIMESTEP 0.3 STORECONFIG ref.config }")
    subprocess.run([QWALK, deck.name], cwd=tmp_path, capture_output=True, timeout=300, check=True)
    R, w, s = engine.read_configs(str(tmp_path / "ref.config"))
    assert R.shape == (6, 14, 3)
    assert np.array_equal(R, _parse(str(tmp_path / "ref.config")))


@needs_ref
@pytest.mark.parametrize("method", ["VMC", "DMC"])
def test_reference_restarts_from_engine_configs(tmp_path, method):
    d = systems.read_deck(os.path.join(GOLDEN, "n2_pseudo.qw"))
    R = systems.random_configs(d, 8, seed=5)
    if method == "DMC":
        engine.write_configs(str(tmp_path / "eng.config"), R, np.full(8, 1.0), np.ones(8))
        meth = "METHOD { DMC NCONFIG 8 NBLOCK 1 NSTEP 4 TIMESTEP 0.01 READCONFIG eng.config STORECONFIG out.config }"
    else:
        engine.write_configs(str(tmp_path / "eng.config"), R)
        meth = "METHOD { VMC NCONFIG 8 NBLOCK 1 NSTEP 4 TIMESTEP 0.3 READCONFIG eng.config STORECONFIG out.config }"
    deck = _deck(tmp_path, meth)
    r = subprocess.run([QWALK, deck.name], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "Read took" in r.stdout  # read_configurations ran on the engine's file
    log = open(str(deck) + ".log").read()
    m = re.findall(r"total_energy \{ (\S+)", log)
    assert len(m) == 1 and np.isfinite(float(m[0]))
    R2, w2, _ = engine.read_configs(str(tmp_path / "out.config"))
    assert R2.shape == (8, 14, 3)
