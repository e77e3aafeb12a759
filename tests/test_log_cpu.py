"""QWalk log output without a GPU: the engine's block entries have the keys,
order and number format of the reference's own log (checked against a log
written by the reference qwalk built from source), and the reference's
gosling analyser reads them back to the same averages."""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
from mainline_b200 import engine

REF = os.path.join(ROOT, "oracle", "_ref")
QWALK = os.path.join(REF, "qwalk-Linux")
GOSLING = os.path.join(REF, "gosling")


def _blocks(text):
    return re.findall(r"block \{ \n(.*?)\n\} \n", text, flags=re.S)


def _keys(block):
    return [ln.split()[0] for ln in block.splitlines() if ln.strip()]


def _write(path, energies, npoints=1000):
    engine.log_header(path, "DMC", "dmc", 0.01)
    for e in energies:
        engine.log_block(path, "dmc", {"energy": e, "kinetic": 10.0, "potential": -25.0, "nonlocal": 3.0,
                                       "weight": 1.0, "npoints": npoints, "var_energy": 2.5, "var_kinetic": 3.0,
                                       "var_potential": 4.0, "var_nonlocal": 1.0, "var_weight": 0.0})


def test_log_block_format(tmp_path):
    p = str(tmp_path / "run.log")
    _write(p, [-12.25, -12.5])
    txt = open(p).read()
    assert txt.startswith("#-------------------------------------------------\n#DMC run: timestep 0.01\n")
    assert "init { \n   label dmc\n}\n" in txt
    bl = _blocks(txt)
    assert len(bl) == 2
    assert _keys(bl[0]) == ["label", "totweight", "nautocorr", "total_energy", "total_energyvar", "weight",
                            "weightvar", "kinetic_energy", "kinetic_energyvar", "potential_energy",
                            "potential_energyvar", "nonlocal_energy", "nonlocal_energyvar", "autocorr_energy"]
    assert "   total_energy { -12.25   } " in bl[0]


@pytest.mark.skipif(not os.path.exists(QWALK), reason="reference qwalk not built (make -C oracle)")
def test_log_matches_reference_layout(tmp_path):
    """Block entries have the same keys in the same order as the blocks the
    reference's own VMC writes for the same deck."""
    for f in ("n2_pseudo.qw", "n2_pseudo.orb"):
        shutil.copy(os.path.join(GOLDEN, f), tmp_path)
    deck = tmp_path / "n2_pseudo.qw"
    with open(deck, "a") as fh:
        fh.write("METHOD { VMC NCONFIG 8 NBLOCK 2 NSTEP 4 TIMESTEP 0.3 }\n")
    subprocess.run([QWALK, "n2_pseudo.qw"], cwd=tmp_path, capture_output=True, timeout=300, check=True)
    ref = open(str(deck) + ".log").read()
    rb = _blocks(ref)
    assert len(rb) == 2
    p = str(tmp_path / "engine.log")
    _write(p, [-12.0])
    ours = _blocks(open(p).read())[0]
    assert _keys(ours) == _keys(rb[0])
    # each line has the reference's shape ("key { value   } ")
    for a, b in zip(ours.splitlines(), rb[0].splitlines()):
        assert re.sub(r"-?[0-9][0-9.e+-]*", "N", a).replace("dmc", "L") == \
            re.sub(r"-?[0-9][0-9.e+-]*", "N", b).replace("vmc", "L")


@pytest.mark.skipif(not os.path.exists(GOSLING), reason="reference gosling not built (make -C oracle)")
def test_gosling_reads_engine_log(tmp_path):
    rng = np.random.default_rng(3)
    e = -12.0 + rng.normal(0.0, 0.05, size=8)
    p = str(tmp_path / "run.log")
    _write(p, e)
    out = subprocess.run([GOSLING, "-no_equil", p], capture_output=True, text=True, timeout=60, check=True).stdout
    m = re.search(r"total_energy0\s+(\S+)\s+\+/-\s+(\S+)", out)
    assert m, out
    assert abs(float(m.group(1)) - e.mean()) < 1e-7  # gosling prints 10 significant digits
    assert "8 total blocks" in out
