"""Batched MO evaluation (qwg_mo_eval) through the C-ABI.

FP64 contexts contract on CUDA cores and must match the oracle's
MO_matrix_blas::updateLap restatement at 1e-10.  Mixed-precision contexts
contract every position in one tensor-core GEMM (tcgen05 kind::tf32 with
split TF32 operands, FP32 accumulation, TMA-staged tiles): each value,
gradient and Laplacian must match FP64 within 1e-5 of the largest orbital
component at that position (measured ~1e-7).  The position counts make the
GEMM's row count (5 per position) cover several 128-row tiles with a
partial last one; the decks span 2 to 128 orbitals per spin (UMMA N = 16 ..
128) and 24 to 832 basis functions (1 to 26 K chunks)."""
import os
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN
import qworacle
from mainline_b200 import engine, systems

pytestmark = pytest.mark.gpu


def _positions(deck, n, seed):
    d = systems.read_deck(deck)
    R = systems.random_configs(d, (n + d.nelec - 1) // d.nelec, seed=seed)
    return R.reshape(-1, 3)[:n]


@pytest.mark.parametrize("name", ["n2_pseudo", "diamond8", "mol43"])
def test_mo_eval_fp64_matches_oracle(name):
    deck = os.path.join(GOLDEN, name + ".qw")
    S = qworacle.System(deck)
    P = _positions(deck, 64, 3)
    if S.periodic:
        P = S.wrap(P[None])[0]
    ref = S.mo_lap(P)
    E = engine.Engine(deck, engine.FP64, max_walkers=1)
    nup, ndn = E.info.nmo_up, E.info.nmo_down
    for s, cols in ((0, slice(0, nup)), (1, slice(nup, nup + ndn))):
        got = E.mo_eval(P, s)
        r = ref[:, cols]
        assert np.max(np.abs(got - r) / np.maximum(1.0, np.abs(r))) < 1e-10
    E.close()


def _tc_vs_fp64(deck, npos, seed=5):
    P = _positions(deck, npos, seed)
    F = engine.Engine(deck, engine.FP64, max_walkers=1)
    M = engine.Engine(deck, engine.MIXED, max_walkers=1)
    worst = 0.0
    for s in (0, 1):
        f = F.mo_eval(P, s)
        m = M.mo_eval(P, s)
        scale = np.maximum(1.0, np.max(np.abs(f), axis=1, keepdims=True))
        err = float(np.max(np.abs(m - f) / scale))
        print(f"TC_MO {os.path.basename(deck)} spin {s}: {npos} positions x {f.shape[1]} orbitals, "
              f"max error {err:.2e} of the largest component")
        worst = max(worst, err)
    F.close()
    M.close()
    return worst


@pytest.mark.parametrize("name", ["n2_pseudo", "mol72", "diamond8", "cell32", "h4pp"])
def test_mo_eval_tensor_cores_match_fp64(name):
    assert _tc_vs_fp64(os.path.join(GOLDEN, name + ".qw"), 333) < 1e-5


def test_mo_eval_tensor_cores_64_atom_cell():
    """The 64-atom cell: 128 orbitals per spin (UMMA N = 128, three-stage
    ring), 832 basis functions (26 K chunks)."""
    tmp = tempfile.mkdtemp(prefix="qwg_tc_")
    deck = systems.write_periodic(tmp, seed=99, name="cell64", supercell=(2, 2, 2)).path
    assert _tc_vs_fp64(deck, 200) < 1e-5


def test_mo_eval_rejects_bad_arguments():
    E = engine.Engine(os.path.join(GOLDEN, "n2_pseudo.qw"), engine.MIXED, max_walkers=1)
    with pytest.raises(engine.QwgError):
        E.mo_eval(np.zeros((4, 3)), 2)
    E.close()
