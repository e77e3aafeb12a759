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


def _vmc_depth1(deck, R0, tc):
    old = os.environ.get("QWG_TC_MOVES")
    os.environ["QWG_TC_MOVES"] = "1" if tc else "0"
    try:
        E = engine.Engine(deck, engine.MIXED, max_walkers=len(R0))
    finally:
        if old is None:
            del os.environ["QWG_TC_MOVES"]
        else:
            os.environ["QWG_TC_MOVES"] = old
    E.set_vmc_dynamics(1, 2.0)
    E.set_walkers(R0)
    st = E.vmc_block(2, 0.1, seed=7)
    R = E.get_walkers()
    E.close()
    return st, R


@pytest.mark.parametrize("name", ["mol72", "cell32"])
def test_tensor_core_moves_follow_cuda_core_moves(name):
    """The per-electron tensor-core move schedule (proposal + basis rows,
    one GEMM over all walkers, decision + Sherman-Morrison update) walks the
    same paths as the one-launch CUDA-core sweep from the same walkers and
    random streams: only decisions within the ~1e-6 difference of the MO
    values can differ, and positions follow to the precision of the drift.""" 
    deck = os.path.join(GOLDEN, name + ".qw")
    d = systems.read_deck(deck)
    R0 = systems.random_configs(d, 1024, seed=11)  # the schedule runs from 1024 walkers
    st_tc, R_tc = _vmc_depth1(deck, R0, True)
    st_cc, R_cc = _vmc_depth1(deck, R0, False)
    # the drift of later moves uses gradients from either contraction, so
    # positions of the same decisions agree to ~1e-7 bohr, not bit for bit
    dev = np.max(np.abs(R_tc - R_cc), axis=-1)
    same = dev < 1e-3  # a different decision moves an electron by ~sqrt(tau) = 0.3 bohr
    print(f"TC_MOVES {name}: {100 * same.mean():.2f}% of electrons within 1e-3 bohr (median deviation "
          f"{np.median(dev):.1e}), acceptance "
          f"{st_tc['acceptance']:.4f} (tensor cores) vs {st_cc['acceptance']:.4f}, energy {st_tc['energy']:.4f} vs "
          f"{st_cc['energy']:.4f}")
    assert same.mean() > 0.99
    assert np.median(dev) < 1e-4
    assert abs(st_tc["acceptance"] - st_cc["acceptance"]) < 0.005
    assert np.isfinite(st_tc["energy"])


def test_tensor_core_moves_dmc_block():
    deck = os.path.join(GOLDEN, "cell32.qw")
    d = systems.read_deck(deck)
    E = engine.Engine(deck, engine.MIXED, max_walkers=1024)
    E.set_walkers(systems.random_configs(d, 1024, seed=12))
    E.vmc_block(2, 0.3, seed=1)
    E.dmc_init(timestep=0.005, nstep=5, seed=3)
    for _ in range(2):
        s = E.dmc_block()
        assert np.isfinite(s["energy"]) and s["nonfinite"] == 0
        assert 0.9 < s["acceptance"] <= 1.0
    E.close()
