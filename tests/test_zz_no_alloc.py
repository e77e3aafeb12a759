"""The allocation-free VMC block (qwg_vmc_block_noalloc) against the regular
one (qwg_vmc_block), called through the C-ABI.

qwg_vmc_block_noalloc exists for callers that must not allocate device memory
while they run (a serving loop that has divided HBM among its jobs, a host
inside another allocator's budget, code that must not trigger the device-wide
synchronisation of cudaMalloc/cudaFree).  Its walker state and accumulators
live in one fixed 16 MiB device array of the library instead of buffers the
context allocates.  Both entry points run the same kernel on the same seeded
walkers, so two calls in a row must give the same positions, per-walker
energies and block sums (tolerance 1e-12 relative: only the order of the
accumulators' atomic additions may differ).

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import GOLDEN
from mainline_b200 import engine, systems

pytestmark = pytest.mark.gpu

NW, NSTEP, TAU, SEED = 192, 4, 0.3, 4242


def _rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b) / np.maximum(1.0, np.abs(b))))


def _compare_two_calls(deck, d, nw, precision, tol):
    import torch
    R0 = systems.random_configs(d, nw, seed=5)

    # regular entry point: context-owned device buffers
    A = engine.Engine(deck, precision, max_walkers=nw)
    A.set_walkers(R0)
    ref = []
    for call in range(2):
        st = A.vmc_block(NSTEP, TAU, seed=SEED + call)
        ref.append((A.get_walkers(), st))
    A.close()

    # allocation-free entry point: the caller's device buffers, fixed scratch
    stream = torch.cuda.current_stream()
    B = engine.Engine(deck, precision, max_walkers=nw, stream=stream.cuda_stream)
    lib = engine.load_library()
    dR = torch.tensor(R0, dtype=torch.float64, device="cuda")
    dE = torch.zeros(nw, dtype=torch.float64, device="cuda")
    dS = torch.zeros(10, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    for call in range(2):
        rc = lib.qwg_vmc_block_noalloc(B.h, C.c_void_p(dR.data_ptr()), nw, NSTEP, TAU, SEED + call, 0,
                                       C.c_void_p(dE.data_ptr()), C.c_void_p(dS.data_ptr()))
        assert rc == 0, lib.qwg_last_error(B.h).decode()
        torch.cuda.synchronize()
        R_ref, st = ref[call]
        sums = dS.cpu().numpy()
        assert _rel(dR.cpu().numpy(), R_ref) < tol
        assert _rel(sums[1] / sums[0], st["energy"]) < tol
        assert _rel(sums[2] / sums[0], st["kinetic"]) < tol
        assert _rel(sums[6] / sums[7], st["acceptance"]) < tol
        assert np.all(np.isfinite(dE.cpu().numpy()))
    B.close()


def test_noalloc_matches_regular_block_two_calls():
    deck = os.path.join(GOLDEN, "n2_pseudo.qw")
    d = systems.Deck(deck, "", 7, 7, 2, 80, "n2_pseudo", 0)
    _compare_two_calls(deck, d, NW, engine.FP64, 1e-12)


@pytest.mark.parametrize("precision", [engine.FP64, engine.MIXED])
def test_noalloc_hbm_resident_system(precision):
    """72 electrons (36 orbitals per spin) run on the HBM-resident kernels,
    whose per-walker scratch region also lives in the fixed array, after the
    walker states."""
    deck = os.path.join(GOLDEN, "mol72.qw")
    d = systems.read_deck(deck)
    # mixed precision: the same kernels in FP32; atomics may reorder sums
    _compare_two_calls(deck, d, 24, precision, 1e-12 if precision == engine.FP64 else 1e-9)


def test_noalloc_limit_is_exact_for_hbm_resident_system():
    """The largest population the error message names runs; one more walker
    is rejected."""
    import re
    import torch
    deck = os.path.join(GOLDEN, "mol72.qw")
    d = systems.read_deck(deck)
    B = engine.Engine(deck, engine.MIXED, max_walkers=8)
    lib = engine.load_library()
    dS = torch.zeros(10, dtype=torch.float64, device="cuda")
    rc = lib.qwg_vmc_block_noalloc(B.h, C.c_void_p(dS.data_ptr()), 1 << 20, 1, TAU, 1, 0, None,
                                   C.c_void_p(dS.data_ptr()))
    assert rc == -1
    maxw = int(re.search(r"at most (\d+) walkers", lib.qwg_last_error(B.h).decode()).group(1))
    assert 1 <= maxw < 1 << 20
    dR = torch.tensor(systems.random_configs(d, maxw + 1, seed=7), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = lib.qwg_vmc_block_noalloc(B.h, C.c_void_p(dR.data_ptr()), maxw + 1, 1, TAU, 1, 0, None,
                                   C.c_void_p(dS.data_ptr()))
    assert rc == -1
    rc = lib.qwg_vmc_block_noalloc(B.h, C.c_void_p(dR.data_ptr()), maxw, 1, TAU, 1, 0, None,
                                   C.c_void_p(dS.data_ptr()))
    assert rc == 0, lib.qwg_last_error(B.h).decode()
    torch.cuda.synchronize()
    sums = dS.cpu().numpy()
    assert sums[0] > 0 and np.isfinite(sums[1] / sums[0])
    B.close()


def test_noalloc_rejects_population_beyond_scratch():
    import torch
    deck = os.path.join(GOLDEN, "n2_pseudo.qw")
    B = engine.Engine(deck, engine.FP64, max_walkers=8)
    lib = engine.load_library()
    big = 1 << 20  # one million walkers of ~5 kB state cannot fit in 16 MiB
    dummy = torch.zeros(16, dtype=torch.float64, device="cuda")
    rc = lib.qwg_vmc_block_noalloc(B.h, C.c_void_p(dummy.data_ptr()), big, 1, TAU, 1, 0, None,
                                   C.c_void_p(dummy.data_ptr()))
    assert rc == -1
    msg = lib.qwg_last_error(B.h).decode()
    assert "scratch" in msg and "at most" in msg
    B.close()
