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


def test_noalloc_matches_regular_block_two_calls():
    import torch
    deck = os.path.join(GOLDEN, "n2_pseudo.qw")
    d = systems.Deck(deck, "", 7, 7, 2, 80, "n2_pseudo", 0)
    R0 = systems.random_configs(d, NW, seed=5)

    # regular entry point: context-owned device buffers
    A = engine.Engine(deck, engine.FP64, max_walkers=NW)
    A.set_walkers(R0)
    ref = []
    for call in range(2):
        st = A.vmc_block(NSTEP, TAU, seed=SEED + call)
        ref.append((A.get_walkers(), st))
    A.close()

    # allocation-free entry point: the caller's device buffers, fixed scratch
    stream = torch.cuda.current_stream()
    B = engine.Engine(deck, engine.FP64, max_walkers=NW, stream=stream.cuda_stream)
    lib = engine.load_library()
    dR = torch.tensor(R0, dtype=torch.float64, device="cuda")
    dE = torch.zeros(NW, dtype=torch.float64, device="cuda")
    dS = torch.zeros(10, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    for call in range(2):
        rc = lib.qwg_vmc_block_noalloc(B.h, C.c_void_p(dR.data_ptr()), NW, NSTEP, TAU, SEED + call, 0,
                                       C.c_void_p(dE.data_ptr()), C.c_void_p(dS.data_ptr()))
        assert rc == 0, lib.qwg_last_error(B.h).decode()
        torch.cuda.synchronize()
        R_ref, st = ref[call]
        sums = dS.cpu().numpy()
        assert _rel(dR.cpu().numpy(), R_ref) < 1e-12
        assert _rel(sums[1] / sums[0], st["energy"]) < 1e-12
        assert _rel(sums[2] / sums[0], st["kinetic"]) < 1e-12
        assert _rel(sums[6] / sums[7], st["acceptance"]) < 1e-12
        assert np.all(np.isfinite(dE.cpu().numpy()))
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
