"""Regenerate the golden vectors in tests/golden/ from the reference itself.

Run in a container that has the reference sources:
    make -C oracle REF=<reference checkout> -j8
    python tests/golden/make_golden.py

For each workload deck it draws seeded electron configurations, quadrature
rotations and single-electron moves, runs the reference harness
(oracle/_ref/qwref_harness, linked against the reference's own objects) and
stores inputs + outputs as <name>.npz next to the deck and .orb file.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from mainline_b200 import systems  # noqa: E402
import refrun  # noqa: E402

NCONF = 256
NMOVE = 2
WORKLOADS = [("n2_allelectron", dict(pseudo=False), 11), ("n2_pseudo", dict(pseudo=True), 12),
             ("diamond8", dict(periodic=True), 13), ("mol43", dict(nelec=43), 14),
             ("mol72", dict(nelec=72), 15), ("cell32", dict(periodic=True, supercell=(2, 2, 1)), 16),
             ("n2_multidet", dict(pseudo=True, expansion=[
                 (0.9, [1, 2, 3, 4, 5, 6, 7], [1, 2, 3, 4, 5, 6, 7]),
                 (-0.25, [1, 2, 3, 4, 5, 6, 8], [1, 2, 3, 4, 5, 6, 7]),
                 (-0.25, [1, 2, 3, 4, 5, 6, 7], [1, 2, 3, 4, 5, 6, 8]),
                 (0.12, [1, 2, 3, 4, 5, 6, 8], [1, 2, 3, 4, 5, 6, 8]),
                 (0.08, [1, 2, 3, 4, 5, 7, 9], [1, 2, 3, 4, 5, 6, 7]),
                 (0.08, [1, 2, 3, 4, 5, 6, 7], [1, 2, 3, 4, 5, 7, 9]),
                 (-0.05, [1, 2, 3, 4, 6, 8, 9], [2, 3, 4, 5, 6, 7, 8])]), 17),
             # twisted boundary conditions: complex orbitals at a general k-point,
             # and real orbitals at an integer (antiperiodic) k-point
             ("diamond8_k", dict(periodic=True, kpoint=(0.5, 0.25, 0.0), complex_orbitals=True), 18),
             ("diamond8_l", dict(periodic=True, kpoint=(1.0, 1.0, 1.0)), 19),
             # F and G shells: every angular order (molecule) and 7F_crystal in a cell
             ("n2_fg", dict(pseudo=True, high_l=True), 20),
             ("diamond8_f", dict(periodic=True, high_l=True), 21),
             # a Slater wave function alone, its BASIS section given twice
             ("n2_slater", dict(pseudo=True, jastrow=False, dup_basis=True), 22),
             # the CUTOFF_MO evaluator: a molecule and a complex k-point cell
             ("n2_cutoff", dict(pseudo=True, mo_kind="CUTOFF_MO"), 23),
             ("diamond8_kc", dict(periodic=True, kpoint=(0.5, 0.25, 0.0), complex_orbitals=True,
                                  mo_kind="CUTOFF_MO"), 24),
             # PADE Jastrow basis, THREEBODY_SPIN on SM_TERMS, 18-point quadrature
             ("n2_jas", dict(pseudo=True, jastrow_variant="pade_spin", aip=18), 25),
             # the 26- and 32-point quadratures
             ("n2_aip26", dict(pseudo=True, aip=26), 26),
             ("n2_aip32", dict(pseudo=True, aip=32), 27),
             # SPIN_DEP radial sets per spin, with ADD_ZEFF
             ("n2_ppspin", dict(pseudo=True, pp_variant="spin_dep"), 28)]


def make(name, kw, seed):
    if kw.get("periodic"):
        sc = kw.get("supercell", (1, 1, 1))
        deck = systems.write_periodic(HERE, seed=seed, name=name, supercell=sc, kpoint=kw.get("kpoint"),
                                      complex_orbitals=kw.get("complex_orbitals", False),
                                      high_l=kw.get("high_l", False), mo_kind=kw.get("mo_kind", "BLAS_MO"))
        nconf = 64 if sc == (1, 1, 1) else 16
    elif "nelec" in kw:  # molecules of the batched-uneven workload (odd count; above 32 per spin)
        deck = systems.write_molecule(HERE, name, seed, kw["nelec"])
        nconf = 64 if kw["nelec"] < 64 else 32
    else:
        deck = systems.write_n2(HERE, seed=seed, name=name, **kw)
        nconf = NCONF if not ({"expansion", "high_l", "jastrow", "mo_kind", "aip", "pp_variant"} & set(kw)) else 64
    R = systems.random_configs(deck, nconf, seed=seed + 1000)
    NCONF_ = nconf
    rng = np.random.default_rng(seed + 2000)
    rot = np.stack([systems.random_rotation(rng) for _ in range(NCONF_)])
    me = rng.integers(0, deck.nelec, size=(NCONF_, NMOVE)).astype(np.int32)
    mp = R[np.arange(NCONF_)[:, None], me] + rng.normal(0.0, 0.4, size=(NCONF_, NMOVE, 3))
    out = refrun.run_harness(deck.path, R, rot, me, mp)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), R=R, rot=rot, move_e=me, move_pos=mp, **out)
    print(name, "logpsi[:3]", out["logpsi"][:3])


if __name__ == "__main__":
    if not refrun.harness_available():
        sys.exit("build the reference harness first: make -C oracle REF=<reference> -j8")
    only = set(sys.argv[1:])
    for name, kw, seed in WORKLOADS:
        if not only or name in only:
            make(name, kw, seed)
