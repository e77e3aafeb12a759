"""Seeded synthetic QWalk input decks for the walker-engine workloads.

Every deck is a plain QWalk input file (SYSTEM / PSEUDO / TRIALFUNC / METHOD
sections, same grammar as the reference's ``qmc_io.cpp`` parser) plus the
``.orb`` file its ORBITALS section names.  The same files drive the reference
CPU build and this engine, so both sides read byte-identical inputs.

Workloads (sizes are fixed; only the seed varies):

* ``n2_allelectron``  two Z=7 atoms at z=+-1.0375 bohr, 14 electrons (7 up,
  7 down); 40 contracted Cartesian Gaussians per atom (10 S + 6 P + 2 6D
  shells, 3 primitives each, exponents log-uniform in [0.1, 1e4]); a random
  orthonormal 80x7 MO block per spin; Jastrow = CUTOFF_CUSP e-e (GAMMA 24,
  like 0.25 / unlike 0.5 cusp) + POLYPADE e-n (BETA0 1.2, 4 functions,
  coefficients ~N(0, 0.1)).
* ``n2_pseudo``  the same molecule and electrons with each nucleus replaced by
  a Z_eff=5 semilocal RGAUSSIAN pseudopotential: l=0 and l=1 nonlocal
  channels (3 Gaussians each, exponents U[1,10], coefficients U(-5,5)) plus a
  local channel whose Z_eff/r Gaussian cancels the ion's -Z_eff/r at the
  nucleus; 12-point quadrature (AIP 12).  Same shell structure (40 functions
  per atom) with valence exponents log-uniform in [0.1, 10].
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

SHELL_NFUNC = {"S": 1, "P": 3, "5D": 5, "6D": 6, "7F": 7, "10F": 10, "7F_crystal": 7, "9G": 9, "15G": 15}


@dataclass
class Deck:
    """Paths and sizes of one generated system."""
    path: str               # QWalk input file
    orb_path: str
    nup: int
    ndown: int
    natoms: int
    nbasis: int             # basis functions (all centers)
    kind: str
    seed: int
    extra: dict = field(default_factory=dict)

    @property
    def nelec(self) -> int:
        return self.nup + self.ndown


def _fmt(x: float) -> str:
    return repr(float(x))


def _basis_shells(rng, nshell: dict, nprim=3, lo=0.1, hi=1e4):
    shells = []
    for sym in nshell:
        for _ in range(nshell[sym]):
            ex = np.exp(rng.uniform(np.log(lo), np.log(hi), size=nprim))
            co = rng.uniform(0.1, 1.0, size=nprim)
            shells.append((sym, ex, co))
    return shells


def _basis_text(label: str, shells, cutoff=None, normtype=None) -> str:
    lines = [f"BASIS {{ {label}", "AOSPLINE"]
    if normtype is not None:
        lines.append(f"NORMTYPE {normtype}")
    if cutoff is not None:
        lines.append(f"CUTOFF {_fmt(cutoff)}")
    lines.append("GAMESS {")
    for sym, ex, co in shells:
        lines.append(f"{sym} {len(ex)}")
        for i, (e, c) in enumerate(zip(ex, co)):
            lines.append(f"  {i + 1} {_fmt(e)} {_fmt(c)}")
    lines.append("}")
    lines.append("}")
    return "\n".join(lines)


def _random_orthonormal(rng, nb: int, nmo: int) -> np.ndarray:
    q, r = np.linalg.qr(rng.standard_normal((nb, nmo)))
    return q * np.sign(np.diag(r))[None, :]


def _write_orb(path: str, coeff: np.ndarray, nfunc_per_center: list[int]) -> None:
    """ORB file: ``mo basis center label`` lines (1-based), COEFFICIENTS, then
    the coefficient list (format read by readorb_noexpand, MO_matrix.h:264-332).
    ``coeff`` is [totbasis, nmo] with basis functions ordered center by center;
    complex coefficients are written as ``(re,im)`` (the stream format of a
    complex number, read by the CORBITALS path)."""
    nb, nmo = coeff.shape
    lines = []
    vals = []
    label = 0
    for mo in range(nmo):
        row = 0
        for c, nf in enumerate(nfunc_per_center):
            for f in range(nf):
                label += 1
                lines.append(f"{mo + 1} {f + 1} {c + 1} {label}")
                vals.append(coeff[row, mo])
                row += 1
    with open(path, "w") as fh:
        fh.write("\n".join(lines))
        fh.write("\nCOEFFICIENTS\n")
        if np.iscomplexobj(coeff):
            for i in range(0, len(vals), 4):
                fh.write(" ".join(f"({float(v.real)!r},{float(v.imag)!r})" for v in vals[i:i + 4]) + "\n")
        else:
            for i in range(0, len(vals), 4):
                fh.write(" ".join(repr(float(v)) for v in vals[i:i + 4]) + "\n")


def _jastrow_text(label: str, onebody: np.ndarray, threebody=None, twobody_pp=None) -> str:
    g2 = [
        "GROUP {",
        f"  EIBASIS {{ {label} POLYPADE BETA0 1.2 NFUNC 4 RCUT 7.5 }}",
        "  ONEBODY {",
        f"    COEFFICIENTS {{ {label} " + " ".join(_fmt(c) for c in onebody) + " }",
        "  }",
    ]
    if threebody is not None:
        g2.insert(1, "  EEBASIS { EE POLYPADE BETA0 0.5 NFUNC 3 RCUT 7.5 }")
        g2 += ["  THREEBODY {",
               f"    COEFFICIENTS {{ {label} " + " ".join(_fmt(c) for c in threebody) + " }",
               "  }"]
        if twobody_pp is not None:
            g2 += ["  TWOBODY {",
                   "    COEFFICIENTS { " + " ".join(_fmt(c) for c in twobody_pp) + " }",
                   "  }"]
    g2.append("}")
    return "\n".join([
        "JASTROW2",
        "GROUP {",
        "  EEBASIS { EE CUTOFF_CUSP GAMMA 24.0 CUSP 1.0 CUTOFF 7.5 }",
        "  EEBASIS { EE CUTOFF_CUSP GAMMA 24.0 CUSP 1.0 CUTOFF 7.5 }",
        "  TWOBODY_SPIN { FREEZE",
        "    LIKE_COEFFICIENTS { 0.25 0.0 }",
        "    UNLIKE_COEFFICIENTS { 0.0 0.5 }",
        "  }",
        "}",
    ] + g2)


def _jastrow_pade_spin_text(rng, label: str) -> str:
    """Jastrow with the PADE radial basis (e-e and e-n), TWOBODY_SPIN and an
    e-e-n THREEBODY_SPIN term on a custom SM_TERMS list, beside the usual
    cusp group."""
    ob = rng.normal(0.0, 0.1, size=3)
    tl, tu = rng.normal(0.0, 0.05, size=4), rng.normal(0.0, 0.05, size=4)
    return "\n".join([
        "JASTROW2",
        "GROUP {",
        "  EEBASIS { EE CUTOFF_CUSP GAMMA 24.0 CUSP 1.0 CUTOFF 7.5 }",
        "  EEBASIS { EE CUTOFF_CUSP GAMMA 24.0 CUSP 1.0 CUTOFF 7.5 }",
        "  TWOBODY_SPIN { FREEZE",
        "    LIKE_COEFFICIENTS { 0.25 0.0 }",
        "    UNLIKE_COEFFICIENTS { 0.0 0.5 }",
        "  }",
        "}",
        "GROUP {",
        "  EEBASIS { EE PADE NFUNC 2 ALPHA0 1.3 }",
        f"  EIBASIS {{ {label} PADE NFUNC 3 ALPHA0 2.0 }}",
        "  ONEBODY {",
        f"    COEFFICIENTS {{ {label} " + " ".join(_fmt(c) for c in ob) + " }",
        "  }",
        "  TWOBODY_SPIN {",
        f"    LIKE_COEFFICIENTS {{ {_fmt(rng.normal(0, 0.1))} {_fmt(rng.normal(0, 0.1))} }}",
        f"    UNLIKE_COEFFICIENTS {{ {_fmt(rng.normal(0, 0.1))} {_fmt(rng.normal(0, 0.1))} }}",
        "  }",
        "  THREEBODY_SPIN {",
        "    SM_TERMS { 1 1 0  1 0 1  2 1 1  0 2 0 }",
        f"    LIKE_COEFFICIENTS {{ {label} " + " ".join(_fmt(c) for c in tl) + " }",
        f"    UNLIKE_COEFFICIENTS {{ {label} " + " ".join(_fmt(c) for c in tu) + " }",
        "  }",
        "}",
    ])


def _oldqmc_lines(rng, zeff: float) -> list:
    lines = ["  OLDQMC {", "  0.0 3", "  3 3 3"]
    for _l in range(2):
        for _ in range(3):
            lines.append(f"    2 {_fmt(rng.uniform(1.0, 10.0))} {_fmt(rng.uniform(-5.0, 5.0))}")
    lines.append(f"    1 {_fmt(rng.uniform(1.0, 10.0))} {_fmt(zeff)}")
    for _ in range(2):
        lines.append(f"    2 {_fmt(rng.uniform(1.0, 10.0))} {_fmt(rng.uniform(-5.0, 5.0))}")
    lines.append("  }")
    return lines


def _pseudo_text_spin(rng, label: str, zeff: float, aip: int, add_zeff: bool) -> str:
    """SPIN_DEP pseudopotential: separate RGAUSSIAN OLDQMC bases for spin-up
    (BASIS_UP) and spin-down (BASIS_DN) electrons, optionally ADD_ZEFF."""
    lines = [f"PSEUDO {{ {label}", "  SPIN_DEP"] + (["  ADD_ZEFF"] if add_zeff else []) + [f"  AIP {aip}"]
    for sec in ("BASIS_UP", "BASIS_DN"):
        lines += [f"  {sec} {{ {label}", "  RGAUSSIAN"] + _oldqmc_lines(rng, zeff) + ["  }"]
    lines.append("}")
    return "\n".join(lines)


def _pseudo_text(rng, label: str, zeff: float, aip: int = 12) -> str:
    """RGAUSSIAN OLDQMC block: channels l=0, l=1 and the local channel (the
    reference treats the LAST listed channel as local, Pseudopotential.cpp:790).
    Nonlocal channels: 3 Gaussians each, exponents U[1,10], coefficients
    U(-5,5).  Local channel: Z_eff/r exp(-a r^2) (cancels the bare -Z_eff/r of
    the ion at the nucleus, as semilocal pseudopotentials do) plus two
    Gaussians of the same distribution."""
    lines = [f"PSEUDO {{ {label}", f"  AIP {aip}", f"  BASIS {{ {label}", "  RGAUSSIAN", "  OLDQMC {",
             "  0.0 3", "  3 3 3"]
    for _l in range(2):
        for _ in range(3):
            lines.append(f"    2 {_fmt(rng.uniform(1.0, 10.0))} {_fmt(rng.uniform(-5.0, 5.0))}")
    lines.append(f"    1 {_fmt(rng.uniform(1.0, 10.0))} {_fmt(zeff)}")
    for _ in range(2):
        lines.append(f"    2 {_fmt(rng.uniform(1.0, 10.0))} {_fmt(rng.uniform(-5.0, 5.0))}")
    lines += ["  }", "  }", "}"]
    return "\n".join(lines)


def write_n2(outdir: str, seed: int = 1234, pseudo: bool = False, method: str | None = None,
             name: str | None = None, expansion=None, high_l: bool = False, jastrow: bool = True,
             dup_basis: bool = False, mo_kind: str = "BLAS_MO", aip: int = 12,
             jastrow_variant: str | None = None, pp_variant: str | None = None) -> Deck:
    """Two-atom molecule of the all-electron (``pseudo=False``) or Z_eff=5
    pseudopotential (``pseudo=True``) workload.  ``method`` is an optional
    METHOD section body written into the deck (e.g. ``"VMC NBLOCK 50 ..."``).
    ``expansion``: optional determinant expansion [(weight, up orbitals,
    down orbitals)], orbitals numbered from 1 within each spin (7 occupied
    plus virtual orbitals up to the largest index used).  ``high_l``: a
    basis with F and G shells in every angular order (6 S, 3 P, 5D, 7F, 10F,
    7F_crystal, 9G, 15G per atom, CRYSTAL normalisation).  ``jastrow=False``
    writes a Slater wave function alone (TRIALFUNC { SLATER ... });
    ``dup_basis`` writes the BASIS section twice (the reference appends both to
    the atoms: the copies' functions carry no orbital coefficients).
    ``aip``: the pseudopotential quadrature (4, 6, 12, 18, 26 or 32 points).
    ``jastrow_variant="pade_spin"``: the PADE / THREEBODY_SPIN / SM_TERMS
    Jastrow of _jastrow_pade_spin_text.  ``pp_variant="spin_dep"``: a SPIN_DEP
    pseudopotential with ADD_ZEFF (_pseudo_text_spin)."""
    os.makedirs(outdir, exist_ok=True)
    rng = np.random.default_rng(seed)
    label = "N"
    charge = 5 if pseudo else 7
    nup = ndown = 7
    # all-electron cores need the tight exponents; pseudopotential atoms use the
    # valence range (with [0.1, 1e4] the random-MO trial function sends the
    # reference's own DMC to E_T < -3e4 Ha within 10 blocks)
    if high_l:
        shells = _basis_shells(rng, {"S": 6, "P": 3, "5D": 1, "7F": 1, "10F": 1, "7F_crystal": 1, "9G": 1, "15G": 1},
                               hi=10.0 if pseudo else 1e4)
    else:
        shells = _basis_shells(rng, {"S": 10, "P": 6, "6D": 2}, hi=10.0 if pseudo else 1e4)
    nper = sum(SHELL_NFUNC[s] for s, _, _ in shells)
    nb = 2 * nper
    nspin_mo = nup if not expansion else max(max(max(u), max(d)) for _, u, d in expansion)
    cup = _random_orthonormal(rng, nb, nspin_mo)
    cdn = _random_orthonormal(rng, nb, nspin_mo)
    onebody = rng.normal(0.0, 0.1, size=4)
    pp = _pseudo_text(rng, label, charge, aip=aip) if pseudo else ""
    if pseudo and pp_variant == "spin_dep":
        pp = _pseudo_text_spin(rng, label, charge, aip, add_zeff=True)
    jtext = _jastrow_pade_spin_text(rng, label) if jastrow_variant == "pade_spin" else _jastrow_text(label, onebody)
    name = name or ("n2_pseudo" if pseudo else "n2_allelectron")
    orb = os.path.join(outdir, f"{name}.orb")
    _write_orb(orb, np.concatenate([cup, cdn], axis=1), [nper, nper])
    if not expansion:
        expansion = [(1.0, list(range(1, nup + 1)), list(range(1, ndown + 1)))]
    detwt = " ".join(_fmt(w) for w, _, _ in expansion)
    states = "\n      ".join(" ".join(str(i) for i in u) + " " + " ".join(str(nspin_mo + i) for i in d)
                              for _, u, d in expansion)
    deck = "\n".join([
        f"# seeded synthetic workload {name} (seed {seed})",
        f"RANDOMSEED {{ {1 + seed % 100000} {7 + seed % 7919} }}",
        "SYSTEM { MOLECULE",
        f"  NSPIN {{ {nup} {ndown} }}",
        f"  ATOM {{ {label} {charge} COOR 0.0 0.0 -1.0375 }}",
        f"  ATOM {{ {label} {charge} COOR 0.0 0.0 1.0375 }}",
        "}",
        pp,
        "TRIALFUNC { SLATER-JASTROW" if jastrow else "TRIALFUNC { SLATER",
        "  WF1 { SLATER" if jastrow else "",
        f"    ORBITALS {{ {mo_kind}",
        f"      NMO {2 * nspin_mo}",
        f"      ORBFILE {os.path.basename(orb)}",
        _basis_text(label, shells, normtype="CRYSTAL" if high_l else None),
        _basis_text(label, shells, normtype="CRYSTAL" if high_l else None) if dup_basis else "",
        "      CENTERS { USEATOMS }",
        "    }",
        f"    DETWT {{ {detwt} }}",
        f"    STATES {{ {states} }}",
        "  }" if jastrow else "",
        "  WF2 {" if jastrow else "",
        jtext if jastrow else "",
        "  }" if jastrow else "",
        "}",
        f"METHOD {{ {method} }}" if method else "",
    ]) + "\n"
    path = os.path.join(outdir, f"{name}.qw")
    with open(path, "w") as fh:
        fh.write(deck)
    return Deck(path=path, orb_path=orb, nup=nup, ndown=ndown, natoms=2, nbasis=nb,
                kind=name, seed=seed)


DIAMOND_FRAC = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0],
                         [.25, .25, .25], [.25, .75, .75], [.75, .25, .75], [.75, .75, .25]])


def write_periodic(outdir: str, seed: int = 4321, a: float = 6.74, image_cutoff: float = 16.0,
                   name: str = "diamond8", method: str | None = None, supercell=(1, 1, 1), kpoint=None,
                   complex_orbitals: bool = False, high_l: bool = False, mo_kind: str = "BLAS_MO") -> Deck:
    """Simple-cubic 8-atom diamond-like cell (lattice constant ``a`` bohr) of
    Z_eff=4 pseudo-atoms, 32 electrons (16 up, 16 down).  Per atom 13 periodic
    Gaussians (4 S + 3 P shells, 3 primitives, exponents log-uniform in
    [0.1, 5], AOSPLINE CUTOFF 16); image centers out to ``image_cutoff`` bohr
    (CUTOFF_DIVIDER = a / image_cutoff); Ewald with EWALD_GMAX 8 (the
    reference's alpha = 5 / smallest cell height); Jastrow with e-e
    (CUTOFF_CUSP), e-n (POLYPADE, 4 coefficients) and e-e-n (8 coefficients)
    terms, all cut off inside half the cell (3.3 bohr) so the minimum-image
    Jastrow is smooth.  ``supercell`` = (n1, n2, n3) repeats the cell along
    the three axes (16 up + 16 down electrons per repeat), e.g. (2, 2, 2) is
    the 64-atom, 256-electron cell with a = 13.48 bohr (64 atoms of Z_eff 4).

    ``kpoint`` = (k1, k2, k3) writes KPOINT (twisted boundary conditions: a
    translation by lattice vector i multiplies the orbitals by exp(i pi k_i));
    ``complex_orbitals`` writes CORBITALS with random complex orthonormal
    coefficients (the imaginary parts are drawn after everything else, so the
    real parts, geometry and Jastrow equal those of the real deck).
    ``high_l``: per atom one S, P, 5D and 7F_crystal shell (16 functions,
    CRYSTAL normalisation) instead of 4 S + 3 P."""
    os.makedirs(outdir, exist_ok=True)
    rng = np.random.default_rng(seed)
    ncell = int(np.prod(supercell))
    label, charge, nup, ndown = "X", 4, 16 * ncell, 16 * ncell
    shells = []
    for sym, n in ((("S", 1), ("P", 1), ("5D", 1), ("7F_crystal", 1)) if high_l else (("S", 4), ("P", 3))):
        for _ in range(n):
            ex = np.exp(rng.uniform(np.log(0.1), np.log(5.0), size=3))
            shells.append((sym, ex, rng.uniform(0.1, 1.0, size=3)))
    nper = sum(SHELL_NFUNC[s] for s, _, _ in shells)
    natoms = len(DIAMOND_FRAC) * ncell
    nb = natoms * nper
    cup = _random_orthonormal(rng, nb, nup)
    cdn = _random_orthonormal(rng, nb, ndown)
    onebody = rng.normal(0.0, 0.1, size=4)
    threebody = rng.normal(0.0, 0.05, size=8)
    pp = _pseudo_text(rng, label, charge)
    coeff = np.concatenate([cup, cdn], axis=1)
    if complex_orbitals:
        # complex orthonormal columns per spin: QR of (real part + i * fresh normals)
        im = rng.standard_normal(coeff.shape)
        parts = []
        for c0, c1 in ((0, nup), (nup, nup + ndown)):
            q, r = np.linalg.qr(coeff[:, c0:c1] + 1j * im[:, c0:c1])
            parts.append(q * (np.diag(r) / np.abs(np.diag(r))).conj()[None, :])
        coeff = np.concatenate(parts, axis=1)
    orb = os.path.join(outdir, f"{name}.orb")
    _write_orb(orb, coeff, [nper] * natoms)
    pos = np.concatenate([(DIAMOND_FRAC + np.array([i, j, k])) * a for i in range(supercell[0])
                          for j in range(supercell[1]) for k in range(supercell[2])])
    edge = [a * n for n in supercell]
    rc = 3.3
    jas = "\n".join([
        "JASTROW2",
        "GROUP {",
        f"  EEBASIS {{ EE CUTOFF_CUSP GAMMA 24.0 CUSP 1.0 CUTOFF {rc} }}",
        f"  EEBASIS {{ EE CUTOFF_CUSP GAMMA 24.0 CUSP 1.0 CUTOFF {rc} }}",
        "  TWOBODY_SPIN { FREEZE",
        "    LIKE_COEFFICIENTS { 0.25 0.0 }",
        "    UNLIKE_COEFFICIENTS { 0.0 0.5 }",
        "  }",
        "}",
        "GROUP {",
        f"  EEBASIS {{ EE POLYPADE BETA0 0.5 NFUNC 3 RCUT {rc} }}",
        f"  EIBASIS {{ {label} POLYPADE BETA0 1.2 NFUNC 4 RCUT {rc} }}",
        "  ONEBODY {",
        f"    COEFFICIENTS {{ {label} " + " ".join(_fmt(c) for c in onebody) + " }",
        "  }",
        "  THREEBODY {",
        f"    COEFFICIENTS {{ {label} " + " ".join(_fmt(c) for c in threebody) + " }",
        "  }",
        "}",
    ])
    states_up = " ".join(str(i + 1) for i in range(nup))
    states_dn = " ".join(str(nup + i + 1) for i in range(ndown))
    deck = "\n".join([
        f"# seeded synthetic workload {name} (seed {seed})",
        f"RANDOMSEED {{ {1 + seed % 100000} {7 + seed % 7919} }}",
        "SYSTEM { PERIODIC",
        f"  NSPIN {{ {nup} {ndown} }}",
        f"  LATTICEVEC {{ {_fmt(edge[0])} 0 0  0 {_fmt(edge[1])} 0  0 0 {_fmt(edge[2])} }}",
        "  ORIGIN { 0 0 0 }",
        f"  CUTOFF_DIVIDER {_fmt(min(edge) / image_cutoff)}",
        "  EWALD_GMAX 8",
    ] + ([f"  KPOINT {{ {_fmt(kpoint[0])} {_fmt(kpoint[1])} {_fmt(kpoint[2])} }}"] if kpoint is not None else []) + [
        f"  ATOM {{ {label} {charge} COOR {_fmt(p[0])} {_fmt(p[1])} {_fmt(p[2])} }}" for p in pos] + [
        "}",
        pp,
        "TRIALFUNC { SLATER-JASTROW",
        "  WF1 { SLATER",
        f"    {'CORBITALS' if complex_orbitals else 'ORBITALS'} {{ {mo_kind}",
        f"      NMO {nup + ndown}",
        f"      ORBFILE {os.path.basename(orb)}",
        _basis_text(label, shells, cutoff=16.0, normtype="CRYSTAL" if high_l else None),
        "      CENTERS { USEGLOBAL }",
        "    }",
        "    DETWT { 1.0 }",
        f"    STATES {{ {states_up} {states_dn} }}",
        "  }",
        "  WF2 {",
        jas,
        "  }",
        "}",
        f"METHOD {{ {method} }}" if method else "",
    ]) + "\n"
    path = os.path.join(outdir, f"{name}.qw")
    with open(path, "w") as fh:
        fh.write(deck)
    return Deck(path=path, orb_path=orb, nup=nup, ndown=ndown, natoms=natoms, nbasis=nb, kind=name, seed=seed,
                extra={"a": a, "cell": edge, "atoms": pos})


MAX_BATCH_ELECTRONS = 192  # 32 atoms of Z_eff <= 6


def write_molecule(outdir: str, name: str, seed: int, nelec: int, max_atoms: int = 32) -> Deck:
    """One seeded molecule of the batched-uneven workload: pseudo-atoms with
    Z_eff 1-6 summing to ``nelec`` (neutral, 2..max_atoms atoms) at random
    positions at least 1.5 bohr apart; 10 Gaussians per atom (4 S + 2 P,
    exponents log-uniform in [0.1, 10]); random orthonormal MOs; Jastrow
    e-e (CUTOFF_CUSP) + e-n (POLYPADE); semilocal pseudopotential per Z_eff
    (as in the two-atom workload)."""
    os.makedirs(outdir, exist_ok=True)
    rng = np.random.default_rng(seed)
    natoms = int(np.clip(round(nelec / rng.uniform(2.5, 4.5)), 2, max_atoms))
    natoms = min(natoms, nelec)
    z = np.ones(natoms, dtype=int)
    for _ in range(nelec - natoms):
        cand = np.flatnonzero(z < 6)
        z[rng.choice(cand)] += 1
    radius = 1.2 * natoms ** (1.0 / 3.0) + 1.0
    pos = []
    while len(pos) < natoms:
        p = rng.uniform(-radius, radius, size=3)
        if np.linalg.norm(p) <= radius and all(np.linalg.norm(p - q) >= 1.5 for q in pos):
            pos.append(p)
    pos = np.array(pos)
    types = sorted(set(int(v) for v in z))
    shells = {t: _basis_shells(rng, {"S": 4, "P": 2}, hi=10.0) for t in types}
    nper = {t: sum(SHELL_NFUNC[sy] for sy, _, _ in shells[t]) for t in types}
    nb = sum(nper[int(v)] for v in z)
    nup, ndn = (nelec + 1) // 2, nelec // 2
    cup = _random_orthonormal(rng, nb, nup)
    cdn = _random_orthonormal(rng, nb, ndn) if ndn else np.zeros((nb, 0))
    orb = os.path.join(outdir, f"{name}.orb")
    _write_orb(orb, np.concatenate([cup, cdn], axis=1), [nper[int(v)] for v in z])
    label = {t: f"Z{t}" for t in types}
    onebody = {t: rng.normal(0.0, 0.1, size=4) for t in types}
    pp = "\n".join(_pseudo_text(rng, label[t], float(t)) for t in types)
    jas = ["JASTROW2", "GROUP {",
           "  EEBASIS { EE CUTOFF_CUSP GAMMA 24.0 CUSP 1.0 CUTOFF 7.5 }",
           "  EEBASIS { EE CUTOFF_CUSP GAMMA 24.0 CUSP 1.0 CUTOFF 7.5 }",
           "  TWOBODY_SPIN { FREEZE", "    LIKE_COEFFICIENTS { 0.25 0.0 }", "    UNLIKE_COEFFICIENTS { 0.0 0.5 }",
           "  }", "}", "GROUP {"]
    for t in types:
        jas.append(f"  EIBASIS {{ {label[t]} POLYPADE BETA0 1.2 NFUNC 4 RCUT 7.5 }}")
    jas.append("  ONEBODY {")
    for t in types:
        jas.append(f"    COEFFICIENTS {{ {label[t]} " + " ".join(_fmt(c) for c in onebody[t]) + " }")
    jas += ["  }", "}"]
    states_up = " ".join(str(i + 1) for i in range(nup))
    states_dn = " ".join(str(nup + i + 1) for i in range(ndn))
    deck = "\n".join([
        f"# seeded synthetic molecule {name} (seed {seed})",
        f"RANDOMSEED {{ {1 + seed % 100000} {7 + seed % 7919} }}",
        "SYSTEM { MOLECULE",
        f"  NSPIN {{ {nup} {ndn} }}",
    ] + [f"  ATOM {{ {label[int(z[a])]} {int(z[a])} COOR {_fmt(pos[a, 0])} {_fmt(pos[a, 1])} {_fmt(pos[a, 2])} }}"
         for a in range(natoms)] + [
        "}",
        pp,
        "TRIALFUNC { SLATER-JASTROW",
        "  WF1 { SLATER",
        "    ORBITALS { BLAS_MO",
        f"      NMO {nup + ndn}",
        f"      ORBFILE {os.path.basename(orb)}",
    ] + [_basis_text(label[t], shells[t]) for t in types] + [
        "      CENTERS { USEATOMS }",
        "    }",
        "    DETWT { 1.0 }",
        f"    STATES {{ {states_up} {states_dn} }}",
        "  }",
        "  WF2 {",
        "\n".join(jas),
        "  }",
        "}",
    ]) + "\n"
    path = os.path.join(outdir, f"{name}.qw")
    with open(path, "w") as fh:
        fh.write(deck)
    return Deck(path=path, orb_path=orb, nup=nup, ndown=ndn, natoms=natoms, nbasis=nb, kind=name, seed=seed,
                extra={"atoms": pos})


def write_batch(outdir: str, nsys: int = 64, seed: int = 777, emin: int = 8,
                emax: int = MAX_BATCH_ELECTRONS) -> list:
    """The batched-uneven workload: ``nsys`` seeded molecules with electron
    counts log-uniform in [emin, emax] and 512-4096 walkers each (log-uniform);
    returns [(deck, walkers)].  With 2-32 atoms of Z_eff 1-6 a neutral
    molecule has at most 192 electrons, the default upper end."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(nsys):
        ne = int(round(np.exp(rng.uniform(np.log(emin), np.log(emax)))))
        nw = int(round(np.exp(rng.uniform(np.log(512), np.log(4096)))))
        d = write_molecule(outdir, f"mol{i:02d}", seed * 1000 + i, ne)
        out.append((d, nw))
    return out


def read_deck(path: str) -> Deck:
    """A Deck record for an existing molecule or cell file (sizes, atom
    positions, lattice edge), enough to draw configurations for it."""
    words = open(path).read().replace("{", " { ").replace("}", " } ").split()
    nup = ndn = 0
    atoms, cell = [], None
    for i, w in enumerate(words):
        u = w.upper()
        if u == "NSPIN":
            nup, ndn = int(words[i + 2]), int(words[i + 3])
        elif u == "COOR":
            atoms.append([float(words[i + 1]), float(words[i + 2]), float(words[i + 3])])
        elif u == "LATTICEVEC":
            v = [float(x) for x in words[i + 2:i + 11]]
            cell = [v[0], v[4], v[8]]
    extra = {"atoms": np.array(atoms)}
    if cell is not None:
        extra = {"a": cell[0], "cell": cell}
    return Deck(path=path, orb_path="", nup=nup, ndown=ndn, natoms=len(atoms), nbasis=0,
                kind=os.path.splitext(os.path.basename(path))[0], seed=0, extra=extra)


def random_configs(deck: Deck, nconf: int, seed: int, spread: float = 1.2) -> np.ndarray:
    """Seeded electron configurations [nconf, nelec, 3]: each electron sits
    near a random atom with a Gaussian spread (bohr)."""
    rng = np.random.default_rng(seed)
    if "a" in deck.extra:  # periodic (orthorhombic) cell: uniform in the cell
        edge = np.asarray(deck.extra.get("cell", [deck.extra["a"]] * 3), dtype=float)
        return rng.uniform(0.0, 1.0, size=(nconf, deck.nelec, 3)) * edge
    atoms = deck.extra.get("atoms", np.array([[0.0, 0.0, -1.0375], [0.0, 0.0, 1.0375]]))
    which = rng.integers(0, len(atoms), size=(nconf, deck.nelec))
    return atoms[which] + rng.normal(0.0, spread, size=(nconf, deck.nelec, 3))


def random_rotation(rng) -> np.ndarray:
    """Uniform random rotation (rows are the rotated x, y, z axes)."""
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q * np.sign(np.diag(r))[None, :]
    if np.linalg.det(q) < 0:
        q[:, 0] *= -1
    return q.T.copy()
