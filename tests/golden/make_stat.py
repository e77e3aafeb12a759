"""Write the statistical-parity fixtures: a low-variance seeded deck and the
reference's own VMC and DMC energies on it (tests/golden/stat_ref.json).

Run in a container that has the reference build (make -C oracle):
    python tests/golden/make_stat.py [--nproc P] [--vmc-blocks B] [--dmc-blocks B]

The deck is a linear chain of four hydrogen pseudo-atoms (2 up, 2 down
electrons).  Each atom carries a weak semilocal pseudopotential in the
reference's RGAUSSIAN OLDQMC form: a local channel Z_eff/r exp(-a r^2) that
cancels the ion's -1/r at the nucleus plus a Gaussian, and an l=0 nonlocal
channel (12-point quadrature).  The orbitals are the restricted Hartree-Fock
orbitals of the chain in an even-tempered s basis (the SCF sees the local
channel and, as a local potential, the s channel), computed here by a small
closed-form Gaussian-integral SCF; with a cusp e-e Jastrow and a
POLYPADE e-n Jastrow the local-energy variance is small enough that a few
minutes of reference CPU time pin the energy to a fraction of a mHa.

The reference (oracle/_ref/qwalk-Linux, the shipped -O3 build) runs one
process per host core with distinct RANDOMSEEDs.  Per process the block
energies after the equilibration blocks give a mean and a reblocked error;
processes combine as independent estimates.  The engine's energies from the
same deck are compared in tests/test_gpu_stat.py.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np
from scipy.special import erf

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from mainline_b200 import systems  # noqa: E402
from statutil import combine, reblock  # noqa: E402

QWALK = os.path.join(ROOT, "oracle", "_ref", "qwalk-Linux")
NAME = "h4pp"
SPACING = 1.8
EXPONENTS = (0.09, 0.27, 0.8, 2.4, 7.2, 21.6)  # even-tempered s primitives per atom
# pseudopotential channels (n, exponent, coefficient): v(r) = sum c r^(n-2) exp(-a r^2)
PP_S = [(2, 1.1, -0.35)]                       # l = 0, nonlocal
PP_LOCAL = [(1, 3.0, 1.0), (2, 1.6, 0.4)]      # local (cancels -1/r at the nucleus)

# Runs whose energies are pinned.  VMC: the reference's default dynamics
# (Split_sampler depth 2); DMC at a large time step, where the time-step
# error of the Green's function, weights and branching is visible.
RUNS = {
    "vmc": dict(method="VMC", tau=0.5, nstep=20, nconfig=256, equil=5),
    "dmc_tau0.05": dict(method="DMC", tau=0.05, nstep=40, nconfig=512, equil=20),
}


# ---------------------------------------------------------------- RHF (s basis)
def _f0(t):
    t = np.asarray(t, float)
    small = t < 1e-12
    ts = np.where(small, 1.0, t)
    return np.where(small, 1.0 - t / 3.0, 0.5 * np.sqrt(np.pi / ts) * erf(np.sqrt(ts)))


def rhf_s(centers, charges, exps, nocc, pot=(), iters=200, tol=1e-11):
    """Closed-shell Hartree-Fock in normalised s-type Gaussian primitives
    (one primitive per basis function, GAMESS normalisation (2a/pi)^(3/4)).
    ``pot``: extra potential terms on every center, (n, a, c) for
    c r^(n-2) exp(-a r^2) with n = 1 or 2 (the OLDQMC radial form).
    Returns (MO coefficients [nbasis, nocc], E_HF)."""
    cen = np.repeat(np.asarray(centers, float), len(exps), axis=0)
    a = np.tile(np.asarray(exps, float), len(centers))
    nb = len(a)
    nrm = (2 * a / np.pi) ** 0.75
    p = a[:, None] + a[None, :]
    mu = a[:, None] * a[None, :] / p
    d2 = np.sum((cen[:, None] - cen[None, :]) ** 2, axis=-1)
    P = (a[:, None, None] * cen[:, None] + a[None, :, None] * cen[None, :]) / p[..., None]
    K = np.exp(-mu * d2) * nrm[:, None] * nrm[None, :]
    S = (np.pi / p) ** 1.5 * K
    T = mu * (3 - 2 * mu * d2) * S
    V = np.zeros((nb, nb))
    for c, z in zip(np.asarray(centers, float), charges):
        V -= z * 2 * np.pi / p * K * _f0(p * np.sum((P - c) ** 2, axis=-1))
        for n, al, co in pot:
            # Gaussian product with exp(-al |r-C|^2): new exponent p + al at P'
            q = p + al
            Kc = K * np.exp(-p * al / q * np.sum((P - c) ** 2, axis=-1))
            if n == 2:
                V += co * Kc * (np.pi / q) ** 1.5
            else:
                Pp = (p[..., None] * P + al * c) / q[..., None]
                V += co * Kc * 2 * np.pi / q * _f0(q * np.sum((Pp - c) ** 2, axis=-1))
    H = T + V
    # (ab|cd)
    pq = p[:, :, None, None] * p[None, None, :, :]
    ps = p[:, :, None, None] + p[None, None, :, :]
    dPQ = np.sum((P[:, :, None, None, :] - P[None, None, :, :, :]) ** 2, axis=-1)
    eri = 2 * np.pi ** 2.5 / (pq * np.sqrt(ps)) * K[:, :, None, None] * K[None, None, :, :] * _f0(pq / ps * dPQ)
    w, U = np.linalg.eigh(S)
    keep = w > 1e-9
    X = U[:, keep] / np.sqrt(w[keep])
    D = np.zeros((nb, nb))
    e_old = 0.0
    for _ in range(iters):
        J = np.einsum("abcd,cd->ab", eri, D)
        Kx = np.einsum("acbd,cd->ab", eri, D)
        F = H + J - 0.5 * Kx
        e, Cp = np.linalg.eigh(X.T @ F @ X)
        C = X @ Cp[:, :nocc]
        Dn = 2 * C @ C.T
        etot = 0.5 * np.sum(Dn * (H + F))
        D = 0.5 * D + 0.5 * Dn if _ < 5 else Dn
        if abs(etot - e_old) < tol:
            break
        e_old = etot
    cc = np.asarray(centers, float)
    enuc = sum(charges[i] * charges[j] / np.linalg.norm(cc[i] - cc[j])
               for i in range(len(cc)) for j in range(i))
    return C, etot + enuc


# ---------------------------------------------------------------- deck
def write_h4pp(outdir: str, name: str = NAME) -> systems.Deck:
    natoms, nup = 4, 2
    z = (np.arange(natoms) - (natoms - 1) / 2) * SPACING
    centers = np.stack([np.zeros(natoms), np.zeros(natoms), z], axis=1)
    # the SCF sees the local channel and, as a local potential, the s channel
    C, ehf = rhf_s(centers, [1.0] * natoms, EXPONENTS, nup, pot=PP_LOCAL + PP_S)
    C = C * np.sign(C[np.argmax(np.abs(C), axis=0), np.arange(nup)])[None, :]
    nper = len(EXPONENTS)
    orb = os.path.join(outdir, f"{name}.orb")
    systems._write_orb(orb, np.concatenate([C, C], axis=1), [nper] * natoms)
    basis = ["BASIS { H", "AOSPLINE", "GAMESS {"]
    for ex in EXPONENTS:
        basis += ["S 1", f"  1 {ex!r} 1.0"]
    basis += ["}", "}"]
    pseudo = ["PSEUDO { H", "  AIP 12", "  BASIS { H", "  RGAUSSIAN", "  OLDQMC {", "  0.0 2",
              f"  {len(PP_S)} {len(PP_LOCAL)}"]
    pseudo += [f"    {n} {a!r} {c!r}" for n, a, c in PP_S + PP_LOCAL]
    pseudo += ["  }", "  }", "}"]
    jas = systems._jastrow_text("H", np.array([-0.05, 0.02, 0.0, 0.0]))
    deck = "\n".join([
        f"# hydrogen pseudo-atom chain (spacing {SPACING} bohr), RHF orbitals (SCF energy {ehf:.6f})",
        "RANDOMSEED { 11 29 }",
        "SYSTEM { MOLECULE", f"  NSPIN {{ {nup} {nup} }}"]
        + [f"  ATOM {{ H 1 COOR 0.0 0.0 {float(zz)!r} }}" for zz in z]
        + ["}", "\n".join(pseudo),
           "TRIALFUNC { SLATER-JASTROW", "  WF1 { SLATER", "    ORBITALS { BLAS_MO", f"      NMO {2 * nup}",
           f"      ORBFILE {os.path.basename(orb)}", "\n".join(basis), "      CENTERS { USEATOMS }", "    }",
           "    DETWT { 1.0 }", "    STATES { 1 2 3 4 }", "  }", "  WF2 {", jas, "  }", "}"]) + "\n"
    path = os.path.join(outdir, f"{name}.qw")
    open(path, "w").write(deck)
    return systems.Deck(path=path, orb_path=orb, nup=nup, ndown=nup, natoms=natoms, nbasis=natoms * nper,
                        kind=name, seed=0, extra={"e_scf": ehf})


# ---------------------------------------------------------------- reference runs
def _block_energies(log_text):
    return np.array([float(x) for x in re.findall(r"total_energy \{ (\S+)", log_text)])


def run_reference(deck_path: str, run: dict, nblock: int, nproc: int) -> dict:
    base = open(deck_path).read()
    work = tempfile.mkdtemp(prefix="qwstat_")
    for f in (deck_path, deck_path[:-3] + ".orb"):
        os.symlink(os.path.abspath(f), os.path.join(work, os.path.basename(f)))
    procs = []
    for p in range(nproc):
        txt = re.sub(r"RANDOMSEED\s*\{[^}]*\}", f"RANDOMSEED {{ {1000 + 17 * p} {3000 + 29 * p} }}", base)
        m = f"{run['method']} NCONFIG {run['nconfig']} NBLOCK {nblock} NSTEP {run['nstep']} TIMESTEP {run['tau']}"
        if run["method"] == "VMC":
            m += " NDECORR 1"
        txt += f"METHOD {{ {m} }}\n"
        fn = f"run{p}.qw"
        open(os.path.join(work, fn), "w").write(txt)
        procs.append(subprocess.Popen([QWALK, fn], cwd=work, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL))
    for pr in procs:
        if pr.wait() != 0:
            raise RuntimeError("reference run failed")
    series = [_block_energies(open(os.path.join(work, f"run{p}.qw.log")).read())[run["equil"]:]
              for p in range(nproc)]
    mean, err = combine([reblock(s) for s in series])
    return {"energy": mean, "error": err, "processes": nproc, "blocks_per_process": nblock,
            "equilibration_blocks": run["equil"], "walkers_per_process": run["nconfig"],
            "steps_per_block": run["nstep"], "timestep": run["tau"], "method": run["method"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nproc", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--vmc-blocks", type=int, default=400)
    ap.add_argument("--dmc-blocks", type=int, default=400)
    args = ap.parse_args()
    deck = write_h4pp(HERE)
    out = {"deck": os.path.basename(deck.path), "e_scf": deck.extra["e_scf"],
           "reference": "oracle/_ref/qwalk-Linux (shipped -O3 -ffast-math flags)"}
    for key, run in RUNS.items():
        nb = args.vmc_blocks if run["method"] == "VMC" else args.dmc_blocks
        out[key] = run_reference(deck.path, run, nb, args.nproc)
        print(key, out[key], flush=True)
    json.dump(out, open(os.path.join(HERE, "stat_ref.json"), "w"), indent=1)


if __name__ == "__main__":
    main()
