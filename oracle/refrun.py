"""Drive the reference harness (oracle/_ref/qwref_harness) on seeded inputs.

TEST INFRASTRUCTURE ONLY.  Used by tests/golden/make_golden.py to write the
golden vectors and by tests that re-check them where the reference build
exists.  The binary layouts are documented in oracle/qwref_harness.cpp.
"""
from __future__ import annotations

import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HARNESS = os.path.join(HERE, "_ref", "qwref_harness")
QWALK = os.path.join(HERE, "_ref", "qwalk-Linux")


def harness_available() -> bool:
    return os.path.exists(HARNESS)


def write_inputs(path: str, R: np.ndarray, rot: np.ndarray, moves_e: np.ndarray,
                 moves_pos: np.ndarray) -> None:
    nconf, nelec, _ = R.shape
    nmove = moves_e.shape[1]
    with open(path, "wb") as fh:
        fh.write(struct.pack("<3i", nconf, nelec, nmove))
        for c in range(nconf):
            fh.write(np.ascontiguousarray(R[c], dtype="<f8").tobytes())
            fh.write(np.ascontiguousarray(rot[c], dtype="<f8").tobytes())
            for m in range(nmove):
                fh.write(struct.pack("<i", int(moves_e[c, m])))
                fh.write(np.ascontiguousarray(moves_pos[c, m], dtype="<f8").tobytes())


def read_outputs(path: str) -> dict:
    with open(path, "rb") as fh:
        nconf, nelec, nmove = struct.unpack("<3i", fh.read(12))
        per = 2 + 3 * nelec + nelec + 3 + nmove * 6
        data = np.frombuffer(fh.read(), dtype="<f8")
    assert data.size == nconf * per, (data.size, nconf * per)
    data = data.reshape(nconf, per)
    o = 0
    out = {"logpsi": data[:, 0].copy(), "sign": data[:, 1].copy()}
    o = 2
    out["grad"] = data[:, o:o + 3 * nelec].reshape(nconf, nelec, 3).copy(); o += 3 * nelec
    out["lap"] = data[:, o:o + nelec].copy(); o += nelec
    out["kinetic"] = data[:, o].copy()
    out["potential"] = data[:, o + 1].copy()
    out["nonlocal"] = data[:, o + 2].copy(); o += 3
    mv = data[:, o:].reshape(nconf, nmove, 6)
    out["move_dlogpsi"] = mv[:, :, 0].copy()
    out["move_sign"] = mv[:, :, 1].copy()
    out["move_grad"] = mv[:, :, 2:5].copy()
    out["move_lap"] = mv[:, :, 5].copy()
    return out


def run_harness(deck_path: str, R, rot, moves_e, moves_pos) -> dict:
    deck_dir = os.path.dirname(os.path.abspath(deck_path))
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "in.bin")
        fout = os.path.join(td, "out.bin")
        write_inputs(fin, R, rot, moves_e, moves_pos)
        subprocess.run([HARNESS, os.path.abspath(deck_path), fin, fout], cwd=deck_dir,
                       check=True, stdout=subprocess.DEVNULL)
        return read_outputs(fout)
