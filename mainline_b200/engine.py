"""Python binding (ctypes) of the walker engine's C-ABI (include/qwg.h).

This mirrors the reference's module surface for the walker path: a context is
built from a QWalk input file (SYSTEM / PSEUDO / TRIALFUNC sections), walkers
are QWalk configurations (N x 3 positions), and the calls map onto the
reference's per-walker operations (Slat_Jastrow::updateLap/getLap/getVal,
System::calcKinetic/calcLoc, Pseudopotential::calcNonlocWithTest,
Vmc_method / Dmc_method blocks).  Errors raise QwgError with the library's
message; there is no CPU fallback: without the built library or a GPU the
calls fail loudly.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("QWG_LIBRARY", os.path.join(HERE, "libqwg.so"))

FP64 = 0
MIXED = 1

EXPORTS = [
    "qwg_version", "qwg_last_error", "qwg_create", "qwg_destroy", "qwg_get_info", "qwg_inspect_deck",
    "qwg_inspect_spline", "qwg_set_walkers", "qwg_get_walkers", "qwg_set_walkers_device",
    "qwg_get_walker_scalars", "qwg_eval", "qwg_mo_eval", "qwg_phase_counters",
    "qwg_ratio", "qwg_set_vmc_dynamics", "qwg_vmc_block", "qwg_dmc_init", "qwg_dmc_block", "qwg_dmc_block_async", "qwg_dmc_block_wait",
    "qwg_vmc_block_noalloc", "qwg_batch_create", "qwg_batch_block", "qwg_batch_destroy", "qwg_autotune",
    "qwg_launch_count", "qwg_reset_launch_count", "qwg_footprint", "qwg_dmc_block_ready", "qwg_time_kernels",
    "qwg_log_header", "qwg_log_block", "qwg_write_configs", "qwg_count_configs", "qwg_read_configs",
    "qwg_store_configs", "qwg_tmove_select",
    "qwg_server_create", "qwg_server_destroy", "qwg_server_submit", "qwg_server_progress",
    "qwg_server_get_status", "qwg_server_last_error",
]


class QwgError(RuntimeError):
    pass


class Info(C.Structure):
    _fields_ = [("nelec", C.c_int), ("nup", C.c_int), ("ndown", C.c_int), ("natoms", C.c_int),
                ("nbasis", C.c_int), ("nshell", C.c_int), ("nmo_up", C.c_int), ("nmo_down", C.c_int),
                ("has_pseudo", C.c_int), ("max_walkers", C.c_int), ("precision", C.c_int),
                ("walkers_per_cta", C.c_int), ("ion_ion", C.c_double), ("device_bytes", C.c_ulonglong),
                ("complex_orbitals", C.c_int)]


class EvalOut(C.Structure):
    _fields_ = [(n, C.POINTER(C.c_double)) for n in
                ("logpsi", "sign", "grad", "lap", "kinetic", "potential", "nonlocal")]


class BlockStats(C.Structure):
    _fields_ = [("energy", C.c_double), ("kinetic", C.c_double), ("potential", C.c_double),
                ("nonlocal", C.c_double), ("weight", C.c_double), ("energy_var", C.c_double),
                ("acceptance", C.c_double), ("etrial", C.c_double), ("block_ms", C.c_double),
                ("nsteps", C.c_int), ("nwalkers", C.c_int), ("nonfinite", C.c_int),
                ("npoints", C.c_double), ("var_energy", C.c_double), ("var_kinetic", C.c_double),
                ("var_potential", C.c_double), ("var_nonlocal", C.c_double), ("var_weight", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class DmcParams(C.Structure):
    _fields_ = [("timestep", C.c_double), ("nstep", C.c_int), ("feedback_interval", C.c_int),
                ("feedback", C.c_double), ("max_poss_weight", C.c_double),
                ("branch_start_cutoff", C.c_double), ("refresh_interval", C.c_int),
                ("deterministic_pp", C.c_int), ("seed", C.c_uint64), ("tmoves", C.c_int)]


class JobDesc(C.Structure):
    _fields_ = [("deck", C.c_char_p), ("precision", C.c_int), ("nwalkers", C.c_int), ("nblocks", C.c_int),
                ("vmc_blocks", C.c_int), ("vmc_steps", C.c_int), ("vmc_timestep", C.c_double),
                ("vmc_seed", C.c_uint64), ("R", C.POINTER(C.c_double)), ("dmc", DmcParams)]


class BlockEvent(C.Structure):
    _fields_ = [("job", C.c_int), ("block", C.c_int), ("latency_ms", C.c_double), ("queue_ms", C.c_double),
                ("stats", BlockStats)]


class ServerStatus(C.Structure):
    _fields_ = [("queued", C.c_int), ("active", C.c_int), ("finished", C.c_int), ("failed", C.c_int),
                ("bytes_in_use", C.c_ulonglong), ("budget_bytes", C.c_ulonglong), ("blocks_done", C.c_longlong),
                ("walker_steps", C.c_double)]


_lib = None


def load_library(path: str = LIB_PATH):
    """Load libqwg.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise QwgError(f"engine library not built: {path} (run python -m mainline_b200.build)")
    lib = C.CDLL(path)
    P = C.POINTER
    dp = P(C.c_double)
    sig = {
        "qwg_version": (C.c_char_p, []),
        "qwg_last_error": (C.c_char_p, [C.c_void_p]),
        "qwg_create": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_void_p, P(C.c_void_p)]),
        "qwg_destroy": (C.c_int, [C.c_void_p]),
        "qwg_get_info": (C.c_int, [C.c_void_p, P(Info)]),
        "qwg_inspect_deck": (C.c_int, [C.c_char_p, P(Info), C.c_char_p, C.c_int]),
        "qwg_inspect_spline": (C.c_int, [C.c_char_p, C.c_int, dp, C.c_int, P(C.c_int), dp, dp]),
        "qwg_set_walkers": (C.c_int, [C.c_void_p, dp, C.c_int]),
        "qwg_get_walkers": (C.c_int, [C.c_void_p, dp, C.c_int]),
        "qwg_set_walkers_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
        "qwg_get_walker_scalars": (C.c_int, [C.c_void_p, dp, dp, C.c_int]),
        "qwg_eval": (C.c_int, [C.c_void_p, dp, P(EvalOut)]),
        "qwg_ratio": (C.c_int, [C.c_void_p, P(C.c_int), dp, dp, dp, dp, dp]),
        "qwg_mo_eval": (C.c_int, [C.c_void_p, dp, C.c_int, C.c_int, dp]),
        "qwg_phase_counters": (C.c_int, [C.c_void_p, P(C.c_ulonglong), C.c_int, C.c_int]),
        "qwg_set_vmc_dynamics": (C.c_int, [C.c_void_p, C.c_int, C.c_double]),
        "qwg_vmc_block": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_uint64, C.c_int, P(BlockStats)]),
        "qwg_dmc_init": (C.c_int, [C.c_void_p, P(DmcParams)]),
        "qwg_dmc_block": (C.c_int, [C.c_void_p, P(BlockStats)]),
        "qwg_dmc_block_async": (C.c_int, [C.c_void_p]),
        "qwg_dmc_block_wait": (C.c_int, [C.c_void_p, P(BlockStats)]),
        "qwg_vmc_block_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_uint64,
                                            C.c_int, C.c_void_p, C.c_void_p]),
        "qwg_batch_create": (C.c_int, [P(C.c_void_p), C.c_int, P(C.c_void_p)]),
        "qwg_batch_block": (C.c_int, [C.c_void_p, P(BlockStats)]),
        "qwg_batch_destroy": (C.c_int, [C.c_void_p]),
        "qwg_autotune": (C.c_int, [C.c_void_p, P(C.c_int)]),
        "qwg_launch_count": (C.c_longlong, [C.c_void_p]),
        "qwg_reset_launch_count": (None, [C.c_void_p]),
        "qwg_footprint": (C.c_int, [C.c_char_p, C.c_int, C.c_int, P(C.c_ulonglong)]),
        "qwg_dmc_block_ready": (C.c_int, [C.c_void_p]),
        "qwg_time_kernels": (C.c_int, [C.c_void_p, C.c_int, dp, dp]),
        "qwg_log_header": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_double, C.c_int, C.c_int]),
        "qwg_log_block": (C.c_int, [C.c_char_p, C.c_char_p, P(BlockStats)]),
        "qwg_write_configs": (C.c_int, [C.c_char_p, dp, dp, dp, C.c_int, C.c_int]),
        "qwg_count_configs": (C.c_int, [C.c_char_p, P(C.c_int), P(C.c_int)]),
        "qwg_read_configs": (C.c_int, [C.c_char_p, dp, dp, dp, C.c_int, C.c_int, P(C.c_int)]),
        "qwg_store_configs": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int]),
        "qwg_tmove_select": (C.c_int, [C.c_void_p, dp, C.c_int, C.c_double, C.c_uint64, P(C.c_int), dp]),
        "qwg_server_create": (C.c_int, [C.c_ulonglong, C.c_int, P(C.c_void_p)]),
        "qwg_server_destroy": (C.c_int, [C.c_void_p]),
        "qwg_server_submit": (C.c_int, [C.c_void_p, P(JobDesc), P(C.c_int)]),
        "qwg_server_progress": (C.c_int, [C.c_void_p, P(BlockEvent), C.c_int, P(C.c_int)]),
        "qwg_server_get_status": (C.c_int, [C.c_void_p, P(ServerStatus)]),
        "qwg_server_last_error": (C.c_char_p, [C.c_void_p]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def inspect_deck(deck_path: str) -> Info:
    lib = load_library()
    info = Info()
    err = C.create_string_buffer(512)
    rc = lib.qwg_inspect_deck(deck_path.encode(), C.byref(info), err, 512)
    if rc != 0:
        raise QwgError(err.value.decode())
    return info


def inspect_spline(deck_path: str, shell: int):
    lib = load_library()
    n = C.c_int(0)
    sp = C.c_double(0)
    cut = C.c_double(0)
    rc = lib.qwg_inspect_spline(deck_path.encode(), shell, None, 0, C.byref(n), C.byref(sp), C.byref(cut))
    if rc != 0:
        raise QwgError(f"qwg_inspect_spline failed ({rc})")
    coef = np.zeros((n.value, 4))
    lib.qwg_inspect_spline(deck_path.encode(), shell, _ptr(coef), n.value, C.byref(n), C.byref(sp), C.byref(cut))
    return coef, sp.value, cut.value


@dataclass
class EvalResult:
    logpsi: np.ndarray
    sign: np.ndarray
    grad: np.ndarray
    lap: np.ndarray
    kinetic: np.ndarray
    potential: np.ndarray
    nonlocal_: np.ndarray

    @property
    def energy(self):
        return self.kinetic + self.potential + self.nonlocal_


class Engine:
    """One GPU walker engine context built from a QWalk deck."""

    def __init__(self, deck_path: str, precision: int = FP64, max_walkers: int = 4096, stream=None):
        self.lib = load_library()
        h = C.c_void_p()
        rc = self.lib.qwg_create(os.path.abspath(deck_path).encode(), precision, max_walkers,
                                 C.c_void_p(stream) if stream else None, C.byref(h))
        if rc != 0:
            raise QwgError(f"qwg_create failed ({rc}): {self.lib.qwg_last_error(None).decode()}")
        self.h = h
        self.info = Info()
        self.lib.qwg_get_info(self.h, C.byref(self.info))
        self.nelec = self.info.nelec
        self.nwalk = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.qwg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != 0:
            raise QwgError(f"{what} failed ({rc}): {self.lib.qwg_last_error(self.h).decode()}")

    def set_walkers(self, R: np.ndarray):
        R = np.ascontiguousarray(R, dtype=np.float64)
        assert R.ndim == 3 and R.shape[1] == self.nelec and R.shape[2] == 3
        self._check(self.lib.qwg_set_walkers(self.h, _ptr(R), R.shape[0]), "qwg_set_walkers")
        self.nwalk = R.shape[0]

    def set_walkers_device(self, ptr: int, nw: int):
        self._check(self.lib.qwg_set_walkers_device(self.h, C.c_void_p(ptr), nw), "qwg_set_walkers_device")
        self.nwalk = nw

    def get_walkers(self) -> np.ndarray:
        R = np.zeros((self.nwalk, self.nelec, 3))
        self._check(self.lib.qwg_get_walkers(self.h, _ptr(R), self.nwalk), "qwg_get_walkers")
        return R

    def walker_scalars(self):
        """(local energy, DMC weight) of every walker after the last step."""
        e, w = np.zeros(self.nwalk), np.zeros(self.nwalk)
        self._check(self.lib.qwg_get_walker_scalars(self.h, _ptr(e), _ptr(w), self.nwalk), "qwg_get_walker_scalars")
        return e, w

    def last_energies(self) -> np.ndarray:
        return self.walker_scalars()[0]

    def eval(self, rot: np.ndarray | None = None) -> EvalResult:
        W, N = self.nwalk, self.nelec
        o = {k: np.zeros(W) for k in ("logpsi", "sign", "kinetic", "potential", "nonlocal")}
        o["grad"] = np.zeros((W, N, 3))
        o["lap"] = np.zeros((W, N))
        out = EvalOut(*[_ptr(o[k]) for k in ("logpsi", "sign", "grad", "lap", "kinetic", "potential", "nonlocal")])
        rp = None
        if rot is not None:
            rot = np.ascontiguousarray(rot, dtype=np.float64).reshape(W, 9)
            rp = _ptr(rot)
        self._check(self.lib.qwg_eval(self.h, rp, C.byref(out)), "qwg_eval")
        return EvalResult(o["logpsi"], o["sign"], o["grad"], o["lap"], o["kinetic"], o["potential"], o["nonlocal"])

    def mo_eval(self, pos: np.ndarray, spin: int) -> np.ndarray:
        """MO value, gradient and Laplacian of every orbital of one spin at
        positions pos [n, 3]: [n, nmo, 5] (tensor-core GEMM in mixed
        precision, FP64 CUDA cores otherwise)."""
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        nmo = self.info.nmo_up if spin == 0 else self.info.nmo_down
        out = np.zeros((pos.shape[0], nmo, 5))
        self._check(self.lib.qwg_mo_eval(self.h, _ptr(pos), pos.shape[0], spin, _ptr(out)), "qwg_mo_eval")
        return out

    PHASES = ["mo_rows", "propose_rest", "accept", "kinetic", "potential", "pp_jastrow", "pp_items", "pp_project",
              "pp_points", "refresh", "walker_launch", "pp_point_jastrow"]

    def phase_counters(self, reset: bool = False) -> dict:
        """Clock cycles per walker-kernel phase (profiling build only)."""
        buf = (C.c_ulonglong * 16)()
        self._check(self.lib.qwg_phase_counters(self.h, buf, 16, int(reset)), "qwg_phase_counters")
        return {name: int(buf[i]) for i, name in enumerate(self.PHASES)}

    def ratio(self, e: np.ndarray, rnew: np.ndarray):
        W = self.nwalk
        e = np.ascontiguousarray(e, dtype=np.int32)
        rnew = np.ascontiguousarray(rnew, dtype=np.float64)
        dl, sg, lp = np.zeros(W), np.zeros(W), np.zeros(W)
        g = np.zeros((W, 3))
        self._check(self.lib.qwg_ratio(self.h, e.ctypes.data_as(C.POINTER(C.c_int)), _ptr(rnew), _ptr(dl),
                                       _ptr(sg), _ptr(g), _ptr(lp)), "qwg_ratio")
        return dl, sg, g, lp

    def set_vmc_dynamics(self, depth: int = 2, divider: float = 2.0) -> None:
        """Split_sampler DEPTH / DIVIDER of the VMC moves (default 2 / 2, as the reference's VMC)."""
        self._check(self.lib.qwg_set_vmc_dynamics(self.h, depth, divider), "qwg_set_vmc_dynamics")

    def vmc_block(self, nstep: int, timestep: float, seed: int = 1, deterministic_pp: bool = False) -> dict:
        st = BlockStats()
        self._check(self.lib.qwg_vmc_block(self.h, nstep, timestep, seed, int(deterministic_pp), C.byref(st)),
                    "qwg_vmc_block")
        return st.as_dict()

    def dmc_init(self, timestep: float, nstep: int = 0, seed: int = 1, feedback_interval: int = 5,
                 feedback: float = 1.0, max_poss_weight: float = 7.0, branch_start_cutoff: float = 10.0,
                 refresh_interval: int = 0, deterministic_pp: bool = False, tmoves: int = 0):
        p = DmcParams(timestep, nstep, feedback_interval, feedback, max_poss_weight, branch_start_cutoff,
                      refresh_interval, int(deterministic_pp), seed, tmoves)
        self._check(self.lib.qwg_dmc_init(self.h, C.byref(p)), "qwg_dmc_init")

    def dmc_block(self) -> dict:
        st = BlockStats()
        self._check(self.lib.qwg_dmc_block(self.h, C.byref(st)), "qwg_dmc_block")
        return st.as_dict()

    def dmc_block_async(self):
        """Enqueue one DMC block (one CUDA graph launch) without waiting."""
        self._check(self.lib.qwg_dmc_block_async(self.h), "qwg_dmc_block_async")

    def dmc_block_wait(self) -> dict:
        st = BlockStats()
        self._check(self.lib.qwg_dmc_block_wait(self.h, C.byref(st)), "qwg_dmc_block_wait")
        return st.as_dict()

    def autotune(self) -> int:
        """Pick the walkers-per-CTA launch shape by timing; before dmc_init."""
        w = C.c_int(0)
        self._check(self.lib.qwg_autotune(self.h, C.byref(w)), "qwg_autotune")
        return w.value

    def time_kernels(self, nstep: int = 5):
        """Mean device ms of the move kernel and the local-energy kernel over
        nstep DMC steps launched one by one (advances the walk)."""
        a, b = C.c_double(0), C.c_double(0)
        self._check(self.lib.qwg_time_kernels(self.h, nstep, C.byref(a), C.byref(b)), "qwg_time_kernels")
        return a.value, b.value

    def tmove_select(self, mode: int, tau: float, seed: int = 1, rot: np.ndarray | None = None):
        """T-move selection (deterministic PP) without moving: (moved [W, N]
        int, target [W, N, 3])."""
        W, N = self.nwalk, self.nelec
        moved = np.zeros((W, N), dtype=np.int32)
        pos = np.zeros((W, N, 3))
        r = None if rot is None else np.ascontiguousarray(rot, dtype=np.float64)
        self._check(self.lib.qwg_tmove_select(self.h, _ptr(r) if r is not None else None, mode, tau, seed,
                                              moved.ctypes.data_as(C.POINTER(C.c_int)), _ptr(pos)),
                    "qwg_tmove_select")
        return moved, pos

    def store_configs(self, path: str, dmc: bool = False):
        """Write the resident walkers as a QWalk configuration file."""
        self._check(self.lib.qwg_store_configs(self.h, path.encode(), int(dmc)), "qwg_store_configs")

    def launch_count(self) -> int:
        return int(self.lib.qwg_launch_count(self.h))

    def reset_launch_count(self):
        self.lib.qwg_reset_launch_count(self.h)


class Batch:
    """One CUDA graph that advances a DMC block of every engine at once
    (batched uneven systems)."""

    def __init__(self, engines):
        self.lib = load_library()
        self.engines = list(engines)
        arr = (C.c_void_p * len(self.engines))(*[e.h for e in self.engines])
        h = C.c_void_p()
        rc = self.lib.qwg_batch_create(arr, len(self.engines), C.byref(h))
        if rc != 0:
            raise QwgError(f"qwg_batch_create failed ({rc}): {self.lib.qwg_last_error(None).decode()}")
        self.h = h

    def block(self) -> list:
        st = (BlockStats * len(self.engines))()
        rc = self.lib.qwg_batch_block(self.h, st)
        if rc != 0:
            raise QwgError(f"qwg_batch_block failed ({rc})")
        return [s.as_dict() for s in st]

    def close(self):
        if getattr(self, "h", None):
            self.lib.qwg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def footprint(deck_path: str, precision: int, walkers: int) -> int:
    """Device bytes a context of this deck, precision and walker count holds."""
    lib = load_library()
    b = C.c_ulonglong(0)
    rc = lib.qwg_footprint(deck_path.encode(), precision, walkers, C.byref(b))
    if rc != 0:
        raise QwgError(f"qwg_footprint failed ({rc}) for {deck_path}")
    return int(b.value)


class Server:
    """Continuous-batching DMC job server (include/qwg_server.h)."""

    def __init__(self, budget_bytes: int, max_active: int = 0):
        self.lib = load_library()
        h = C.c_void_p()
        rc = self.lib.qwg_server_create(budget_bytes, max_active, C.byref(h))
        if rc != 0:
            raise QwgError(f"qwg_server_create failed ({rc})")
        self.h = h
        self._ev = (BlockEvent * 256)()

    def submit(self, deck: str, R: np.ndarray, precision: int, nblocks: int, dmc: dict,
               vmc_blocks: int = 2, vmc_steps: int = 10, vmc_timestep: float = 0.3, vmc_seed: int = 1) -> int:
        R = np.ascontiguousarray(R, dtype=np.float64)
        p = DmcParams()
        d = dict(timestep=0.01, nstep=10, feedback_interval=5, feedback=1.0, max_poss_weight=7.0,
                 branch_start_cutoff=10.0, refresh_interval=32, deterministic_pp=0, seed=1)
        d.update(dmc)
        for k, v in d.items():
            setattr(p, k, v)
        j = JobDesc(deck=deck.encode(), precision=precision, nwalkers=R.shape[0], nblocks=nblocks,
                    vmc_blocks=vmc_blocks, vmc_steps=vmc_steps, vmc_timestep=vmc_timestep, vmc_seed=vmc_seed,
                    R=_ptr(R), dmc=p)
        jid = C.c_int(-1)
        rc = self.lib.qwg_server_submit(self.h, C.byref(j), C.byref(jid))
        if rc != 0:
            raise QwgError(f"qwg_server_submit failed ({rc}): {self.lib.qwg_server_last_error(self.h).decode()}")
        return jid.value

    def progress(self) -> list:
        """One scheduling pass; returns the finished blocks as dicts."""
        out = []
        while True:
            n = C.c_int(0)
            rc = self.lib.qwg_server_progress(self.h, self._ev, len(self._ev), C.byref(n))
            if rc != 0:
                raise QwgError(f"qwg_server_progress failed ({rc}): {self.lib.qwg_server_last_error(self.h).decode()}")
            for i in range(n.value):
                e = self._ev[i]
                d = e.stats.as_dict()
                d.update(job=e.job, block=e.block, latency_ms=e.latency_ms, queue_ms=e.queue_ms)
                out.append(d)
            if n.value < len(self._ev):
                return out

    def status(self) -> dict:
        st = ServerStatus()
        self.lib.qwg_server_get_status(self.h, C.byref(st))
        return {k: getattr(st, k) for k, _ in ServerStatus._fields_}

    def close(self):
        if self.h:
            self.lib.qwg_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def log_header(path: str, method: str, label: str, timestep: float, nconfig: int = 0, nstep: int = 0) -> None:
    """Append the run banner and init entry of a QWalk log file (runid.log)."""
    rc = load_library().qwg_log_header(path.encode(), method.encode(), label.encode(), timestep, nconfig, nstep)
    if rc != 0:
        raise QwgError(f"qwg_log_header failed ({rc}) for {path}")


def log_block(path: str, label: str, stats: dict) -> None:
    """Append one block entry (as returned by vmc_block / dmc_block) in the
    format the reference's gosling analyser reads."""
    st = BlockStats()
    for k, _ in BlockStats._fields_:
        if k in stats:
            setattr(st, k, stats[k])
    rc = load_library().qwg_log_block(path.encode(), label.encode(), C.byref(st))
    if rc != 0:
        raise QwgError(f"qwg_log_block failed ({rc}) for {path}")


def write_configs(path: str, R: np.ndarray, weight=None, sign=None) -> None:
    """Write walkers [W, N, 3] (and DMC weights/signs) as a QWalk configuration file."""
    R = np.ascontiguousarray(R, dtype=np.float64)
    W, N = R.shape[0], R.shape[1]
    w = None if weight is None else np.ascontiguousarray(weight, dtype=np.float64)
    sg = None if sign is None else np.ascontiguousarray(sign, dtype=np.float64)
    rc = load_library().qwg_write_configs(path.encode(), _ptr(R), _ptr(w) if w is not None else None,
                                          _ptr(sg) if sg is not None else None, W, N)
    if rc != 0:
        raise QwgError(f"qwg_write_configs failed ({rc}) for {path}")


def read_configs(path: str):
    """Read a QWalk configuration file: (R [W, N, 3], weight [W], sign [W])."""
    lib = load_library()
    nw, ne = C.c_int(0), C.c_int(0)
    if lib.qwg_count_configs(path.encode(), C.byref(nw), C.byref(ne)) != 0:
        raise QwgError(f"malformed configuration file {path}")
    R = np.zeros((nw.value, ne.value, 3))
    w, sg = np.zeros(nw.value), np.zeros(nw.value)
    n = C.c_int(0)
    if nw.value and lib.qwg_read_configs(path.encode(), _ptr(R), _ptr(w), _ptr(sg), nw.value, ne.value,
                                         C.byref(n)) != 0:
        raise QwgError(f"malformed configuration file {path}")
    return R, w, sg
