"""Benchmark: DMC walker-steps/s of the B200 walker engine (mixed precision vs
FP64) with p50/p99 block latency, on the seeded Z_eff=5 pseudopotential
two-atom molecule (14 electrons, 80 basis functions, 4096 walkers, tau=0.01).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

A step is one DMC step of the whole population: every walker moves each of
its 14 electrons (drift-diffusion Metropolis, node restriction), evaluates its
local energy (kinetic + Coulomb + nonlocal pseudopotential) and updates its
weight; branching runs every 5 steps (feedback interval).  walker-steps/s =
walkers x steps / device time.  One process per GPU; the population does not
shard (independent replicas, scaling "weak"); rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from mainline_b200.replicas import aggregate_rate, max_over_ranks, replica_seed  # noqa: E402

NWALK = 4096
TAU = 0.01
FEEDBACK_INTERVAL = 5
SEED = 20261203


FP32_SPEC_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12
ATOMS = np.array([[0.0, 0.0, -1.0375], [0.0, 0.0, 1.0375]])


def _tensor_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        if "bf16_tflops" in d:
            return d["bf16_tflops"], "measured (cuBLAS bf16 burst)"
    return 1590.0, "fallback"


def move_flops_per_walker(N, M, nb, natoms, k_ee, k_en):
    """Algorithmic flops of one sweep of N single-electron moves: MO value,
    gradient and Laplacian (N*5*nb*M*2), ratio and gradient/Laplacian dots
    (N*5*M*2), Sherman-Morrison updates (N*4*M^2) and the Jastrow of the moved
    electron (N*((N-1)*k_ee + A*k_en)*12*5)."""
    return N * 5 * nb * M * 2 + N * 5 * M * 2 + N * 4 * M * M + N * ((N - 1) * k_ee + natoms * k_en) * 60


def pp_flops_per_walker(npairs, N, M, nb, natoms, k_ee, k_en, nq=12):
    """Algorithmic flops of the nonlocal pseudopotential quadrature: per
    (electron, atom) pair inside the cutoff, nq ratio evaluations (MO values,
    determinant ratio, Jastrow value)."""
    return npairs * nq * (nb * M * 2 + 2 * M + 12 * (N * k_ee + natoms * k_en))


def pp_pairs(R, atoms, cut):
    """Mean number of (electron, atom) pairs inside the pseudopotential cutoff."""
    d = np.linalg.norm(R[:, :, None, :] - atoms[None, None], axis=-1)
    return float(np.mean(np.sum(d < cut, axis=(1, 2))))


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 3 + i and
                          s[3 + i].lower() in ("active", "1")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def make_workload(tmpdir):
    from mainline_b200 import systems
    deck = systems.write_n2(tmpdir, seed=12, pseudo=True, name="n2_pseudo_bench")
    R0 = systems.random_configs(deck, NWALK, seed=SEED)
    return deck, R0


def _traffic_per_launch(kernel):
    """DRAM bytes (read + write) of one launch of the given kernel of this
    workload, from the committed ncu summary (profiles/traffic.json), or None."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    return json.load(open(p)).get(kernel, {}).get("dram_bytes_per_launch")


def walker_state_bytes(N, M, precision_bytes):
    """Resident walker state: positions, both inverse matrices, MO
    gradient/Laplacian rows, Jastrow gradients/Laplacians, scalars."""
    return 8 * 3 * N + precision_bytes * (2 * M * M + N * M * 4) + 8 * 4 * N + 64


def algorithmic_bytes_per_walker_step(N, M, nb, precision_bytes):
    """Resident walker state read + written once per step."""
    return 2 * walker_state_bytes(N, M, precision_bytes)


def run_engine(args, rank, world):
    import torch
    from mainline_b200 import engine
    torch.cuda.set_device(rank % max(torch.cuda.device_count(), 1))
    dev = torch.device("cuda", rank % max(torch.cuda.device_count(), 1))
    tmp = tempfile.mkdtemp(prefix="qwg_bench_")
    deck, R0 = make_workload(tmp)
    stream = torch.cuda.Stream(device=dev)
    results = {}
    arms = (("fp64", engine.FP64), ("mixed", engine.MIXED))
    if args.precision != "both":
        arms = tuple(a for a in arms if a[0] == args.precision)
    for label, prec in arms:
        E = engine.Engine(deck.path, prec, max_walkers=NWALK, stream=stream.cuda_stream)
        E.set_walkers(R0)
        for b in range(3):  # VMC equilibration from the seeded start
            E.vmc_block(20, 0.3, seed=replica_seed(SEED, rank) + 17 * b)
        steps = max(FEEDBACK_INTERVAL, (args.steps // FEEDBACK_INTERVAL) * FEEDBACK_INTERVAL)
        E.dmc_init(timestep=TAU, nstep=steps, seed=replica_seed(SEED, rank))
        for _ in range(max(args.warmup, 3) // 1):
            E.dmc_block()  # warm-up blocks (untimed)
        # timed: one block of `steps` steps, CUDA events on the engine's stream
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
        lat = []
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        torch.cuda.synchronize(dev)
        if world > 1:
            torch.distributed.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        E.reset_launch_count()
        with ClockSampler(rank % max(torch.cuda.device_count(), 1)) as cs:
            e0.record(stream)
            st = E.dmc_block()
            e1.record(stream)
            torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1)
        launches = E.launch_count()
        # per-kernel durations (move kernel, local-energy kernel), CUDA events
        # around individual launches of the same kernels the block graph holds
        sweep_ms, eloc_ms = E.time_kernels(5)
        # block latency: several shorter blocks (20 steps), host wall time from
        # block start to block statistics on the host
        E.dmc_init(timestep=TAU, nstep=20, seed=replica_seed(SEED + 99, rank))
        energies = []
        for b in range(args.latency_blocks):
            t0 = time.perf_counter()
            s2 = E.dmc_block()
            lat.append((time.perf_counter() - t0) * 1e3)
            energies.append(s2["energy"])
        results[label] = {"ms": ms, "steps": steps, "stats": st, "launches": launches, "clocks": cs.summary(),
                          "lat": lat, "energies": energies, "kernel_ms": st["block_ms"], "sweep_ms": sweep_ms,
                          "eloc_ms": eloc_ms, "R": E.get_walkers()}
        E.close()
    # end-to-end through the C-ABI with host buffers: upload walkers from
    # pinned host memory, run the block, download walkers + statistics
    e2e = {}
    for label, prec in arms:
        e2e[label] = _e2e_block(engine, deck, R0, prec, results[label]["steps"], stream, dev)
    corr = correlated_mixed_vs_fp64(engine, deck, R0, stream) if args.precision == "both" else None
    return results, e2e, corr, deck


def _e2e_block(engine, deck, R0, prec, steps, stream, dev):
    import torch
    E = engine.Engine(deck.path, prec, max_walkers=NWALK, stream=stream.cuda_stream)
    E.set_walkers(R0)
    E.vmc_block(20, 0.3, seed=SEED)
    E.dmc_init(timestep=TAU, nstep=steps, seed=SEED + 5)
    E.dmc_block()
    Rh = E.get_walkers()
    Rpinned = torch.from_numpy(Rh).pin_memory().numpy()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    E.set_walkers(Rpinned)
    E.dmc_init(timestep=TAU, nstep=steps, seed=SEED + 6)
    E.dmc_block()
    E.get_walkers()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    E.close()
    return ms


def correlated_mixed_vs_fp64(engine, deck, R0, stream, npair=8, nblock=10, nstep=20):
    """Mixed minus FP64 DMC energy at equal statistics.

    (1) Common random numbers on the low-variance H4 pseudo-atom chain
    (tests/golden/h4pp.qw, RHF orbitals, tau=0.05): both contexts start from
    the same walkers with the same seed, so their walks coincide except where
    a decision falls inside the precision difference; the per-block energy
    difference (mean and standard error over blocks) is the precision bias.
    (2) On the headline molecule, whose random-orbital walks part within a
    block, the bias of the mixed local-energy estimator: the same
    configurations (the mixed run's walkers) and quadrature rotation
    evaluated in both precisions."""
    from mainline_b200 import systems
    h4 = os.path.join(ROOT, "tests", "golden", "h4pp.qw")
    F = engine.Engine(h4, engine.FP64, max_walkers=NWALK, stream=stream.cuda_stream)
    F.set_walkers(systems.random_configs(systems.read_deck(h4), NWALK, seed=SEED % 1000))
    for b in range(10):
        F.vmc_block(20, 0.5, seed=SEED + b)
    Rh = F.get_walkers()
    F.close()
    # independent pairs (fresh seeds), each a short walk from the same
    # equilibrated walkers: pairs whose walks stay together measure the bias
    # to ~1e-6 mHa; a pair that parts adds its block noise to the spread
    pair_means, en_f, en_m = [], [], []
    for k in range(npair):
        energies = {}
        for label, prec in (("fp64", engine.FP64), ("mixed", engine.MIXED)):
            E = engine.Engine(h4, prec, max_walkers=NWALK, stream=stream.cuda_stream)
            E.set_walkers(Rh)
            E.dmc_init(timestep=0.05, nstep=nstep, seed=SEED + 77 + 1000 * k)
            energies[label] = np.array([E.dmc_block()["energy"] for _ in range(nblock)])
            E.close()
        pair_means.append(float(np.mean(energies["mixed"] - energies["fp64"]) * 1e3))
        en_f.append(np.mean(energies["fp64"]))
        en_m.append(np.mean(energies["mixed"]))
    d = np.array(pair_means)
    # estimator bias on the headline workload
    M = engine.Engine(deck.path, engine.MIXED, max_walkers=NWALK, stream=stream.cuda_stream)
    M.set_walkers(R0)
    for b in range(3):
        M.vmc_block(20, 0.3, seed=SEED + 31 * b)
    M.dmc_init(timestep=TAU, nstep=20, seed=SEED + 78)
    M.dmc_block()
    Rfinal = M.get_walkers()
    rng = np.random.default_rng(5)
    rot = np.stack([_rotation(rng) for _ in range(NWALK)])
    M.set_walkers(Rfinal)
    em = M.eval(rot).energy
    M.close()
    F = engine.Engine(deck.path, engine.FP64, max_walkers=NWALK, stream=stream.cuda_stream)
    F.set_walkers(Rfinal)
    ef = F.eval(rot).energy
    F.close()
    de = (em - ef) * 1e3
    return {"common_random_numbers": {
                "workload": "h4pp: 4 H pseudo-atoms, 4 electrons, RHF orbitals, DMC tau=0.05",
                "mean": float(np.mean(d)), "sem": float(np.std(d, ddof=1) / np.sqrt(len(d))),
                "per_pair": [round(x, 6) for x in pair_means], "pairs": npair,
                "blocks_per_pair": nblock, "steps_per_block": nstep, "walkers": NWALK,
                "fp64_energy": float(np.mean(en_f)), "mixed_energy": float(np.mean(en_m))},
            "estimator_bias_headline": {"mean": float(np.mean(de)),
                                        "sem": float(np.std(de, ddof=1) / np.sqrt(len(de))),
                                        "median_abs": float(np.median(np.abs(de))), "walkers": NWALK}}


def _rotation(rng):
    q = rng.standard_normal(4)
    a, b, c, d = q / np.linalg.norm(q)
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def run_extras(stream, dev, seconds=30.0):
    """Bounded samples of the other workloads, mixed precision vs FP64:
    the periodic cell (DMC), a batch of uneven molecules advanced by one
    graph per block, and the Poisson job stream through the job server."""
    import torch
    from mainline_b200 import engine, serving, systems
    tmp = tempfile.mkdtemp(prefix="qwg_extra_")
    out = {}
    # cfg 1: the all-electron molecule in FP64 VMC (256 walkers, tau 0.3,
    # 100-step blocks, Split_sampler depth 2 as the reference's VMC)
    ae = systems.write_n2(tmp, seed=11, pseudo=False, name="n2_allelectron_bench")
    E = engine.Engine(ae.path, engine.FP64, max_walkers=256, stream=stream.cuda_stream)
    E.set_walkers(systems.random_configs(ae, 256, seed=SEED))
    E.vmc_block(100, 0.3, seed=SEED)
    vst = [E.vmc_block(100, 0.3, seed=SEED + 1 + b) for b in range(10)]
    E.close()
    vms = float(np.sum([v["block_ms"] for v in vst]))
    out["vmc_allelectron"] = {
        "fp64": {"walker_steps_per_s": 256 * 100 * len(vst) / (vms / 1e3), "block_ms": vms / len(vst),
                 "energy": float(np.mean([v["energy"] for v in vst])),
                 "acceptance": float(np.mean([v["acceptance"] for v in vst]))},
        "config": "cfg 1: two all-electron Z=7 atoms, 14 electrons, 80 Cartesian Gaussians (exponents 0.1-1e4), "
                  "FP64 VMC, 256 walkers, tau=0.3, 10 timed blocks of 100 steps; the random-orbital trial function "
                  "of the tight all-electron basis has local energies of order 1e3 Ha, so the energy is a "
                  "throughput by-product, not a physical value"}
    # the reference on the host cores, same deck, VMC with its default sampler
    out["vmc_allelectron"]["cpu_baseline"] = cpu_reference(os.path.abspath(ae.path), repeats=1, short_blocks=1,
                                                           long_blocks=3, nconf=64, nstep=100, tau=0.3,
                                                           method="VMC")
    # periodic: 8-atom cell, 32 electrons, tau 0.005, 16384 walkers
    cell = systems.write_periodic(tmp, seed=13, name="diamond8_bench")
    Rc = systems.random_configs(cell, 16384, seed=SEED)
    per = {}
    for label, prec in (("fp64", engine.FP64), ("mixed", engine.MIXED)):
        E = engine.Engine(cell.path, prec, max_walkers=16384, stream=stream.cuda_stream)
        E.set_walkers(Rc)
        E.vmc_block(5, 0.3, seed=SEED + 1)
        E.dmc_init(timestep=0.005, nstep=10, seed=SEED + 2)
        E.dmc_block()
        sts = [E.dmc_block() for _ in range(3)]
        bms = float(np.median([x["block_ms"] for x in sts]))
        per[label] = {"walker_steps_per_s": 16384 * 10 / (bms / 1e3), "block_ms": bms,
                      "energy": float(np.mean([x["energy"] for x in sts]))}
        E.close()
    per["mixed_vs_fp64"] = per["mixed"]["walker_steps_per_s"] / per["fp64"]["walker_steps_per_s"]
    per["config"] = "8 Z_eff=4 atoms, a=6.74 bohr, 32 electrons, 104 basis fns + images, Ewald, e-e-n Jastrow; " \
                    "16384 walkers, tau=0.005, 10-step blocks, median of 3 after one warm-up block"
    per["cpu_baseline"] = cpu_reference(os.path.abspath(cell.path), repeats=1, short_blocks=1, long_blocks=3,
                                        nconf=16, nstep=10, tau=0.005)
    out["periodic"] = per
    # twisted boundary conditions: the same cell with complex orbitals at
    # k = (0.5, 0.25, 0) on the complex-orbital kernels
    ccell = systems.write_periodic(tmp, seed=13, name="diamond8k_bench", kpoint=(0.5, 0.25, 0.0),
                                   complex_orbitals=True)
    cpx = {}
    for label, prec in (("fp64", engine.FP64), ("mixed", engine.MIXED)):
        E = engine.Engine(ccell.path, prec, max_walkers=16384, stream=stream.cuda_stream)
        E.set_walkers(Rc)
        E.vmc_block(5, 0.3, seed=SEED + 1)
        E.dmc_init(timestep=0.005, nstep=10, seed=SEED + 2)
        E.dmc_block()
        st = E.dmc_block()
        cpx[label] = {"walker_steps_per_s": 16384 * 10 / (st["block_ms"] / 1e3), "block_ms": st["block_ms"],
                      "energy": st["energy"]}
        E.close()
    cpx["mixed_vs_fp64"] = cpx["mixed"]["walker_steps_per_s"] / cpx["fp64"]["walker_steps_per_s"]
    cpx["vs_gamma_real_mixed"] = cpx["mixed"]["walker_steps_per_s"] / per["mixed"]["walker_steps_per_s"]
    cpx["config"] = "the periodic cell with complex orbitals (CORBITALS) at k=(0.5,0.25,0); 16384 walkers, " \
                    "tau=0.005, 10-step blocks"
    out["periodic_complex"] = cpx
    # HBM-resident kernels: the 72-electron molecule and the 128-electron cell
    # in mixed precision with the default move schedule, with the per-electron
    # tensor-core schedule forced on or off beside it, and in FP64
    def hbm_rates(deck_path, nw, tau, nstep, variants):
        R = systems.random_configs(systems.read_deck(deck_path), nw, seed=SEED % 1000)
        res = {}
        for label, prec, tc in variants:
            old_tc = os.environ.get("QWG_TC_MOVES")
            if tc is None:
                os.environ.pop("QWG_TC_MOVES", None)
            else:
                os.environ["QWG_TC_MOVES"] = tc
            try:
                E = engine.Engine(deck_path, prec, max_walkers=nw, stream=stream.cuda_stream)
            finally:
                if old_tc is None:
                    os.environ.pop("QWG_TC_MOVES", None)
                else:
                    os.environ["QWG_TC_MOVES"] = old_tc
            E.set_walkers(R)
            E.vmc_block(2, 0.1, seed=SEED + 3)
            E.dmc_init(timestep=tau, nstep=nstep, seed=SEED + 4)
            E.dmc_block()
            st = E.dmc_block()
            res[label] = {"walker_steps_per_s": nw * nstep / (st["block_ms"] / 1e3), "block_ms": st["block_ms"],
                          "energy": st["energy"]}
            E.close()
        return res

    m72 = os.path.join(ROOT, "tests", "golden", "mol72.qw")
    hm = hbm_rates(m72, 4096, 0.01, 5, (("mixed", engine.MIXED, None),
                                        ("mixed_tensor_core_moves", engine.MIXED, "1"),
                                        ("fp64", engine.FP64, None)))
    hm["mixed_vs_fp64"] = hm["mixed"]["walker_steps_per_s"] / hm["fp64"]["walker_steps_per_s"]
    hm["tensor_core_schedule_gain"] = (hm["mixed_tensor_core_moves"]["walker_steps_per_s"] /
                                       hm["mixed"]["walker_steps_per_s"])
    hm["config"] = ("mol72: 10 atoms, 72 electrons (36 per spin), 180 basis functions, HBM-resident kernels; 4096 "
                    "walkers, DMC tau=0.01, 5-step blocks; mixed = the default move schedule (one-launch CUDA-core "
                    "sweep below 16384 basis functions x orbitals), mixed_tensor_core_moves = the per-electron "
                    "tensor-core MO contraction (tcgen05 split TF32) forced on")
    out["hbm_molecule"] = hm
    c32 = os.path.join(ROOT, "tests", "golden", "cell32.qw")
    hc = hbm_rates(c32, 2048, 0.005, 5, (("mixed", engine.MIXED, None),
                                         ("mixed_cuda_core_moves", engine.MIXED, "0"),
                                         ("fp64", engine.FP64, None)))
    hc["mixed_vs_fp64"] = hc["mixed"]["walker_steps_per_s"] / hc["fp64"]["walker_steps_per_s"]
    hc["tensor_core_schedule_gain"] = hc["mixed"]["walker_steps_per_s"] / hc["mixed_cuda_core_moves"]["walker_steps_per_s"]
    hc["config"] = ("cell32: 32 Z_eff=4 atoms, 13.48x13.48x6.74 bohr, 128 electrons (64 per spin), 416 basis functions "
                    "+ images, HBM-resident kernels; 2048 walkers, DMC tau=0.005, 5-step blocks; mixed = the default "
                    "move schedule (per-electron tensor-core MO contraction), mixed_cuda_core_moves = the one-launch "
                    "CUDA-core sweep forced on")
    out["hbm_cell"] = hc
    # batched uneven molecules: 64 systems, 8-192 electrons, 512-4096 walkers
    mols = systems.write_batch(os.path.join(tmp, "batch"), nsys=64, seed=SEED % 1000)
    bat = {}
    for label, prec in (("fp64", engine.FP64), ("mixed", engine.MIXED)):
        engines = []
        for i, (d, nw) in enumerate(mols):
            E = engine.Engine(d.path, prec, max_walkers=nw)
            E.set_walkers(systems.random_configs(d, nw, seed=SEED + i))
            E.vmc_block(3, 0.3, seed=SEED + i)
            E.dmc_init(timestep=0.01, nstep=5, seed=SEED + 100 + i)
            engines.append(E)
        B = engine.Batch(engines)
        B.block()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        sts = B.block()
        wall = time.perf_counter() - t0
        ws = sum(s["nwalkers"] * s["nsteps"] for s in sts)
        bat[label] = {"walker_steps_per_s": ws / wall, "block_wall_ms": wall * 1e3}
        B.close()
        for E in engines:
            E.close()
    bat["mixed_vs_fp64"] = bat["mixed"]["walker_steps_per_s"] / bat["fp64"]["walker_steps_per_s"]
    bat["config"] = ("64 seeded molecules, 2-32 atoms Z_eff 1-6, electrons log-uniform 8-192 (" +
                     ",".join(str(d.nelec) for d, _ in mols) + "), 512-4096 walkers, one 5-step DMC block of "
                     "every system per graph launch; host wall time")
    out["batched"] = bat
    # serving: Poisson 2 jobs/s, bounded window
    jobs = serving.workload(os.path.join(tmp, "serve"), njobs=12, seed=SEED % 997, emin=16, emax=128)
    srv = {}
    for label, prec in (("fp64", engine.FP64), ("mixed", engine.MIXED)):
        r = serving.run(jobs, prec, budget_bytes=120 << 30, nstep=5, time_limit=seconds)
        r.pop("events")
        srv[label] = r
    srv["mixed_vs_fp64"] = srv["mixed"]["walker_steps_per_s"] / srv["fp64"]["walker_steps_per_s"]
    srv["config"] = (f"12 jobs, Poisson 2/s, seeded molecules and cells of 16-128 electrons, 1024-8192 "
                     f"walkers, 20-100 blocks of 5 steps, 120 GiB admission budget; first {seconds:.0f} s of the "
                     "stream (jobs still running at the limit are counted up to it)")
    out["serving"] = srv
    return out


def pp_cutoff(deck_text):
    """Radius beyond which every nonlocal channel of the deck's RGAUSSIAN
    OLDQMC pseudopotential is below 1e-5 (the scan of Pseudopotential::read:
    from 20 bohr down in 0.05 steps)."""
    body = re.search(r"OLDQMC\s*\{([^}]*)\}", deck_text).group(1).split()
    nl = int(body[1])
    nper = [int(x) for x in body[2:2 + nl]]
    terms, it = [], 2 + nl
    for n in nper:
        terms.append([(int(float(body[it + 3 * j])) - 2, float(body[it + 3 * j + 1]), float(body[it + 3 * j + 2]))
                      for j in range(n)])
        it += 3 * n
    r = 20.0
    while r > 0:
        if any(abs(sum(c * r ** k * np.exp(-a * r * r) for k, a, c in ch)) > 1e-5 for ch in terms[:-1]):
            return r
        r -= 0.05
    return 0.0


def cpu_reference(deck_path, repeats=3, short_blocks=1, long_blocks=9, cores=None, nconf=64, nstep=50, tau=None,
                  method="DMC"):
    """Reference qwalk (oracle/_ref/qwalk-Linux, shipped -O3 -ffast-math flags)
    on the host cores: one process per core, DMC (or VMC) on the same deck.
    Per-block cost from the difference of a short and a long run (removes
    start-up and the reference's own configuration generation); the pair is
    repeated and the fastest rate reported with the spread."""
    qw = os.path.join(ROOT, "oracle", "_ref", "qwalk-Linux")
    if not os.path.exists(qw):
        return None
    cores = cores or os.cpu_count() or 1
    tau = TAU if tau is None else tau
    base = open(deck_path).read()
    d = os.path.dirname(deck_path)

    stem = os.path.splitext(os.path.basename(deck_path))[0]

    def run(nblock, rep):
        # file names per deck: qwalk picks up <input>.config from an earlier run of the same name
        procs = []
        t0 = time.perf_counter()
        for p in range(cores):
            path = os.path.join(d, f"cpu_{stem}_{rep}_{nblock}_{p}.qw")
            txt = re.sub(r"RANDOMSEED\s*\{[^}]*\}", f"RANDOMSEED {{ {101 + p + 1000 * rep} {203 + p} }}", base)
            txt += (f"\nMETHOD {{ {method} NCONFIG {nconf} NBLOCK {nblock} NSTEP {nstep} TIMESTEP {tau} }}\n")
            open(path, "w").write(txt)
            procs.append(subprocess.Popen([qw, os.path.basename(path)], cwd=d, stdout=subprocess.DEVNULL,
                                          stderr=subprocess.DEVNULL))
        codes = [p.wait() for p in procs]
        if any(codes):
            raise RuntimeError(f"reference qwalk exited with status {max(codes, key=abs)} on {stem}")
        return time.perf_counter() - t0

    rates, walls = [], []
    for rep in range(repeats):
        try:
            ts, tl = run(short_blocks, rep), run(long_blocks, rep)
        except RuntimeError:
            return None
        if not tl > ts + 0.05:  # the longer run must take longer: anything else is a failed run
            return None
        per_block = max((tl - ts) / (long_blocks - short_blocks), 1e-6)
        rates.append(cores * nconf * nstep / per_block)
        walls.append((round(ts, 1), round(tl, 1)))
    # the host is shared with other jobs: contention only slows a run, so the
    # fastest repeat is the reference's own speed
    return {"value": float(np.max(rates)), "unit": "walker-steps/s", "cores": cores, "kind": "reference",
            "repeats": [float(r) for r in rates],
            "spread": float((max(rates) - min(rates)) / np.median(rates)),
            "sample": f"{cores} qwalk processes x {nconf} walkers x {nstep} {method} steps/block; per-block time from "
                      f"{long_blocks}-block minus {short_blocks}-block wall, {repeats} repeats (walls s: {walls}); "
                      "the fastest repeat reported"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--latency-blocks", type=int, default=12)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="only the headline workload")
    ap.add_argument("--precision", default="both", choices=["both", "mixed", "fp64"],
                    help="arms of the headline workload (profiling runs use one)")
    ap.add_argument("--probe", default=None,
                    help="profiling driver only, no report line: tc-sweep = one mixed-precision sweep of the "
                         "72-electron molecule (4096 walkers) on the tensor-core move schedule (forced on); "
                         "branch:<deck>:<walkers> = two mixed-precision DMC blocks of 5 steps of a golden deck "
                         "(population control share)")
    args = ap.parse_args()
    if args.probe and args.probe.startswith("phases:"):
        # walker-kernel phase counters of the profiling library (built by
        # python -m mainline_b200.build --phases): DMC blocks of a golden deck
        os.environ["QWG_LIBRARY"] = os.path.join(ROOT, "mainline_b200", "libqwg_phases.so")
        from mainline_b200 import engine, systems
        _, name, nw = args.probe.split(":")
        deck = os.path.join(ROOT, "tests", "golden", name + ".qw")
        nw = int(nw)
        out = {"deck": name, "walkers": nw}
        for label, prec in (("mixed", engine.MIXED), ("fp64", engine.FP64)):
            E = engine.Engine(deck, prec, max_walkers=nw)
            E.set_walkers(systems.random_configs(systems.read_deck(deck), nw, seed=1))
            E.vmc_block(2, 0.1, seed=2)
            E.dmc_init(timestep=0.01, nstep=10, seed=3)
            E.dmc_block()
            E.phase_counters(reset=True)
            st = E.dmc_block()
            ph = E.phase_counters()
            ws = nw * 10
            out[label] = {"block_ms": st["block_ms"],
                          "cycles_per_walker_step": {k: round(v / ws) for k, v in ph.items()}}
            E.close()
        print(json.dumps(out))
        return
    if args.probe and args.probe.startswith("branch:"):
        from mainline_b200 import engine, systems
        _, name, nw = args.probe.split(":")
        deck = os.path.join(ROOT, "tests", "golden", name + ".qw")
        nw = int(nw)
        E = engine.Engine(deck, engine.MIXED, max_walkers=nw)
        E.set_walkers(systems.random_configs(systems.read_deck(deck), nw, seed=1))
        E.vmc_block(2, 0.1, seed=2)
        E.dmc_init(timestep=0.01, nstep=5, seed=3)
        for _ in range(2):
            st = E.dmc_block()
        print("branch probe", name, nw, "block ms", st["block_ms"])
        E.close()
        return
    if args.probe == "tc-sweep":
        from mainline_b200 import engine, systems
        deck = os.path.join(ROOT, "tests", "golden", "mol72.qw")
        os.environ["QWG_TC_MOVES"] = "1"  # below the schedule's size rule: forced on
        E = engine.Engine(deck, engine.MIXED, max_walkers=NWALK)
        E.set_walkers(systems.random_configs(systems.read_deck(deck), NWALK, seed=1))
        E.set_vmc_dynamics(1, 2.0)
        print("tc-sweep acceptance", E.vmc_block(1, 0.1, seed=2)["acceptance"])
        E.close()
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))

    if args.impl == "reference":
        if rank != 0:
            return
        tmp = tempfile.mkdtemp(prefix="qwg_ref_")
        deck, _ = make_workload(tmp)
        ref = cpu_reference(deck.path)
        if ref is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/qwalk-Linux was not built"}))
            return
        line = {"impl": "reference", "metric": "DMC walker-steps/s", "value": ref["value"],
                "unit": "walker-steps/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
                "higher_is_better": True, "dtype": "f64", "data": "synthetic (seeded deck)",
                "config": {"workload": "n2_pseudo: 2 Z_eff=5 atoms, 14 e, 80 basis fns, tau=0.01"},
                "cpu_baseline": ref,
                "e2e": {"value": ref["value"], "unit": "walker-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", rank)))
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    results, e2e, corr, deck = run_engine(args, rank, world)
    if args.precision != "both":  # profiling run: no report line
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    mx = results["mixed"]
    fp = results["fp64"]
    steps = mx["steps"]
    # max over ranks of the device times (every rank takes part)
    ms, ms64, e2e_ms, e2e64_ms = max_over_ranks([mx["ms"], fp["ms"], e2e["mixed"], e2e["fp64"]], "cuda")
    ws = aggregate_rate(NWALK * steps, world, ms)
    ws64 = aggregate_rate(NWALK * fp["steps"], world, ms64)
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    N, M, nb = 14, 7, 80
    hbm, src = _peaks()
    # dominant kernel: the move kernel (one launch = one sweep of every
    # walker); algorithmic bytes per launch = walkers x resident state read +
    # written once.  The local-energy kernel reads the state and writes 16 B.
    sb = walker_state_bytes(N, M, 4)
    kern = {"sweep": (mx["sweep_ms"], NWALK * 2 * sb), "eloc": (mx["eloc_ms"], NWALK * (sb + 16))}
    dom = max(kern, key=lambda k: kern[k][0])
    kern_ms_per_launch, bytes_launch = kern[dom]
    achieved = bytes_launch / (kern_ms_per_launch / 1e3) / 1e9
    flops = move_flops_per_walker(N, M, nb, natoms=2, k_ee=1, k_en=4)
    pcut = pp_cutoff(open(deck.path).read())
    npairs = pp_pairs(results["mixed"]["R"], ATOMS, pcut)
    pp_flops = pp_flops_per_walker(npairs, N, M, nb, natoms=2, k_ee=1, k_en=4)
    tflops_peak, tsrc = _tensor_peak()
    lat = np.array(mx["lat"])
    e2e_h2d = NWALK * N * 3 * 8 / steps
    e2e_d2h = (NWALK * N * 3 * 8 + 96) / steps
    line = {
        "metric": "DMC walker-steps/s",
        "value": ws, "unit": "walker-steps/s", "n_gpus": world, "steps": steps, "warmup": args.warmup,
        "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32/f64 mixed (FP64 refresh, energies, weights)", "data": "synthetic (seeded QWalk deck)",
        "precision": "mixed (the FP64 arm is the fp64 object)",
        "config": {"workload": "n2_pseudo DMC: 2 Z_eff=5 atoms, 14 electrons, 80 basis fns, 12-pt quadrature",
                   "walkers_per_gpu": NWALK, "tau": TAU, "feedback_interval": FEEDBACK_INTERVAL,
                   "basis_exponents": "log-uniform in [0.1, 10] (valence range); the configuration text's "
                                      "[0.1, 1e4] is the all-electron range, with which the reference's own DMC "
                                      "diverges on the random-orbital trial function",
                   "parallelism": f"replicas x{world}", "l2": "walker state resident (working set < L2); "
                   "256 MiB buffer written before the timed block"},
        "fp64": {"value": ws64, "unit": "walker-steps/s", "ms_per_step": ms64 / fp["steps"],
                 "e2e": {"value": aggregate_rate(NWALK * steps, world, e2e64_ms), "unit": "walker-steps/s",
                         "h2d_bytes_per_step": e2e_h2d, "d2h_bytes_per_step": e2e_d2h},
                 "block_energy_mean": float(np.mean(fp["energies"])),
                 "block_energy_sem": float(np.std(fp["energies"]) / np.sqrt(len(fp["energies"])))},
        "mixed_vs_fp64": ws / ws64,
        "mixed_block_energy": {"mean": float(np.mean(mx["energies"])),
                               "sem": float(np.std(mx["energies"]) / np.sqrt(len(mx["energies"])))},
        "mixed_minus_fp64_mHa": corr,
        "block_latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                             "steps_per_block": 20, "walkers": NWALK},
        "e2e": {"value": aggregate_rate(NWALK * steps, world, e2e_ms), "unit": "walker-steps/s",
                "h2d_bytes_per_step": e2e_h2d, "d2h_bytes_per_step": e2e_d2h},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_source": src, "traffic": _traffic_per_launch(dom),
                     "kernel": {"sweep": "k_walkers<float,8,KM_SWEEP>", "eloc": "k_walkers<float,8,KM_ELOC>"}[dom],
                     "kernel_ms": {"sweep": mx["sweep_ms"], "eloc": mx["eloc_ms"]},
                     "algorithmic_bytes_per_launch": bytes_launch,
                     "note": "per launch every walker's resident state is read (and, for the move kernel, "
                             "written) once; the state fits L2, so the kernel is latency/issue-bound, not HBM-bound"},
        "roofline_compute": {
            "sweep": {"algorithmic_flops_per_launch": NWALK * flops,
                      "achieved_tflops": NWALK * flops / (mx["sweep_ms"] / 1e3) / 1e12},
            "eloc": {"algorithmic_flops_per_launch": NWALK * pp_flops, "pp_pairs_per_walker": npairs,
                     "pp_cutoff_bohr": pcut, "achieved_tflops": NWALK * pp_flops / (mx["eloc_ms"] / 1e3) / 1e12},
            "tensor_peak_tflops": tflops_peak, "tensor_peak_source": tsrc,
            "fp32_cuda_core_peak_tflops": FP32_SPEC_TFLOPS,
            "fp32_peak_source": "spec arithmetic (148 SMs x 128 FP32 lanes x 2 x 1.965 GHz), not measured",
            "note": "flops from the per-walker-step formulas of the path (MO products, ratios, Sherman-Morrison, "
                    "Jastrow; pseudopotential quadrature with the measured pair count); the kernels issue their "
                    "work on CUDA cores and are issue-bound (ncu issue slots ~48% / 34% busy)"},
        "gpu_launches": mx["launches"],
        "clocks": mx["clocks"],
    }
    for k in ("sweep", "eloc"):
        a = line["roofline_compute"][k]["achieved_tflops"]
        line["roofline_compute"][k]["frac_of_tensor_peak"] = a / tflops_peak
        line["roofline_compute"][k]["frac_of_fp32_peak"] = a / FP32_SPEC_TFLOPS
    if not args.no_extras and world == 1:
        import torch
        dev = torch.device("cuda", 0)
        line["workloads"] = run_extras(torch.cuda.Stream(device=dev), dev)
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_reference(os.path.abspath(deck.path))
    print(json.dumps(line))


if __name__ == "__main__":
    main()
