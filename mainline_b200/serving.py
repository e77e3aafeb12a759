"""Serving workload and driver for the continuous-batching DMC job server.

The server itself is native (include/qwg_server.h, csrc/qwg_server.cpp);
this module draws a seeded Poisson stream of DMC jobs and drives the server
in real time, reporting throughput and per-block latency percentiles.

Workload (the serving configuration): jobs arrive as a Poisson process
(mean ``rate`` jobs/s); each job is a seeded molecule (Z_eff 1-6 pseudo-atoms)
or a periodic cell of the 8-atom Z_eff=4 family (supercells of 1, 4 or 8
cells: 32, 128 or 256 electrons) with electron counts log-uniform in
[emin, emax], 1024-8192 walkers and 20-100 blocks (log-uniform).
"""
from __future__ import annotations

import os
import time
from dataclasses import dataclass

import numpy as np

from . import engine, systems

# electrons of the neutral cell -> supercell repeats of the 8-atom, 32-electron
# cell; (2, 2, 2) is the 64-atom cell with a = 13.48 bohr and 832 basis
# functions (64 atoms of Z_eff 4: 128 up, 128 down electrons)
CELL_SIZES = {32: (1, 1, 1), 128: (2, 2, 1), 256: (2, 2, 2)}


@dataclass
class Job:
    arrival: float          # seconds after the start of the stream
    deck: systems.Deck
    walkers: int
    blocks: int
    seed: int


def workload(outdir: str, njobs: int = 20, rate: float = 2.0, seed: int = 2024, emin: int = 16, emax: int = 512,
             wmin: int = 1024, wmax: int = 8192, bmin: int = 20, bmax: int = 100, cell_fraction: float = 0.25):
    """Seeded job stream; decks are written to outdir (one per job)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    jobs = []
    for i in range(njobs):
        t += rng.exponential(1.0 / rate)
        ne = int(round(np.exp(rng.uniform(np.log(emin), np.log(emax)))))
        cells = [n for n in CELL_SIZES if emin <= n <= emax]
        if cells and rng.uniform() < cell_fraction:
            n = min(cells, key=lambda c: abs(np.log(c / ne)))
            deck = systems.write_periodic(outdir, seed=seed * 100 + i, name=f"job{i:03d}_cell{n}e",
                                          supercell=CELL_SIZES[n])
        else:
            ne = min(ne, 6 * 32)  # 32 atoms of Z_eff <= 6
            deck = systems.write_molecule(outdir, f"job{i:03d}_mol{ne}e", seed * 100 + i, ne)
        w = int(round(np.exp(rng.uniform(np.log(wmin), np.log(wmax)))))
        b = int(round(np.exp(rng.uniform(np.log(bmin), np.log(bmax)))))
        jobs.append(Job(arrival=t, deck=deck, walkers=w, blocks=b, seed=seed * 1000 + i))
    return jobs


def run(jobs, precision: int, budget_bytes: int, nstep: int = 5, timestep: float = 0.01, max_active: int = 0,
        vmc_blocks: int = 1, vmc_steps: int = 5, poll_s: float = 2e-4, time_limit: float | None = None) -> dict:
    """Submit each job at its arrival time and drive the server until every
    job has finished (or time_limit seconds have passed).  Returns the block
    events and the summary: DMC walker-steps/s over the run, block latency
    p50/p99 (enqueue -> statistics on the host)."""
    srv = engine.Server(budget_bytes, max_active)
    events = []
    nxt = 0
    t0 = time.perf_counter()
    try:
        while True:
            now = time.perf_counter() - t0
            while nxt < len(jobs) and jobs[nxt].arrival <= now:
                j = jobs[nxt]
                R = systems.random_configs(j.deck, j.walkers, seed=j.seed)
                srv.submit(j.deck.path, R, precision, j.blocks,
                           dict(timestep=timestep, nstep=nstep, seed=j.seed + 7),
                           vmc_blocks=vmc_blocks, vmc_steps=vmc_steps, vmc_timestep=0.3, vmc_seed=j.seed + 3)
                nxt += 1
            ev = srv.progress()
            events += ev
            st = srv.status()
            if nxt == len(jobs) and st["queued"] == 0 and st["active"] == 0:
                break
            if time_limit is not None and now > time_limit:
                break
            if not ev:
                time.sleep(poll_s)
        wall = time.perf_counter() - t0
        st = srv.status()
    finally:
        srv.close()
    lat = np.array([e["latency_ms"] for e in events]) if events else np.zeros(1)
    return dict(events=events, wall_s=wall, walker_steps=st["walker_steps"],
                walker_steps_per_s=st["walker_steps"] / wall, blocks=len(events), finished=st["finished"],
                failed=st["failed"], latency_p50_ms=float(np.percentile(lat, 50)),
                latency_p99_ms=float(np.percentile(lat, 99)))
