"""Hamiltonian parameter scan: many independent XXZ chains of uneven length and
bond dimension solved concurrently on one GPU (and sharded over ranks).

Each worker thread owns a Context (its own CUDA stream and scratch) and takes
instances from a shared queue; the library releases the GIL during its calls,
so the workers' launch streams overlap on the device.  The chains never
exchange data: across GPUs the instances are partitioned by rank with no
collective on the data path.

Instance model (the measurement plan's XXZ scan):
    H = sum_i [Jxy (Sx Sx + Sy Sy) + Jz Sz Sz] - hz sum_i Sz,  S = 1/2, open,
Jxy = 1, Jz ~ U[-0.5, 1.5], hz ~ U[0, 0.5], L ~ U{32..96}, D ~ U{32, 64, 128}.
The reference's MPO adds +hz Sz (Hamiltonian_1D_NN_Heisenberg.C:35-79), so the
field coefficient passed on is -hz.
"""
from __future__ import annotations

import queue
import threading
import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import api


@dataclass
class ScanInstance:
    L: int
    D: int
    Jxy: float
    Jz: float
    hz: float
    seed: int


@dataclass
class ScanResult:
    instance: ScanInstance
    energy_per_site: float
    variance: float
    seconds: float
    matvecs: int
    worker: int


def make_xxz_scan(n: int = 64, seed: int = 777, Lmin: int = 32, Lmax: int = 96,
                  Ds=(32, 64, 128)) -> List[ScanInstance]:
    """The scan's instances from a seeded generator (numpy default_rng(seed))."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        out.append(ScanInstance(L=int(rng.integers(Lmin, Lmax + 1)), D=int(rng.choice(Ds)), Jxy=1.0,
                                Jz=float(rng.uniform(-0.5, 1.5)), hz=float(rng.uniform(0.0, 0.5)),
                                seed=int(seed * 1000 + i)))
    return out


def schedule_lines(D: int, sweeps: int = 2, Dstart: int = 16):
    """(max_sweeps, Dmax, deltaD) lines doubling D from Dstart to D."""
    lines, d = [], min(Dstart, D)
    lines.append((sweeps, d, d))
    while d < D:
        nd = min(2 * d, D)
        lines.append((sweeps, nd, nd - d))
        d = nd
    return lines


def solve(ctx: api.Context, inst: ScanInstance, options: api.SolverOptions, eps_eigen: float = 1e-10,
          sweeps: int = 2, dstart: int = 16) -> dict:
    """Factory -> Hamiltonian -> MPS::FindVariationalGroundState for one instance."""
    f = api.Factory(ctx)
    H = f.Make1D_NN_HeisenbergHamiltonian(inst.L, 0.5, api.RegularLower, inst.Jxy, inst.Jz, -inst.hz)
    lines = schedule_lines(inst.D, sweeps, dstart)
    psi = H.CreateMPS(lines[0][1], 1e-12, 1e-12)
    psi.InitializeWith(api.Random, seed=inst.seed)
    sched = api.IterationSchedule()
    for (ms, Dm, dD) in lines:
        eps = api.Epsilons(1e-12)
        eps.itsEigenSolverEpsilon = eps_eigen
        sched.Insert(api.IterationScheduleLine(ms, Dm, dD, eps))
    var = psi.FindVariationalGroundState(H, sched, options)
    E = psi.GetExpectation(H)
    return {"energy_per_site": E / inst.L, "variance": var, "matvecs": psi.last_stats["matvecs"]}


def run_scan(instances: List[ScanInstance], workers: int = 8, device: int = 0,
             options: Optional[api.SolverOptions] = None, eps_eigen: float = 1e-10,
             sweeps: int = 2, dstart: int = 16) -> tuple:
    """Solve every instance with `workers` concurrent contexts; returns
    (results in instance order, wall seconds)."""
    options = options or api.SolverOptions(precision=api.MIXED)
    q: "queue.Queue[int]" = queue.Queue()
    for i in range(len(instances)):
        q.put(i)
    results: List[Optional[ScanResult]] = [None] * len(instances)
    errors: List[BaseException] = []

    def work(w: int):
        try:
            ctx = api.Context(device)
            while True:
                try:
                    i = q.get_nowait()
                except queue.Empty:
                    break
                t0 = time.perf_counter()
                r = solve(ctx, instances[i], options, eps_eigen, sweeps, dstart)
                results[i] = ScanResult(instances[i], r["energy_per_site"], r["variance"],
                                        time.perf_counter() - t0, r["matvecs"], w)
            ctx.synchronize()
        except BaseException as e:  # pragma: no cover - surfaced below
            errors.append(e)

    t0 = time.perf_counter()
    threads = [threading.Thread(target=work, args=(w,)) for w in range(max(1, workers))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    wall = time.perf_counter() - t0
    if errors:
        raise errors[0]
    return results, wall
