"""Batched replica exchange of water boxes of uneven size (the C4 workload).

64 replicas, water counts log-uniform on [256, 4096] (seed 4), each its own
box at 0.997 g/cm^3 with P3M at ~1.04 A spacing (order 5), rc 9 A, skin 1.5 A
(clipped by the library when the box is small), temperatures geometric from
280 to 450 K, 2 fs steps, an exchange attempt every 500 steps.  All replicas
advance together: one CUDA graph launch per step with a branch per replica
(mmnb_md_batch).  The exchange follows MDyn::try_replica_exchange's rule
(src/mdyn.cpp:317-351) with temperature labels swapped (replicas differ in
size) and velocities rescaled by sqrt(T_new / T_old); its uniforms come from a
seeded stream, so a run is reproducible.

  python -m molmodel_b200.replica_bench [--replicas 64] [--steps 1000] [--interval 500]
"""
import argparse
import json
import math
import time

import numpy as np

from . import ElecLJ, maxwell_boltzmann, water_box_n
from .md import MDyn, ReplicaBatch
from .replicas import exchange_labels
from .water import splitmix64_uniform


def replica_sizes(n, seed=4, lo=256, hi=4096):
    u = splitmix64_uniform(seed, n)
    return [int(round(math.exp(math.log(lo) + x * (math.log(hi) - math.log(lo))))) for x in u]


def temperatures(n, tmin=280.0, tmax=450.0):
    return [tmin * (tmax / tmin) ** (i / max(1, n - 1)) for i in range(n)]


def build(n, precision="mixed", dt=0.002, seed=4):
    sizes = replica_sizes(n, seed)
    temps = temperatures(n)
    reps = []
    for i, (nw, t) in enumerate(zip(sizes, temps)):
        wb = water_box_n(nw, seed=1000 * seed + i)
        pot = ElecLJ(precision=precision, rspace_cutoff=9.0, ewald_screening=0.35, neighbor_list_width=1.5,
                     use_p3m=True, p3m_grid_spacing=1.04, p3m_assignment_order=5).init(wb)
        md = MDyn(pot, wb.masses, timestep=dt)
        md.set_state(wb.positions, maxwell_boltzmann(wb, t, seed=2000 * seed + i))
        reps.append((wb, pot, md))
    return sizes, dict(enumerate(temps)), reps


def run_exchange(batch, reps, temps, steps, interval, seed=4):
    """steps in blocks of `interval`, an exchange attempt after each block."""
    nrep = len(reps)
    accepted = attempts = 0
    k = 0
    for _ in range(steps // interval):
        e = batch.run(interval)
        energies = {i: float(e[i][-1, 1]) for i in range(nrep)}
        uni = splitmix64_uniform(seed ^ 0xE7C4, nrep - 1, offset=k * (nrep - 1))
        k += 1
        new, acc = exchange_labels(temps, energies, uni)
        for i in range(nrep):
            if new[i] != temps[i]:
                reps[i][2].scale_velocities(math.sqrt(new[i] / temps[i]))
        temps = new
        accepted += acc
        attempts += nrep - 1
    return temps, accepted, attempts


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--replicas", type=int, default=64)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--interval", type=int, default=500)
    ap.add_argument("--precision", default="mixed")
    ap.add_argument("--no-sequential", action="store_true")
    ap.add_argument("--autotune", action="store_true", help="tune each replica's launch choices first")
    args = ap.parse_args()
    sizes, temps, reps = build(args.replicas, args.precision)
    tunings = None
    if args.autotune:
        tunings = [pot.autotune(wb.positions, iters=5) for wb, pot, _ in reps]
    batch = ReplicaBatch([r[2] for r in reps])
    batch.run(20)  # warm-up (graph capture)
    t0 = time.perf_counter()
    temps, acc, att = run_exchange(batch, reps, temps, args.steps, args.interval)
    t_batch = time.perf_counter() - t0
    nsite = sum(3 * s for s in sizes)
    out = dict(workload=f"{args.replicas} replicas, {min(sizes)}..{max(sizes)} waters ({sum(sizes)} total), "
                        f"P3M ~1.04 A order 5, rc 9 A, 2 fs, exchange every {args.interval} steps",
               precision=args.precision, steps=args.steps, batched_s=t_batch,
               replica_steps_per_s=args.replicas * args.steps / t_batch,
               site_steps_per_s=nsite * args.steps / t_batch,
               exchange_acceptance=acc / max(1, att))
    if tunings is not None:
        out["tunings"] = {str(t): tunings.count(t) for t in sorted(set(tunings))}
    if not args.no_sequential:
        # the same replicas, each advanced by its own graph in turn (no batching)
        t0 = time.perf_counter()
        for _, _, md in reps:
            md.run(args.steps // 4)
        t_seq = (time.perf_counter() - t0) * 4
        out.update(sequential_s_estimate=t_seq, batching_speedup=t_seq / t_batch)
    batch.close()
    for _, pot, md in reps:
        md.close()
        pot.close()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
