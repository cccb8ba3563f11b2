"""Batched replica exchange of water boxes of uneven size (the C4 workload).

64 replicas, water counts log-uniform on [256, 4096] (seed 4), each its own
box at 0.997 g/cm^3 with P3M at ~1.04 A spacing (order 5), rc 9 A, skin 1.5 A
(clipped by the library when the box is small), temperatures geometric from
280 to 450 K, 2 fs steps, an exchange attempt every 500 steps.  On each GPU
the replicas it owns advance together: one CUDA graph launch per step with a
branch per replica (mmnb_md_batch).  The exchange follows
MDyn::try_replica_exchange's rule (src/mdyn.cpp:317-351) with temperature
labels swapped (replicas differ in size) and velocities rescaled by
sqrt(T_new / T_old); its uniforms come from a seeded stream, so a run is
reproducible.  Under torchrun (one process per GPU, NCCL) the replicas are
spread over the ranks by longest processing time on their site counts and the
ranks meet once per exchange (molmodel_b200.remd.ReplicaExchange).

  python -m molmodel_b200.replica_bench [--replicas 64] [--steps 1000] [--interval 500] [--merged]
  torchrun --nproc-per-node N -m molmodel_b200.replica_bench ...
"""
import argparse
import json
import math
import os
import time

import numpy as np

from . import ElecLJ, maxwell_boltzmann, water_box_n
from .md import MDyn, ReplicaBatch
from .remd import ReplicaExchange, replica_sizes, run_exchange, temperature_ladder


def temperatures(n, tmin=280.0, tmax=450.0):
    return temperature_ladder(n, tmin, tmax)


def build(n, precision="mixed", dt=0.002, seed=4, ids=None):
    """The replicas `ids` (default: all) of the n-replica set."""
    sizes = replica_sizes(n, seed)
    temps = temperatures(n)
    reps = {}
    for i in (range(n) if ids is None else ids):
        wb = water_box_n(sizes[i], seed=1000 * seed + i)
        pot = ElecLJ(precision=precision, rspace_cutoff=9.0, ewald_screening=0.35, neighbor_list_width=1.5,
                     use_p3m=True, p3m_grid_spacing=1.04, p3m_assignment_order=5).init(wb)
        md = MDyn(pot, wb.masses, timestep=dt)
        md.set_state(wb.positions, maxwell_boltzmann(wb, temps[i], seed=2000 * seed + i))
        reps[i] = (wb, pot, md)
    return sizes, temps, reps


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--replicas", type=int, default=64)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--interval", type=int, default=500)
    ap.add_argument("--precision", default="mixed")
    ap.add_argument("--no-sequential", action="store_true")
    ap.add_argument("--autotune", action="store_true", help="tune each replica's launch choices first")
    ap.add_argument("--merged", action="store_true",
                    help="also time one box holding all the replicas' waters (the bound a single fused launch "
                         "over the replicas could approach)")
    args = ap.parse_args()
    import torch
    rank, world = int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    sizes = replica_sizes(args.replicas)
    exch = ReplicaExchange([3 * s for s in sizes], temperatures(args.replicas), rank, world,
                           device=f"cuda:{local}")
    _, _, reps = build(args.replicas, args.precision, ids=exch.mine)
    tunings = None
    if args.autotune:
        tunings = [pot.autotune(wb.positions, iters=5) for wb, pot, _ in reps.values()]
    ids = sorted(reps)
    batch = ReplicaBatch([reps[i][2] for i in ids])
    batch.run(20)  # warm-up (graph capture)

    def advance(nsteps):
        e = batch.run(nsteps)
        return {rid: float(e[k][-1, 1]) for k, rid in enumerate(ids)}

    def scale(rid, f):
        reps[rid][2].scale_velocities(f)

    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    run_exchange(exch, advance, scale, args.steps // args.interval, args.interval)
    ev1.record()
    torch.cuda.synchronize()
    t = torch.tensor([ev0.elapsed_time(ev1) / 1e3], dtype=torch.float64, device=f"cuda:{local}")
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    t_batch = float(t.item())
    nsite = sum(3 * s for s in sizes)
    steps = (args.steps // args.interval) * args.interval
    out = dict(workload=f"{args.replicas} replicas, {min(sizes)}..{max(sizes)} waters ({sum(sizes)} total), "
                        f"P3M ~1.04 A order 5, rc 9 A, 2 fs, exchange every {args.interval} steps",
               precision=args.precision, steps=steps, ranks=world, batched_s=t_batch,
               replica_steps_per_s=args.replicas * steps / t_batch,
               site_steps_per_s=nsite * steps / t_batch,
               exchange_acceptance=exch.accepted / max(1, exch.attempts * (args.replicas - 1)),
               timing="CUDA events around the exchange loop, max over ranks")
    if tunings is not None:
        out["tunings"] = {str(tt): tunings.count(tt) for tt in sorted(set(tunings))}
    if not args.no_sequential and world == 1:
        # the same replicas, each advanced by its own graph in turn (no batching)
        t0 = time.perf_counter()
        for i in ids:
            reps[i][2].run(args.steps // 4)
        t_seq = (time.perf_counter() - t0) * 4
        out.update(sequential_s_estimate=t_seq, batching_speedup=t_seq / t_batch)
    batch.close()
    for _, pot, md in reps.values():
        md.close()
        pot.close()
    if args.merged and world == 1:
        # one box with the same total number of waters and the same settings:
        # every kernel of a step is one launch over all of them, so its
        # water-steps per second bound what fusing the replicas' launches
        # into persistent kernels could reach
        total = sum(sizes)
        wb = water_box_n(total, seed=77)
        pot = ElecLJ(precision=args.precision, rspace_cutoff=9.0, ewald_screening=0.35, neighbor_list_width=1.5,
                     use_p3m=True, p3m_grid_spacing=1.04, p3m_assignment_order=5).init(wb)
        md = MDyn(pot, wb.masses, timestep=0.002)
        md.set_state(wb.positions, maxwell_boltzmann(wb, 300.0, seed=78))
        md.run(20)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        md.run(steps)
        e1.record()
        torch.cuda.synchronize()
        t_m = e0.elapsed_time(e1) / 1e3
        out.update(merged_waters=total, merged_s=t_m, merged_water_steps_per_s=total * steps / t_m,
                   batch_water_steps_per_s=total * steps / t_batch, batch_over_merged=t_m / t_batch)
        md.close()
        pot.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
