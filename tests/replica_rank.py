"""One CPU rank of tests/test_replicas_gloo.py (run as a subprocess with
RANK, WORLD_SIZE, MASTER_ADDR and MASTER_PORT set; WORLD_SIZE 1 runs without
a process group): the full replica-exchange loop of molmodel_b200.remd on small
water replicas of uneven size, energies from the oracle, prints the
temperature history and the final energies as JSON."""
import json
import os
import sys
from datetime import timedelta

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import numpy as np

from molmodel_b200.remd import ReplicaExchange, run_exchange, temperature_ladder
from molmodel_b200.water import splitmix64_uniform, water_box_n
from oracle.oracle import make_config, port

SIZES = [40, 64, 50, 80, 45, 70]
BLOCKS, INTERVAL = 4, 10


def main():
    rank, world = int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    exch = ReplicaExchange([3 * s for s in SIZES], temperature_ladder(len(SIZES)), rank, world, device="cpu")
    reps = {}
    for rid in exch.mine:
        wb = water_box_n(SIZES[rid], seed=100 + rid)
        o = port().eleclj(make_config(wb.box, rspace_cutoff=0.0, ewald_screening=-1.0, kspace_cutoff=5.0),
                          wb.nsite, wb.groups, wb.exclusions, wb.site_mask, wb.q, wb.sigma, wb.epsilon, wb.rscreen)
        reps[rid] = dict(wb=wb, o=o, r=wb.positions.copy(), v=1.0, block=0)

    def advance(nsteps):
        # a stand-in for the dynamics: every molecule moved rigidly by a seeded
        # step whose size follows the replica's velocity scale
        out = {}
        for rid, st in reps.items():
            n = len(st["r"]) // 3
            u = splitmix64_uniform(7919 * rid + st["block"], 3 * n).reshape(n, 3) - 0.5
            st["r"] = (st["r"].reshape(n, 3, 3) + 0.01 * nsteps * st["v"] * u[:, None, :]).reshape(-1, 3)
            st["block"] += 1
            out[rid] = st["o"].eval(st["r"])["total"]
        return out

    def scale(rid, f):
        reps[rid]["v"] *= f

    history = run_exchange(exch, advance, scale, BLOCKS, INTERVAL)
    energies = {rid: st["o"].eval(st["r"])["total"] for rid, st in reps.items()}
    if world > 1:
        from molmodel_b200.replicas import gather_energies
        energies = gather_energies(energies)
        dist.barrier()
        dist.destroy_process_group()
    print(json.dumps(dict(rank=rank, mine=exch.mine, history=[sorted(h.items()) for h in history],
                          energies=sorted(energies.items()), accepted=exch.accepted, attempts=exch.attempts)))


if __name__ == "__main__":
    main()
