"""One CPU rank of tests/test_replicas_gloo.py (run as a subprocess with
RANK, WORLD_SIZE, MASTER_ADDR and MASTER_PORT set): gathers the replica
energies over gloo and prints its exchange result as JSON."""
import json
import os
import sys
from datetime import timedelta

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import numpy as np
import torch.distributed as dist

from molmodel_b200.replicas import exchange_labels, gather_energies, lpt_partition

SIZES = [256, 4096, 1024, 512, 2048, 300]


def main():
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    temps = {i: 280.0 * (450.0 / 280.0) ** (i / 5) for i in range(len(SIZES))}
    mine = lpt_partition(SIZES, world)[rank]
    local = {rid: -10.0 * SIZES[rid] - rid for rid in mine}
    energies = gather_energies(local)
    uni = np.random.default_rng(11).uniform(size=len(SIZES) - 1)
    new, n = exchange_labels(temps, energies, uni)
    dist.barrier()
    dist.destroy_process_group()
    print(json.dumps(dict(rank=rank, mine=mine, energies=sorted(energies.items()), temps=sorted(new.items()),
                          accepted=n)))


if __name__ == "__main__":
    main()
