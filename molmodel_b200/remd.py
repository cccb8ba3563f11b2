"""Replica exchange across ranks: MDyn::try_replica_exchange (src/mdyn.cpp:317-351)
for replicas spread over GPUs, one process per GPU.

The reference runs one MPI rank per replica and, at an exchange, sends
potential energies up and down the temperature ladder and swaps coordinates
between equal systems.  Here each rank owns a set of replicas (longest
processing time on their cost, replicas.lpt_partition) and advances them
without any collective on the data path; every exchange interval the ranks
make ONE all-gather of (replica id, temperature, potential energy) -- a fixed
[width, 3] float64 tensor per rank, on the GPU under NCCL or on the CPU under
gloo -- and every rank then runs the same Metropolis pass
(replicas.exchange_labels) on the same seeded uniform numbers, so all ranks
reach the same temperature assignment without further messages.  Replicas of
different sizes swap temperature labels (the same move as swapping the
coordinates of equal systems); a replica whose temperature changed has its
velocities multiplied by sqrt(T_new / T_old) (mmnb_md_scale_velocities).
"""
import math

import numpy as np

from .replicas import exchange_labels, lpt_partition
from .water import splitmix64_uniform


class ReplicaExchange:
    """Temperature bookkeeping of one rank.

    costs: per replica (all ranks pass the same list), e.g. its site count;
    temperatures: per replica, K; rank, world: this process and the number
    of processes; device: where the gathered tensor lives ("cuda:k" under
    NCCL, "cpu" under gloo or without torch.distributed); seed: the stream of
    uniform numbers (the same on every rank)."""

    def __init__(self, costs, temperatures, rank=0, world=1, device="cpu", seed=4):
        self.n = len(costs)
        if len(temperatures) != self.n or self.n < 2:
            raise ValueError("one temperature per replica, at least two replicas")
        self.parts = lpt_partition(list(costs), world)
        self.rank, self.world, self.device, self.seed = rank, world, device, seed
        self.mine = list(self.parts[rank])
        self.width = max(len(p) for p in self.parts)
        self.temps = {i: float(t) for i, t in enumerate(temperatures)}
        self.attempts = 0      # exchange passes made
        self.accepted = 0      # swaps accepted over all passes

    def _gather(self, energies):
        """{replica id: U} of this rank -> (temperature, U) of every replica."""
        import torch
        import torch.distributed as dist
        local = torch.full((self.width, 3), -1.0, dtype=torch.float64)
        for k, rid in enumerate(self.mine):
            local[k, 0] = rid
            local[k, 1] = self.temps[rid]
            local[k, 2] = energies[rid]
        if self.world > 1 and dist.is_available() and dist.is_initialized():
            local = local.to(self.device)
            out = torch.empty((self.world * self.width, 3), dtype=torch.float64, device=self.device)
            dist.all_gather_into_tensor(out, local)
            rows = out.cpu().numpy()
        else:
            rows = local.numpy()
        temps, energy = {}, {}
        for rid, t, u in rows:
            if rid >= 0:
                temps[int(rid)] = float(t)
                energy[int(rid)] = float(u)
        if sorted(energy) != list(range(self.n)):
            raise RuntimeError("replica exchange: the gathered replicas do not cover every replica once")
        return temps, energy

    def attempt(self, energies):
        """One exchange pass.  energies: {replica id: U} for this rank's replicas
        (kcal/mol).  Returns {replica id: velocity factor} for this rank's
        replicas whose temperature changed."""
        temps, energy = self._gather(energies)
        if temps != self.temps:
            raise RuntimeError("replica exchange: ranks disagree on the temperature assignment")
        uniforms = splitmix64_uniform(self.seed ^ 0xE7C4, self.n - 1, offset=self.attempts * (self.n - 1))
        new, acc = exchange_labels(self.temps, energy, uniforms)
        factors = {rid: math.sqrt(new[rid] / self.temps[rid]) for rid in self.mine if new[rid] != self.temps[rid]}
        self.temps = new
        self.attempts += 1
        self.accepted += acc
        return factors


def run_exchange(exchange, advance, scale, blocks, interval):
    """blocks x interval steps on this rank's replicas, an exchange attempt
    after each block.  advance(nsteps) -> {replica id: potential energy at the
    block's end} for this rank's replicas; scale(replica id, factor) rescales
    a replica's velocities.  Returns the temperature assignment after every
    attempt (a list of dicts)."""
    history = []
    for _ in range(blocks):
        energies = advance(interval)
        for rid, f in exchange.attempt(energies).items():
            scale(rid, f)
        history.append(dict(exchange.temps))
    return history


def replica_sizes(n, seed=4, lo=256, hi=4096):
    """Water counts of the uneven replica set: log-uniform on [lo, hi], seeded."""
    u = splitmix64_uniform(seed, n)
    return [int(round(math.exp(math.log(lo) + x * (math.log(hi) - math.log(lo))))) for x in u]


def temperature_ladder(n, tmin=280.0, tmax=450.0):
    """Geometric temperatures from tmin to tmax."""
    return list(tmin * (tmax / tmin) ** (np.arange(n) / max(1, n - 1)))
