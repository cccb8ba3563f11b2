"""Replica bookkeeping across ranks: partitioning and temperature exchange.

Replicas are independent units: each rank evaluates and integrates its own
replicas with no collective on the data path.  Every exchange interval the
ranks gather (replica id, potential energy) and run the same Metropolis pass
on the same uniform numbers, so every rank reaches the same temperature
assignment without further messages.

The acceptance rule is MDyn::try_replica_exchange's (src/mdyn.cpp:317-351):
for neighbours in temperature, replica a at kT0 and b at kT1,
    du = -u_b/kT0 - u_a/kT1 + u_a/kT0 + u_b/kT1,
accept if du < 0 or uniform < exp(-du), visiting the pairs from the hottest
down as the reference's chain of sends resolves.  The reference swaps the
coordinates of equal systems; for replicas of different sizes the
temperature labels are swapped instead, which is the same move for equal
systems.
"""
import math

from .units import K_to_kcal_mol


def lpt_partition(costs, nranks):
    """Longest-processing-time assignment: replica ids per rank, heaviest
    first onto the least-loaded rank (ties to the lower rank)."""
    load = [0.0] * nranks
    out = [[] for _ in range(nranks)]
    for rid in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        r = min(range(nranks), key=lambda k: (load[k], k))
        out[r].append(rid)
        load[r] += costs[rid]
    for ids in out:
        ids.sort()
    return out


def exchange_labels(temperature_of, energy_of, uniforms):
    """One exchange pass.  temperature_of: replica id -> temperature (K);
    energy_of: replica id -> potential energy (kcal/mol); uniforms: numbers in
    [0, 1), one per neighbouring pair (consumed hottest pair first).  Returns
    the new temperature_of and the number of accepted swaps."""
    t = dict(temperature_of)
    order = sorted(t, key=lambda rid: (t[rid], rid))  # coldest first
    accepted = 0
    k = 0
    for i in range(len(order) - 2, -1, -1):
        a, b = order[i], order[i + 1]
        kt0, kt1 = K_to_kcal_mol(t[a]), K_to_kcal_mol(t[b])
        ua, ub = energy_of[a], energy_of[b]
        du = -ub / kt0 - ua / kt1 + ua / kt0 + ub / kt1
        u = uniforms[k]
        k += 1
        if du < 0 or u < math.exp(-du):
            t[a], t[b] = t[b], t[a]
            order[i], order[i + 1] = b, a
            accepted += 1
    return t, accepted


def gather_energies(local):
    """local: {replica id: energy} of this rank -> the same dict over all
    ranks (torch.distributed all_gather_object: NCCL or gloo)."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return dict(local)
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, dict(local))
    out = {}
    for p in parts:
        out.update(p)
    return out
