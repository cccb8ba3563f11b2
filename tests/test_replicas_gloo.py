"""Replica bookkeeping on CPU ranks (gloo, world size 2): LPT partition,
energy gather and a temperature exchange that every rank computes alike."""
import json
import math
import os
import socket
import subprocess
import sys

import numpy as np

from molmodel_b200.replicas import exchange_labels, lpt_partition
from molmodel_b200.units import K_to_kcal_mol

HERE = os.path.dirname(os.path.abspath(__file__))


def test_lpt_partition_balances_uneven_replicas():
    sizes = np.round(np.exp(np.random.default_rng(4).uniform(np.log(256), np.log(4096), 64))).astype(int)
    parts = lpt_partition(list(sizes), 8)
    assert sorted(sum(parts, [])) == list(range(64))
    loads = [sizes[p].sum() for p in parts]
    assert max(loads) - min(loads) <= sizes.max()


def test_exchange_rule_is_the_reference_acceptance():
    """Two replicas, the reference's du, and both sides of the acceptance test."""
    t = {0: 300.0, 1: 330.0}
    u0, u1 = -990.0, -1000.0  # the hotter replica lower in energy: du > 0
    kt0, kt1 = K_to_kcal_mol(300.0), K_to_kcal_mol(330.0)
    du = -u1 / kt0 - u0 / kt1 + u0 / kt0 + u1 / kt1
    assert du > 0
    new, n = exchange_labels(t, {0: u0, 1: u1}, [math.exp(-du) * 0.999])
    assert n == 1 and new == {0: 330.0, 1: 300.0}
    new, n = exchange_labels(t, {0: u0, 1: u1}, [math.exp(-du) * 1.001])
    assert n == 0 and new == t


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _run_ranks(world):
    port = _free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.join(HERE, "replica_rank.py")], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            so, se = p.communicate(timeout=240)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        assert p.returncode == 0, se
        outs.append(json.loads(so.strip().splitlines()[-1]))
    return outs


def test_exchange_loop_over_two_ranks_matches_one_process():
    """The full loop (advance, one all-gather of (id, T, U), the same Metropolis
    pass on every rank, velocity rescaling of the swapped replicas) on two gloo
    ranks gives the single process's temperature history and energies."""
    a, b = _run_ranks(2)
    (one,) = _run_ranks(1)
    assert sorted(a["mine"] + b["mine"]) == list(range(6))
    assert a["history"] == b["history"] == one["history"]
    assert a["accepted"] == b["accepted"] == one["accepted"] and a["attempts"] == 4
    assert a["energies"] == b["energies"] == one["energies"]
    # temperatures move: some swap was accepted, and the ladder is kept
    assert one["accepted"] > 0
    for h in one["history"]:
        assert sorted(t for _, t in h) == sorted(t for _, t in one["history"][0])
