"""Free-energy perturbation over lambda windows, the windows run as one
replica batch.

Mirrors the reference's pieces: ElecLJ::set_lambda (src/eleclj.cpp:273-319)
interpolates every site's charge, sigma, epsilon and screening radius
linearly between two parameter sets, (1 - lambda) p1 + lambda p2, and
FEP::update (src/msimprog.cpp:97-106) evaluates the perturbed potential at
the start and end lambda on the current configuration, dU = U(end) -
U(start).  Each window here is its own potential handle and integrator; all
windows advance together in one mmnb_md_batch, and every `sample_every`
steps each window's configuration is evaluated at its neighbours' lambdas.
The free-energy difference between neighbouring windows is the exponential
average of dU (Zwanzig), summed along the path.
"""
import math

import numpy as np

from . import ElecLJ, maxwell_boltzmann
from .md import MDyn, ReplicaBatch
from .units import K_to_kcal_mol


def lambda_params(p1, p2, lam):
    """Site arrays at lambda from two dicts of arrays (q, sigma, epsilon,
    rscreen; site_mask taken from p1 with LJ set where either state has it)."""
    t = 1.0 - lam
    out = {k: t * np.asarray(p1[k], dtype=np.float64) + lam * np.asarray(p2[k], dtype=np.float64)
           for k in ("q", "sigma", "epsilon", "rscreen")}
    out["site_mask"] = np.asarray(p1["site_mask"]) | np.asarray(p2["site_mask"])
    return out


def set_lambda(pot, p1, p2, lam):
    p = lambda_params(p1, p2, lam)
    pot.set_params(p["site_mask"], p["q"], p["sigma"], p["epsilon"], p["rscreen"])


def energy_difference(pot, p1, p2, r, start, end):
    """FEP::update: U(end) - U(start) at configuration r, using `pot` as the
    perturbed potential (its parameters are left at `end`)."""
    set_lambda(pot, p1, p2, start)
    u0 = pot.compute(r)["total"]
    set_lambda(pot, p1, p2, end)
    u1 = pot.compute(r)["total"]
    return u1 - u0


def run_windows(system, p1, p2, lambdas, cfg, temperature=300.0, steps=2000, sample_every=100, dt=0.002,
                precision="mixed", seed=1):
    """Run the windows as one batch; returns dict with the forward and
    backward exponential averages between neighbouring windows and their
    sum (kcal/mol)."""
    n = len(lambdas)
    wins = []
    for k, lam in enumerate(lambdas):
        pot = ElecLJ(precision=precision, **cfg).init(system)
        set_lambda(pot, p1, p2, lam)
        md = MDyn(pot, system.masses, timestep=dt)
        md.set_state(system.positions, maxwell_boltzmann(system, temperature, seed=seed + k))
        wins.append((pot, md))
    pert = ElecLJ(precision=precision, **cfg).init(system)
    batch = ReplicaBatch([m for _, m in wins])
    kt = K_to_kcal_mol(temperature)
    fwd = [[] for _ in range(n - 1)]
    bwd = [[] for _ in range(n - 1)]
    for _ in range(steps // sample_every):
        batch.run(sample_every)
        for k, (_, md) in enumerate(wins):
            r, _ = md.state()
            if k + 1 < n:
                fwd[k].append(energy_difference(pert, p1, p2, r, lambdas[k], lambdas[k + 1]))
            if k > 0:
                bwd[k - 1].append(energy_difference(pert, p1, p2, r, lambdas[k], lambdas[k - 1]))
    batch.close()
    for pot, md in wins:
        md.close()
        pot.close()
    pert.close()

    def zwanzig(du):
        du = np.asarray(du)
        m = du.min()
        return m - kt * math.log(np.mean(np.exp(-(du - m) / kt)))

    dA_f = [zwanzig(x) for x in fwd]
    dA_b = [-zwanzig(x) for x in bwd]
    return dict(lambdas=list(lambdas), dA_forward=dA_f, dA_backward=dA_b, total_forward=float(sum(dA_f)),
                total_backward=float(sum(dA_b)), samples_per_window=steps // sample_every)
