"""Accuracy and energy-conservation report of the mixed-precision form.

For each water-box configuration: RMS and max relative force error and the
relative energy error of the mixed form against the FP64 form (which matches
the reference's own code to 1e-10) on seeded configurations, and the NVE
drift of the conserved energy (kinetic + potential, the quantity the
reference prints as "Conserved energy", src/mdyn.cpp:358) of both forms.

  python -m molmodel_b200.report [--configs C1,C2,C3] [--seeds 10] [--out file.json]
"""
import argparse
import json
import time

import numpy as np

from . import ElecLJ, maxwell_boltzmann, water_box
from .md import MDyn, nve_drift

# side (waters per edge), reciprocal space, timestep (ps), NVE steps
CONFIGS = {
    "C1": dict(side=6, recip=dict(kspace_cutoff=7.0), dt=0.001, nve_steps=1000,
               text="216 waters, L 18.64 A, Ewald k-sum kc 7, 1 fs"),
    "C2": dict(side=16, recip=dict(use_p3m=True, mesh=48, p3m_assignment_order=5), nlw=1.5, dt=0.002,
               nve_steps=5000, text="4096 waters, L 49.72 A, P3M 48^3 order 5, skin 1.5 A, 2 fs"),
    "C3": dict(side=32, recip=dict(use_p3m=True, mesh=96, p3m_assignment_order=5), nlw=1.5, dt=0.002,
               nve_steps=25000, text="32768 waters, L 99.44 A, P3M 96^3 order 5, skin 1.5 A, 2 fs (50 ps)"),
}


def config(name, box):
    c = CONFIGS[name]
    cfg = dict(rspace_cutoff=9.0, smoothing_width=1.0, ewald_screening=0.35)
    if "nlw" in c:
        cfg["neighbor_list_width"] = c["nlw"]
    rec = dict(c["recip"])
    if rec.pop("use_p3m", False):
        cfg.update(use_p3m=True, p3m_grid_spacing=box / rec.pop("mesh"), **rec)
    else:
        cfg.update(rec)
    return cfg


def errors(name, seeds):
    out = []
    for seed in seeds:
        wb = water_box(CONFIGS[name]["side"], seed=seed)
        cfg = config(name, wb.box)
        a = ElecLJ(precision="fp64", **cfg).init(wb)
        g64 = a.compute(wb.positions)
        a.close()
        b = ElecLJ(precision="mixed", **cfg).init(wb)
        g32 = b.compute(wb.positions)
        b.close()
        df = g32["f"] - g64["f"]
        rms_f = float(np.sqrt((g64["f"] ** 2).sum(1).mean()))
        out.append(dict(seed=seed, rms_rel_force=float(np.sqrt((df ** 2).sum() / (g64["f"] ** 2).sum())),
                        max_rel_force=float(np.sqrt((df ** 2).sum(1)).max() / rms_f),
                        rel_energy=abs(g32["total"] - g64["total"]) / abs(g64["total"])))
    return out


def nve(name, precision, seed=1, temperature=300.0):
    c = CONFIGS[name]
    wb = water_box(c["side"], seed=seed)
    pot = ElecLJ(precision=precision, **config(name, wb.box)).init(wb)
    md = MDyn(pot, wb.masses, timestep=c["dt"])
    md.set_state(wb.positions, maxwell_boltzmann(wb, temperature, seed=seed + 100))
    t0 = time.perf_counter()
    e = md.run(c["nve_steps"])
    wall = time.perf_counter() - t0
    md.close()
    pot.close()
    return dict(precision=precision, steps=c["nve_steps"], dt_ps=c["dt"], temperature_start_K=temperature,
                drift_kcal_mol_per_ns_per_molecule=float(nve_drift(e, c["dt"], wb.nwater)),
                conserved_std_kcal_mol=float(e[:, 2].std()), kinetic_std_kcal_mol=float(e[:, 0].std()),
                conserved_first_last=[float(e[0, 2]), float(e[-1, 2])], wall_s=wall,
                steps_per_s_including_launch=c["nve_steps"] / wall)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--configs", default="C1,C2,C3")
    ap.add_argument("--seeds", type=int, default=10)
    ap.add_argument("--out", default=None)
    ap.add_argument("--no-nve", action="store_true")
    args = ap.parse_args()
    report = {}
    for name in args.configs.split(","):
        errs = errors(name, range(1, args.seeds + 1))
        r = dict(config=CONFIGS[name]["text"], errors=errs,
                 worst=dict(rms_rel_force=max(x["rms_rel_force"] for x in errs),
                            max_rel_force=max(x["max_rel_force"] for x in errs),
                            rel_energy=max(x["rel_energy"] for x in errs)))
        if not args.no_nve:
            r["nve"] = [nve(name, "mixed"), nve(name, "fp64")]
        report[name] = r
        print(json.dumps({name: {k: v for k, v in r.items() if k != "errors"}}), flush=True)
    if args.out:
        with open(args.out, "w") as f:
            json.dump(report, f, indent=1)


if __name__ == "__main__":
    main()
