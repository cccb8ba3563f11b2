"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run in a checkout where the reference sources are present:

    make -C oracle ref REF=/root/reference
    python tests/golden/make_golden.py /root/reference

Everything numeric comes from oracle/_ref/libref.so, i.e. the reference's own
src/rspace.c, src/pppm.c, src/kspace.c, src/cheby.c, src/pbin.c and
src/nbrlist.cpp compiled unmodified (oracle/Makefile), driven on the seeded
synthetic water boxes of molmodel_b200.water.  The PairBinary known-answer
test is read from the reference's own self-test (src/pbin.c:152-214): the
pairs its main() adds and the rows and membership matrix its comment says it
prints.  Tests compare the oracle's restatement (and, on a GPU, the product)
against these files; nothing at test time reads the reference tree.
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from molmodel_b200.water import water_box  # noqa: E402
from oracle.oracle import make_config, reference  # noqa: E402

C1 = dict(rspace_cutoff=9.0, smoothing_width=1.0, ewald_screening=0.35, kspace_cutoff=7.0)
P3M_SMALL = dict(rspace_cutoff=7.0, ewald_screening=0.35, use_p3m=True, p3m_grid_spacing=0.8,
                 p3m_assignment_order=5)


def canon(p):
    p = np.sort(np.asarray(p, dtype=np.int64), axis=1)
    p = np.unique(p, axis=0)
    return p.astype(np.int32)


def run(lib, wb, cfg, pairs14=None, **sysover):
    sysd = dict(nsite=wb.nsite, groups=wb.groups, exclusions=wb.exclusions, site_mask=wb.site_mask,
                q=wb.q, sig=wb.sigma, eps=wb.epsilon, rscreen=wb.rscreen)
    sysd.update(sysover)
    c = make_config(wb.box, **cfg)
    o = lib.eleclj(c, sysd["nsite"], sysd["groups"], sysd["exclusions"], sysd["site_mask"], sysd["q"],
                   sysd["sig"], sysd["eps"], sysd["rscreen"], pairs14=pairs14)
    out = o.eval(wb.positions)
    nl = o.nbrlist()
    return out, canon(nl.pairs()), nl.cells(wb.ngroup), nl.ncell(), o.eta, o.nlw


def save(name, wb, cfg, out, pairs, cells, ncell, eta, nlw, **extra):
    np.savez_compressed(
        os.path.join(HERE, name), positions=wb.positions, f=out["f"], phi=out["phi"], evec=out["evec"],
        ljf=out["ljf"], energies=np.array([out["elec"], out["lj"], out["lj_correction"], out["total"]]),
        pairs=pairs, cells=cells, ncell=ncell, eta=eta, nlw=nlw, box=wb.box, seed=wb.seed,
        n=round(wb.nwater ** (1 / 3)), config=json.dumps(cfg), **extra)


def pbin_kat(reference_root):
    src = open(os.path.join(reference_root, "src", "pbin.c")).read()
    main = src[src.index("int main()"):]
    adds = [[int(a), int(b)] for a, b in re.findall(r"PairBinary_add\(p,(\d+),(\d+)\)", main)]
    comment = src[src.index("should print out"):src.index("*/", src.index("should print out"))]
    rows, matrix = {}, []
    for line in comment.splitlines():
        m = re.match(r"\s*(\d+):\s*(.*)$", line)
        if m:
            rows[int(m.group(1))] = [int(x) for x in m.group(2).split()]
        elif re.match(r"^\s*([01] )+[01]?\s*$", line):
            matrix.append([int(x) for x in line.split()])
    n = len(rows)
    return dict(source="src/pbin.c:152-214", n=n, adds=adds, rows=[rows[i] for i in range(n)], exists=matrix)


def esp_fixture(ref):
    """Potential at points (ElecLJ::electrostatic_potential_at_gridpoints): a
    neutral box with the k-sum, and a charged box with screening radii whose
    forces use P3M (the potential at points still uses the k-sum)."""
    rng = np.random.default_rng(11)
    out = {}
    for tag, n, seed, cfg, charged in (("ksum", 6, 1, C1, False), ("p3m", 5, 3, P3M_SMALL, True)):
        wb = water_box(n, seed=seed)
        q = wb.q.copy()
        rscreen = wb.rscreen.copy()
        if charged:
            q[0] += 0.2 * q[1]
            rscreen = np.where(np.arange(wb.nsite) % 3 == 0, 1.6, 0.0)
        # points anywhere in (and slightly outside) the box, and points 0.4-2.5 A
        # from sites (closed-form erfc below r = 2 A, the screening radius, the table)
        far = rng.uniform(-0.1 * wb.box, 1.1 * wb.box, size=(96, 3))
        k = rng.choice(wb.nsite, size=96, replace=False)
        d = rng.normal(size=(96, 3))
        d *= (rng.uniform(0.4, 2.5, size=96) / np.linalg.norm(d, axis=1))[:, None]
        pts = np.concatenate([far, wb.positions[k] + d])
        o = ref.eleclj(make_config(wb.box, **cfg), wb.nsite, wb.groups, wb.exclusions, wb.site_mask, q,
                       wb.sigma, wb.epsilon, rscreen)
        out[tag + "_n"] = n
        out[tag + "_seed"] = seed
        out[tag + "_config"] = json.dumps(cfg)
        out[tag + "_q"] = q
        out[tag + "_rscreen"] = rscreen
        out[tag + "_points"] = pts
        out[tag + "_phi"] = o.phi_at_points(wb.positions, pts)
    np.savez_compressed(os.path.join(HERE, "esp_points.npz"), **out)


def main():
    reference_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MMNB_REFERENCE", "/root/reference")
    ref = reference()
    if ref is None:
        raise SystemExit("oracle/_ref/libref.so is missing: run `make -C oracle ref` first")
    with open(os.path.join(HERE, "pbin_kat.json"), "w") as fh:
        json.dump(pbin_kat(reference_root), fh, indent=1)
    wb = water_box(6, seed=1)
    save("c1_ewald.npz", wb, C1, *run(ref, wb, C1))
    wb5 = water_box(5, seed=3)
    save("p3m_small.npz", wb5, P3M_SMALL, *run(ref, wb5, P3M_SMALL))
    ik = dict(P3M_SMALL, p3m_ik_differentiate=True, p3m_assignment_order=4)
    save("p3m_small_ik.npz", wb5, ik, *run(ref, wb5, ik))
    # cross-group exclusions, screening radii and scaled 1-4 pairs
    rng = np.random.default_rng(3)
    k = rng.choice(wb.nwater - 1, size=wb.nwater // 4, replace=False)
    excl = np.concatenate([wb.exclusions, np.stack([3 * k, 3 * (k + 1)], 1),
                           np.stack([3 * k + 1, 3 * (k + 1) + 2], 1)]).astype(np.int32)
    rscreen = np.where(np.arange(wb.nsite) % 3 == 0, 1.6, 0.0)
    j = rng.choice(wb.nwater - 2, size=wb.nwater // 5, replace=False)
    p14 = np.stack([3 * j, 3 * (j + 2) + 1], 1).astype(np.int32)
    cfg = dict(C1, elec_1_4_scale_factor=0.5, lj_1_4_scale_factor=0.7)
    save("c1_topology.npz", wb, cfg, *run(ref, wb, cfg, pairs14=p14, exclusions=excl, rscreen=rscreen),
         exclusions=excl, rscreen=rscreen, pairs14=p14)
    mn, mx, inv, coeff = ref.chebyshev(9.0, 0.35)
    np.savez_compressed(os.path.join(HERE, "cheb_9_0.35.npz"), min=mn, max=mx, inv_dx=inv, coeff=coeff)
    esp_fixture(ref)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
