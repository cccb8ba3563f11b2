"""Test infrastructure: an FP64 restatement, on the CPU, of the per-site
parameter gradients of one evaluation (what the library's mmnb_site_gradients
returns), for the Ewald k-sum form.

Given the oracle's own results at the positions r (site potentials phi, fields
E, its group-pair list), per site i:
  dU/dq_i = phi_i;  dU/dsigma_i, dU/depsilon_i from the switched LJ pair terms,
  the 1-4 LJ terms and the LJ tail;
and for a loss L of the forces with g = dL/dF:
  dL/dq_i = g_i . E_i + psi_i,  psi_i = the potential at site i of the dipoles
  q_j g_j as the real-space group-pair sum (with the switch term: the switch
  force on the anchors is ds times the unswitched pair energies, linear in
  each charge), the exclusion and 1-4 corrections and the Ewald k-sum see them;
  dL/dsigma_i, dL/depsilon_i from the LJ forces' sigma/epsilon derivatives.

Reference semantics restated: RSpaceEwald's group-pair loop (src/rspace.c:
413-491: anchors' image shift, quintic switch, the switch derivative on the
anchors, group_excluded), its Chebyshev erfc table (src/rspace.c:25-37, the
oracle's orc_chebyshev gives the reference's own coefficients) with
erfc/exp outside it (:104-156), the exclusion and 1-4 terms (:492-557),
kspace_field (src/kspace.c:35-174), the LJ tail (src/eleclj.cpp:283-308,
1247-1266).  Only tests import this module.
"""
import math

import numpy as np

TWO_OVER_SQRTPI = 2.0 / math.sqrt(math.pi)


def _table_b(cheb, eta, r2):
    """b0 = erfc(eta r)/r and b1 = -2 db0/d(r^2) as the reference evaluates
    them: its table inside (min, max), erfc and exp outside."""
    mn, mx, inv, c = cheb
    r2 = np.asarray(r2, dtype=np.float64)
    b0 = np.empty_like(r2)
    b1 = np.empty_like(r2)
    inside = (r2 > mn) & (r2 < mx)
    x = (r2[inside] - mn) * inv
    i = x.astype(np.int64)
    x = x - i
    cc = c[i]
    b0[inside] = ((cc[:, 3] * x + cc[:, 2]) * x + cc[:, 1]) * x + cc[:, 0]
    b1[inside] = (cc[:, 6] * x + cc[:, 5]) * x + cc[:, 4]
    out = ~inside
    if out.any():
        r = np.sqrt(r2[out])
        er = eta * r
        e = np.exp(-(er * er))
        b0o = np.array([math.erfc(v) for v in er]) / r
        b0[out] = b0o
        b1[out] = (b0o + eta * TWO_OVER_SQRTPI * e) / r2[out]
    return b0, b1


def _min_image(d, box):
    return d - box * np.floor(d / box + 0.5)


def _lj(si, sj, ei, ej, geometric, r2):
    """u, du (force = du d), and the sigma_i / sigma_j derivatives of u and du."""
    if geometric:
        sg = si * sj
        ki, kj = 3.0 / si, 3.0 / sj
    else:
        hs = 0.5 * (si + sj)
        sg = hs * hs
        ki = kj = 6.0 / (si + sj)
    s6 = sg ** 3
    b = 4.0 * np.sqrt(ei * ej) * s6
    aa = b * s6
    ir2 = 1.0 / r2
    ir6 = ir2 ** 3
    a12, b6 = aa * ir6 * ir6, b * ir6
    u = a12 - b6
    du = (12 * a12 - 6 * b6) * ir2
    us = 2 * a12 - b6
    dus = (24 * a12 - 6 * b6) * ir2
    return u, du, ki * us, kj * us, ki * dus, kj * dus


def lj_tail_coefficients(rc, width, volume):
    """cA, cB with U_tail = cA totA + cB totB (src/eleclj.cpp:1247-1266)."""
    rhi, rlo = rc, rc - width

    def tail(A, B):
        rlo3, rlo6 = rlo ** 3, rlo ** 6
        rlo9 = rlo6 * rlo3
        rhi3, rhi4, rhi5, rhi6, rhi7 = rhi ** 3, rhi ** 4, rhi ** 5, rhi ** 6, rhi ** 7
        return 2 * math.pi / volume * (
            A / (9 * rlo9) + B / (3 * rlo3) -
            (rhi - rlo) / (63 * rhi3 * rlo9 * (rhi + rlo) ** 5) *
            (3 * B * rhi3 * rlo6 * (7 * rhi4 + 42 * rhi3 * rlo + 112 * rhi ** 2 * rlo ** 2 + 150 * rhi * rlo3 +
                                    25 * rlo ** 4) +
             A * (7 * rhi7 + 42 * rhi6 * rlo + 112 * rhi5 * rlo ** 2 + 182 * rhi4 * rlo3 + 217 * rhi3 * rlo ** 4 +
                  224 * rhi ** 2 * rlo ** 5 + 192 * rhi * rlo6 + 32 * rlo ** 7)))
    return tail(1.0, 0.0), tail(0.0, 1.0)


def _key(v):
    return float(f"{v:12.6g}")


def site_gradients(lib, system, cfg, r, dl_df, pairs14=None):
    """Per-site gradients of U and of L (g = dl_df, nsite x 3) at positions r
    for `system` (box, groups, exclusions, site_mask, q, sigma, epsilon,
    rscreen) with the oracle configuration `cfg` (make_config keywords; Ewald
    k-sum, cubic or orthorhombic box).  lib: the oracle (port() or
    reference()).  Returns dict du_dq, du_dsig, du_deps, dl_dq, dl_dsig,
    dl_deps."""
    from oracle.oracle import make_config
    n = system.nsite
    r = np.ascontiguousarray(r, dtype=np.float64).reshape(n, 3)
    g = np.ascontiguousarray(dl_df, dtype=np.float64).reshape(n, 3)
    box = np.broadcast_to(np.asarray(system.box, dtype=np.float64), (3,)).copy()
    q, sig, eps = np.asarray(system.q, float), np.asarray(system.sigma, float), np.asarray(system.epsilon, float)
    rs = np.asarray(system.rscreen, float)
    mask = np.asarray(system.site_mask)
    hasq, haslj = (mask & 1) != 0, (mask & 2) != 0
    o = lib.eleclj(make_config(box, **cfg), n, system.groups, system.exclusions, mask, q, sig, eps, rs,
                   pairs14=pairs14)
    out = o.eval(r)
    eta = o.eta
    rc = cfg["rspace_cutoff"]
    width = cfg.get("smoothing_width", 1.0)
    geometric = bool(cfg.get("geometric_combining_for_sigma", False))
    cheb = lib.chebyshev(rc, eta)
    groups = np.asarray(system.groups)
    excl = np.asarray(system.exclusions).reshape(-1, 2)
    exset = set(map(tuple, np.sort(excl, axis=1).tolist()))
    gof = np.empty(n, dtype=np.int64)
    for k, (a, b) in enumerate(groups):
        gof[a:b] = k
    gex = set()
    for i, j in exset:
        if gof[i] != gof[j]:
            gex.add((min(gof[i], gof[j]), max(gof[i], gof[j])))

    psi = np.zeros(n)
    dus, due, dls, dle = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n)
    rhi2, rlo2 = rc * rc, (rc - width) ** 2
    inv_sw = 1.0 / (rhi2 - rlo2) if rhi2 > rlo2 else 0.0
    # real space: every listed group pair once
    for gi, gj in o.nbrlist().pairs():
        ai, aj = groups[gi][0], groups[gj][0]
        R = r[ai] - r[aj]
        shift = -box * np.floor(R / box + 0.5)
        R = R + shift
        R2 = float(R @ R)
        if R2 > rhi2:
            continue
        S, ds = 1.0, 0.0
        if R2 > rlo2:
            z = (R2 - rlo2) * inv_sw
            S = ((-6 * z + 15) * z - 10) * z ** 3 + 1
            ds = ((60 * z - 120) * z + 60) * z * z * inv_sw
        GR = float((g[ai] - g[aj]) @ R)
        ex = (min(gi, gj), max(gi, gj)) in gex
        si = np.arange(groups[gi][0], groups[gi][1])
        sj = np.arange(groups[gj][0], groups[gj][1])
        ia, jb = np.meshgrid(si, sj, indexing="ij")
        ia, jb = ia.ravel(), jb.ravel()
        if ex:
            keep = np.array([(min(a, b), max(a, b)) not in exset for a, b in zip(ia, jb)], dtype=bool)
            ia, jb = ia[keep], jb[keep]
        d = r[ia] - r[jb] + shift
        r2 = np.einsum("ij,ij->i", d, d)
        mq = hasq[ia] & hasq[jb]
        if mq.any():
            a_, b_, dq, r2q = ia[mq], jb[mq], d[mq], r2[mq]
            b0, b1 = _table_b(cheb, eta, r2q)
            rsum = rs[a_] + rs[b_]
            scr = r2q < rsum * rsum
            if scr.any():
                invr = 1 / np.sqrt(r2q[scr])
                inv3 = 1 / rsum[scr] ** 3
                b0[scr] += (-0.5 * r2q[scr] * inv3 + 1.5 / rsum[scr]) - invr
                b1[scr] += inv3 - invr ** 3
            gbd = np.einsum("ij,ij->i", g[b_], dq)
            gad = np.einsum("ij,ij->i", g[a_], dq)
            np.add.at(psi, a_, q[b_] * (ds * GR * b0 - S * b1 * gbd))
            np.add.at(psi, b_, q[a_] * (ds * GR * b0 + S * b1 * gad))
        ml = haslj[ia] & haslj[jb]
        if ml.any():
            a_, b_, dl, r2l = ia[ml], jb[ml], d[ml], r2[ml]
            u, du, usa, usb, dusa, dusb = _lj(sig[a_], sig[b_], eps[a_], eps[b_], geometric, r2l)
            gd = np.einsum("ij,ij->i", g[a_] - g[b_], dl)
            np.add.at(dus, a_, S * usa)
            np.add.at(dus, b_, S * usb)
            np.add.at(due, a_, S * u)
            np.add.at(due, b_, S * u)
            np.add.at(dls, a_, S * dusa * gd + ds * GR * usa)
            np.add.at(dls, b_, S * dusb * gd + ds * GR * usb)
            np.add.at(dle, a_, S * du * gd + ds * GR * u)
            np.add.at(dle, b_, S * du * gd + ds * GR * u)
    # exclusion corrections: -erf(eta r)/r per excluded charged pair
    for i, j in exset:
        if not (hasq[i] and hasq[j]):
            continue
        d = _min_image(r[i] - r[j], box)
        r2 = float(d @ d)
        rm = math.sqrt(r2)
        b0 = -math.erf(eta * rm) / rm
        b1 = (b0 + eta * TWO_OVER_SQRTPI * math.exp(-(eta * rm) ** 2)) / r2
        psi[i] -= q[j] * b1 * float(g[j] @ d)
        psi[j] += q[i] * b1 * float(g[i] @ d)
    # 1-4 pairs: (factor - 1) x the full pair when scaling, the full pair otherwise
    if pairs14 is not None and len(pairs14):
        f_e = cfg.get("elec_1_4_scale_factor", 1.0)
        f_l = cfg.get("lj_1_4_scale_factor", 1.0)
        se = f_e - 1 if abs(f_e - 1) > 1e-10 else 1.0
        sl = f_l - 1 if abs(f_l - 1) > 1e-10 else 1.0
        for i, j in np.asarray(pairs14).reshape(-1, 2):
            d = _min_image(r[i] - r[j], box)
            r2 = float(d @ d)
            if hasq[i] and hasq[j]:
                rsum = rs[i] + rs[j]
                b1 = 1 / rsum ** 3 if r2 < rsum * rsum else r2 ** -1.5
                b1 *= se
                psi[i] -= q[j] * b1 * float(g[j] @ d)
                psi[j] += q[i] * b1 * float(g[i] @ d)
            if haslj[i] and haslj[j]:
                u, du, usa, usb, dusa, dusb = _lj(sig[i], sig[j], eps[i], eps[j], geometric, r2)
                gd = float((g[i] - g[j]) @ d)
                dus[i] += sl * usa
                dus[j] += sl * usb
                due[i] += sl * u
                due[j] += sl * u
                dls[i] += sl * dusa * gd
                dls[j] += sl * dusb * gd
                dle[i] += sl * du * gd
                dle[j] += sl * du * gd
    # Ewald k-sum: psi_i += sum_k 2 a_k (Ds cos k.r_i - Dc sin k.r_i) over the
    # half space |n|^2 <= kc^2 (the summand is even in k, so which half is taken
    # does not matter), Dc + i Ds = sum_j q_j (k . g_j) exp(i k . r_j)
    kc = cfg["kspace_cutoff"]
    nmax = int(math.floor(kc))
    rng = np.arange(-nmax, nmax + 1)
    nv = np.stack(np.meshgrid(rng, rng, rng, indexing="ij"), -1).reshape(-1, 3)
    n2 = (nv ** 2).sum(1)
    half = (nv[:, 0] > 0) | ((nv[:, 0] == 0) & (nv[:, 1] > 0)) | ((nv[:, 0] == 0) & (nv[:, 1] == 0) & (nv[:, 2] > 0))
    nv = nv[half & (n2 <= kc * kc + 1e-8)]
    kv = 2 * math.pi * nv / box
    k2 = (kv ** 2).sum(1)
    volume = float(np.prod(box))
    ak = 4 * math.pi / volume * np.exp(-k2 / (4 * eta * eta)) / k2
    qq = np.where(hasq, q, 0.0)
    ph = r @ kv.T
    cs, sn = np.cos(ph), np.sin(ph)
    w = qq[:, None] * (g @ kv.T)
    Dc, Ds = (w * cs).sum(0), (w * sn).sum(0)
    psi += (2 * ak[None, :] * (Ds[None, :] * cs - Dc[None, :] * sn)).sum(1)

    du_dq = np.where(hasq, out["phi"], 0.0)
    dl_dq = np.where(hasq, np.einsum("ij,ij->i", g, out["evec"]) + psi, 0.0)
    live = haslj & (eps > 0)
    inv2e = np.where(live, 0.5 / np.where(live, eps, 1.0), 0.0)
    du_dsig, dl_dsig = np.where(live, dus, 0.0), np.where(live, dls, 0.0)
    du_deps, dl_deps = due * inv2e, dle * inv2e
    # LJ tail over the (sigma, epsilon) classes printed with %12.6g
    if cfg.get("include_lj_correction", True) and live.any():
        cA, cB = lj_tail_coefficients(rc, width, volume)
        keys = [(_key(sig[i]), _key(eps[i])) for i in range(n) if live[i]]
        classes = {}
        for kk in keys:
            classes[kk] = classes.get(kk, 0) + 1
        tail_s, tail_e = {}, {}
        for (sa, ea) in classes:
            ts = te = 0.0
            for (sb, eb), nb in classes.items():
                s6 = (math.sqrt(sa * sb) if geometric else 0.5 * (sa + sb)) ** 6
                kap = 3 / sa if geometric else 6 / (sa + sb)
                bb = 4 * math.sqrt(ea * eb) * s6
                aa = bb * s6
                ts += 2 * nb * (cA * 2 * kap * aa - cB * kap * bb)
                te += 2 * nb * (cA * aa - cB * bb) / (2 * ea)
            tail_s[(sa, ea)], tail_e[(sa, ea)] = ts, te
        for i in np.nonzero(live)[0]:
            kk = (_key(sig[i]), _key(eps[i]))
            du_dsig[i] += tail_s[kk]
            du_deps[i] += tail_e[kk]
    return dict(du_dq=du_dq, du_dsig=du_dsig, du_deps=du_deps, dl_dq=dl_dq, dl_dsig=dl_dsig, dl_deps=dl_deps,
                eval=out)
