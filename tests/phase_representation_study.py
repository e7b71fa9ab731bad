"""How the opacity surrogate's phase-function representation moves the
temperatures, with everything else exact: the oracle's serial transport on a
reduced learned-opacities deck (60 x 40 cells, 100 wavelengths, three
compositions in 10 bins each, settled, random walk on), with ComputePart's
exact opacities and three Mueller matrices.  The matrices are ComputePart's
own rows, and the same rows reduced to the surrogate's Legendre moments
(order 12) and rebuilt by surrogate_phase.h: the plain clipped series and
the delta-M form.  Each run is compared with the exact matrix's run on seed
1: per-cell temperature (EJv^(1/4)) of the cells with >= 1e3 absorption
events, and the inclination-summed SED where both sides have > 2500 packets.
The exact matrix on seed 2 gives the Monte Carlo floor.  Six runs in
parallel on the host cores; 1e7 packets take about 7 minutes.

With `network`, the runs use the trained surrogate's own predictions instead:
the network (tests/mlp_ref.py, BF16 emulated) on each bin's sizes and
wavelengths, aggregated over the sizes as mcg_compute_part_surrogate does,
with its matrices rebuilt by delta-M or the plain series, and the two mixed
cases (network opacities with exact matrices, exact opacities with the
network's delta-M matrices).

    python tests/phase_representation_study.py [NPHOT] [network]"""
import json
import math
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

NA, L = 180, 12
th = np.pi * (np.arange(NA) + 0.5) / NA
mu, w = np.cos(th), np.sin(th)
P = np.zeros((L + 1, NA))
P[0], P[1] = 1.0, mu
for l in range(1, L):
    P[l + 1] = ((2 * l + 1) * mu * P[l] - l * P[l - 1]) / (l + 1)


def rebuild(F, dm):
    """ComputePart's row F[6][180] -> its Legendre moments (as the
    surrogate's training targets define them) -> surrogate_phase.h"""
    import hostcheck_ffi as H
    s0 = np.sum(F[0] * w)
    mom = [np.array([np.sum(F[e] * w * P[l]) / s0 for l in range(L + 1)]) for e in (0, 1, 3, 4)]
    return H.surr_phase(*mom, deltam=int(dm))


def network_optics(parts, deltam):
    """(Kabs, Ksca, F) of the trained surrogate for every bin, as
    mcg_compute_part_surrogate forms them; None for a bin outside the
    training box"""
    import hostcheck_ffi as H
    import mlp_ref as R
    from mcmax_b200 import surrogate as S
    params, _ = S.load(os.path.join(os.path.dirname(HERE), "mcmax_b200", "data", "surrogate_nf20.npz"))
    out = []
    for p in parts:
        lam, n, k = np.asarray(p["lam"], float), np.atleast_2d(p["e1"])[0], np.atleast_2d(p["e2"])[0]
        ns, por = int(p["ns"]), (p["porosity"] if p["blend"] else 0.0)
        lo, hi = math.log10(p["amin"]), math.log10(p["amax"])
        r = 10.0 ** (lo + (hi - lo) * np.arange(ns) / (ns - 1)) if ns > 1 else np.array([10.0 ** ((lo + hi) / 2)])
        mw = r ** (-p["apow"] + 1.0) * r ** 3 if ns > 1 else np.ones(1)
        mw = mw / mw.sum()
        v = np.array([[math.log10(rk), math.log10(lam[l]), n[l], math.log10(k[l]), por, p["fmax"]]
                      for rk in r for l in range(lam.size)])
        if np.any(v < S.BOX_LO) or np.any(v > S.BOX_HI):
            out.append(None)
            continue
        x = (2.0 * (v - S.BOX_LO) / (S.BOX_HI - S.BOX_LO) - 1.0).astype(np.float32)
        y = R.forward(params, x)[0].astype(np.float64).reshape(ns, lam.size, -1)
        scale = S.RHO_TRAIN / float(np.atleast_1d(p["rho"])[0])
        ksk = 10.0 ** y[:, :, 1] * scale
        kabs = np.sum(mw[:, None] * 10.0 ** y[:, :, 0] * scale, 0)
        ksca = np.sum(mw[:, None] * ksk, 0)
        wgt = mw[:, None] * ksk
        F = np.zeros((lam.size, 6, NA))
        for l in range(lam.size):
            m = lambda i0, n0: np.sum(wgt[:, l, None] * y[:, l, i0:i0 + n0], 0) / wgt[:, l].sum()
            chi = np.r_[1.0, m(2, L)]
            F[l] = H.surr_phase(chi, m(14, L + 1), m(27, L + 1), m(40, L + 1), deltam=int(deltam))
        out.append((kabs, ksca, F))
    return out


def build(nrad=60, ntheta=40, nlam=100, ngrains=10):
    """Model fields of the reduced learned-opacities deck (the builder of
    model.learned_disk_model with the oracle's ComputePart)"""
    import oracle_ffi as O
    from mcmax_b200 import model as M, api
    lam, nu = M.wavelength_grid(0.1, 3000.0, nlam)
    rstar_cm = 2.5 * M.RSUN
    R, Theta, thet, SinTheta = M.spatial_grid(rstar_cm, 0.5, 100.0, nrad, ntheta)
    zone = dict(rin=0.5, rout=100.0, mdust=1e-3, denspow=1.0, sh=0.05 * math.sqrt(2.0), rsh=1.0, shpow=1.125)
    dens, V = M.zones_density(R, Theta, thet, [zone])
    BB = api.bb_table(lam)
    Fstar = np.array([math.pi * rstar_cm ** 2 * api.planck(10000.0, x) for x in lam])
    Lstar = M.integrate(nu, Fstar)
    parts, bins = M.learned_disk_parts(lam, ngrains)
    res = [O.compute_part(p["lam"], p["e1"], p["e2"], p["frac"], p["rho"], p["amin"], p["amax"], p["apow"], p["fmax"],
                          p["blend"], p["porosity"], p["ns"], p["nf"]) for p in parts]
    Kabs = np.array([r["kabs"] for r in res])
    Ksca = np.array([r["ksca"] for r in res])
    F = np.array([r["F"] for r in res])
    rg = [math.sqrt(a * b) * 1e-4 for a, b in bins]
    wmrn = M.mrn_abundances(rg, 0.01e-4, 1000e-4, 3.5)
    w0 = np.concatenate([wmrn / 3 for _ in range(3)])
    nr, nc = R.size - 1, Theta.size - 1
    wt = np.tile(w0, (nr, nc, 1))
    rho_grain = np.array([r["rho_av"] for r in res])
    rv = np.array([M.grain_rv(p["amin"], p["amax"], 3.5, p["ns"]) for p in parts])
    dens2, w2 = M.fixed_mp_settling(R, Theta, ntheta, dens, V, wt, rho_grain, rv, 1e-3, zone)
    kw = dict(nr=nr, nt=Theta.size, R=R, Theta=Theta, SinTheta=SinTheta, thet=thet, dens=dens2.reshape(-1),
              V=V.reshape(-1), ncomp=len(parts), comp_w=w2.reshape(nr * nc, len(parts)), nlam=nlam, lam=lam, nu=nu,
              Kabs=Kabs, Ksca=Ksca, F=F, BB=BB, Fstar=Fstar, Lstar=Lstar, Tstar=10000.0, Rstar_cm=rstar_cm,
              scat_how=2, bins=bins, w=w0, rho_grain=rho_grain, rv=rv)
    kw["_parts"] = parts
    return kw


def run(args):
    """one oracle run with the exact, clipped or delta-M matrices"""
    kw, variant, seed, nphot = args
    import oracle_ffi as O
    from mcmax_b200 import model as M
    kw = dict(kw)
    parts = kw.pop("_parts")
    if variant in ("clipped", "deltam"):
        F = kw["F"].copy()
        for c in range(F.shape[0]):
            for l in range(F.shape[1]):
                F[c, l] = rebuild(F[c, l], variant == "deltam")
        kw["F"] = F
    elif variant != "exact":
        net = network_optics(parts, variant != "net_plain")
        Kabs, Ksca, F = kw["Kabs"].copy(), kw["Ksca"].copy(), kw["F"].copy()
        for c, o in enumerate(net):
            if o is None:
                continue
            if variant in ("net_deltam", "net_plain", "netk_exactF"):
                Kabs[c], Ksca[c] = o[0], o[1]
            if variant in ("net_deltam", "net_plain", "exactk_netF"):
                F[c] = o[2]
        kw.update(Kabs=Kabs, Ksca=Ksca, F=F)
    m = M.Model(**kw)
    t0 = time.time()
    o = O.mcradiation(m, nphot, seed=seed, randomwalk=True, factRW=10.0, maxinteract=100000)
    return variant, seed, time.time() - t0, o["EJv"], o["Nabs"], o["spec"], o["ispec"], m.nt


if __name__ == "__main__":
    nphot = int(float(sys.argv[1])) if len(sys.argv) > 1 else 10_000_000
    import hostcheck_ffi
    hostcheck_ffi.load()  # build the harness once, before the workers start
    t0 = time.time()
    kw = build()
    print("built in %.0f s" % (time.time() - t0), flush=True)
    if "network" in sys.argv[2:]:
        variants = [("exact", 2), ("net_deltam", 1), ("net_deltam", 3), ("net_plain", 1), ("netk_exactF", 1),
                    ("exactk_netF", 1)]
    else:
        variants = [("exact", 2), ("clipped", 1), ("deltam", 1), ("clipped", 3), ("deltam", 3)]
    jobs = [(kw, "exact", 1, nphot)] + [(kw, v, sd, nphot) for v, sd in variants]
    with mp.get_context("spawn").Pool(min(len(jobs), os.cpu_count() or 1)) as pool:
        outs = pool.map(run, jobs)
    _, _, _, ej_ref, nabs_ref, spec_ref, ispec_ref, nt = outs[0]
    # cells outside the star cell with >= 1e3 absorption events in the reference run
    sel = (nabs_ref >= 1000) & (np.arange(ej_ref.size) >= nt - 1) & (ej_ref > 0)
    res = {"cells": int(sel.sum())}
    for variant, seed, dt, ej, _, spec, ispec, _ in outs[1:]:
        rel = np.abs((ej[sel] / ej_ref[sel]) ** 0.25 - 1)  # T ~ EJv^(1/4)
        a, b = spec_ref[:, 1:].sum(1), spec[:, 1:].sum(1)
        ok = (ispec_ref[:, 1:].sum(1) > 2500) & (ispec[:, 1:].sum(1) > 2500) & (a > 0)
        res["%s_s%d" % (variant, seed)] = {"time_s": round(dt), "T_within_1pct": float(np.mean(rel < 0.01)),
                                           "T_median_rel": float(np.median(rel)),
                                           "sed_lam_median_rel": float(np.median(np.abs(b[ok] / a[ok] - 1)))}
    print(json.dumps(res))
