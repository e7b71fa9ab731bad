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

    python tests/phase_representation_study.py [NPHOT]"""
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
    return kw


def run(args):
    """one oracle run with the exact, clipped or delta-M matrices"""
    kw, variant, seed, nphot = args
    import oracle_ffi as O
    from mcmax_b200 import model as M
    kw = dict(kw)
    if variant != "exact":
        F = kw["F"].copy()
        for c in range(F.shape[0]):
            for l in range(F.shape[1]):
                F[c, l] = rebuild(F[c, l], variant == "deltam")
        kw["F"] = F
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
    jobs = [(kw, "exact", 1, nphot), (kw, "exact", 2, nphot), (kw, "clipped", 1, nphot), (kw, "deltam", 1, nphot),
            (kw, "clipped", 3, nphot), (kw, "deltam", 3, nphot)]
    with mp.get_context("spawn").Pool(6) as pool:
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
