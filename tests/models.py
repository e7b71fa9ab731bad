"""Small test models built on the CPU (opacities from the oracle), shared
by the CPU and GPU tests."""
import math

import numpy as np

import oracle_ffi as O
from mcmax_b200 import model as M


def small_disk(nrad=20, ntheta=12, nlam=30, ngrains=3, ns=2, nf=4, mdust=1e-5, scat_how=2, lam2=3000.0, kpref=0.03,
               amin=0.1, amax=1.0, tstar=10000.0, rstar=2.5, rin=0.5, rout=100.0, blend=True, porosity=0.25,
               fmax=0.8, cache={}):
    key = (nrad, ntheta, nlam, ngrains, ns, nf, mdust, scat_how, lam2, kpref, amin, amax, tstar, rstar, rin, rout,
           blend, porosity, fmax, M.AU, M.RSUN, M.MSUN)
    if key in cache:
        return cache[key]
    import hashlib
    import os
    import tempfile
    fn = os.path.join(tempfile.gettempdir(), "mcmax_test_models",
                      hashlib.sha1(repr(key).encode()).hexdigest()[:16] + ".npz")
    if os.path.exists(fn):
        z = np.load(fn, allow_pickle=False)
        d = {k: z[k] for k in z.files}
        for k in ("nr", "nt", "ncomp", "nlam", "scat_how"):
            d[k] = int(d[k])
        for k in ("Lstar", "Tstar", "Rstar_cm"):
            d[k] = float(d[k])
        d["bins"] = [tuple(b) for b in d["bins"]]
        mdl = M.Model(**d)
        cache[key] = mdl
        return mdl
    lam, nu = M.wavelength_grid(0.1, lam2, nlam)
    n, k = M.synthetic_lnk(lam, kpref)
    bins = M.grain_bins(amin, amax, ngrains)
    Kabs, Ksca, F = [], [], []
    for a, b in bins:
        r = O.compute_part(lam, n, k, [1.0], [3.0], a, b, 3.5, fmax, blend, porosity, ns, nf)
        Kabs.append(r["kabs"])
        Ksca.append(r["ksca"])
        F.append(r["F"])
    rstar_cm = rstar * M.RSUN
    R, Theta, thet, SinTheta = M.spatial_grid(rstar_cm, rin, rout, nrad, ntheta)
    dens, V = M.zones_density(R, Theta, thet, [dict(rin=rin, rout=rout, mdust=mdust, denspow=1.0,
                                                    sh=0.05 * math.sqrt(2.0), rsh=1.0, shpow=1.125)])
    BB = O.bb_table(lam)
    L = O.load()
    Fstar = np.array([math.pi * rstar_cm ** 2 * L.orc_planck(tstar, float(x)) for x in lam])
    Lstar = M.integrate(nu, Fstar)
    rg = [math.sqrt(a * b) * 1e-4 for a, b in bins]
    w = M.mrn_abundances(rg, amin * 1e-4, amax * 1e-4, 3.5)
    nr = R.size - 1
    nt = Theta.size
    Ksca = np.array(Ksca)
    if scat_how == 0:
        Ksca = np.zeros_like(Ksca)
    mdl = M.Model(nr=nr, nt=nt, R=R, Theta=Theta, SinTheta=SinTheta, thet=thet, dens=dens.reshape(-1),
                  V=V.reshape(-1), ncomp=len(bins), comp_w=np.tile(w, (nr * (nt - 1), 1)), nlam=nlam, lam=lam,
                  nu=nu, Kabs=np.array(Kabs), Ksca=Ksca, F=np.array(F), BB=BB, Fstar=Fstar, Lstar=Lstar,
                  Tstar=tstar, Rstar_cm=rstar_cm, scat_how=scat_how, bins=bins, w=w)
    cache[key] = mdl
    try:
        os.makedirs(os.path.dirname(fn), exist_ok=True)
        np.savez(fn + ".tmp.npz", **{k: np.asarray(v) for k, v in mdl.__dict__.items()})
        os.replace(fn + ".tmp.npz", fn)
    except OSError:
        pass
    return mdl
