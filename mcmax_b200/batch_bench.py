"""Batched models (the 256-disk sweep): one launch over all models vs one
mcg_mcradiation call per model.

    python -m mcmax_b200.batch_bench [--nmodels 256] [--scale 1.0] [--seed 3]

Sweep (seeded): Mdust log-uniform 1e-6..1e-2 Msun, Rin uniform 0.1..5 AU,
flaring index uniform 1.0..1.3, surface-density exponent uniform 0.5..1.5,
nr uniform 60..250, ntheta uniform 40..160, nlam 100 (0.1..3000 micron),
packets log-uniform 1e6..1e7 (times --scale).  Dust: one synthetic .lnk,
MRN 0.1-1 micron in 20 bins (DHS opacities computed once on the GPU), full
Mueller scattering, maxinteract 1e5, modified random walk (factRW 10; a
uniform mixture's thick cells share one diffusion row), mixed transport.
Prints one JSON line: packets/s of the batched launch (autotuned shape,
CUDA graph) and of the per-model calls."""
import argparse
import json
import math
import time

import numpy as np

from . import api
from . import model as M


def sweep(ctx, nmodels, seed):
    rng = np.random.default_rng(seed)
    lam, nu = M.wavelength_grid(0.1, 3000.0, 100)
    base = M.disk_model(ctx, nrad=20, ntheta=12, nlam=100, mdust=1e-5)  # opacities and star once
    out = []
    for _ in range(nmodels):
        mdust = 10 ** rng.uniform(-6, -2)
        rin = rng.uniform(0.1, 5.0)
        shpow = rng.uniform(1.0, 1.3)
        denspow = rng.uniform(0.5, 1.5)
        nrad = int(rng.integers(60, 251))
        ntheta = int(rng.integers(40, 161))
        R, Theta, thet, SinTheta = M.spatial_grid(base.Rstar_cm, rin, 100.0, nrad, ntheta)
        dens, V = M.zones_density(R, Theta, thet, [dict(rin=rin, rout=100.0, mdust=mdust, denspow=denspow,
                                                        sh=0.05 * math.sqrt(2.0), rsh=1.0, shpow=shpow)])
        nr, nt = R.size - 1, Theta.size
        m = M.Model(nr=nr, nt=nt, R=R, Theta=Theta, SinTheta=SinTheta, thet=thet, dens=dens.reshape(-1),
                    V=V.reshape(-1), ncomp=base.ncomp, comp_w=np.tile(base.w, (nr * (nt - 1), 1)), nlam=base.nlam,
                    lam=base.lam, nu=base.nu, Kabs=base.Kabs, Ksca=base.Ksca, F=base.F, BB=base.BB,
                    Fstar=base.Fstar, Lstar=base.Lstar, Tstar=base.Tstar, Rstar_cm=base.Rstar_cm, scat_how=2,
                    bins=base.bins, w=base.w)
        out.append((m, int(10 ** rng.uniform(6, 7))))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nmodels", type=int, default=256)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--sequential", type=int, default=1, help="also time one call per model")
    a = ap.parse_args()
    ctx = api.Context(0)
    t0 = time.perf_counter()
    ms = sweep(ctx, a.nmodels, a.seed)
    ids = [ctx.add_model(m) for m, _ in ms]
    t_build = time.perf_counter() - t0
    nphot = [max(1000, int(n * a.scale)) for _, n in ms]
    run = dict(precision="mixed", randomwalk=True, factRW=10.0, maxinteract=100000)
    seeds = list(range(1000, 1000 + a.nmodels))
    # warm-up + autotune (1/50 of the packets per shape), then graph capture
    _, _, info0 = ctx.mcradiation_batch(ids, nphot, seeds, autotune=True, use_graph=True, fetch=False, **run)
    _, outs, info = ctx.mcradiation_batch(ids, nphot, [s + 7 for s in seeds], autotune=True, use_graph=True,
                                          fetch=False, **run)
    total = sum(nphot)
    line = {"nmodels": a.nmodels, "packets": total, "build_s": t_build, "batched_ms": info["device_ms"],
            "batched_packets_per_s": total / (info["device_ms"] * 1e-3),
            "shape": {k: info[k] for k in ("block", "blocks_per_sm", "chunk")}}
    if a.sequential:
        seq_ms = 0.0
        for (m, _), n, s in zip(ms, nphot, seeds):
            ctx.set_model(m)
            _, o = ctx.mcradiation(n, seed=s + 11, fetch=False, **run)
            seq_ms += o["device_ms"]
        line.update(sequential_ms=seq_ms, sequential_packets_per_s=total / (seq_ms * 1e-3),
                    speedup=seq_ms / info["device_ms"])
    print(json.dumps(line))


if __name__ == "__main__":
    main()
