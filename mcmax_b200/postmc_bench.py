"""The steps after the packet loop on the precision disk deck's grid:
Diffuse (mcg_diffuse), the vertical structure (mcg_disk_structure), the
ray-traced spectrum (mcg_trace_spectrum) and the rectangular image
(mcg_trace_image: 500 x 500 pixels, 1000 points per image cell, at the
observation file's default wavelength, the middle of the grid's range),
each timed through the C-ABI.

    python -m mcmax_b200.postmc_bench [--nphot 2e7] [--angles 20,45,80] [--reps 3] [--npix 500] [--nint 1000]

Deck: Mdust 1e-3 Msun ZONES disk, nr 200 (+ star cell) x ntheta 120, nlam
200 from 0.1 to 3000 micron, MRN 0.1-1 micron in 20 DHS bins, full Mueller
scattering, random walk with factRW 10 (the bench.py workload).  One
mixed-precision packet run gives the temperatures, packet counts and
errors; then each step is run --reps times on them (the structure step on
the zone taken as not fixed, so that it integrates every column).  Prints
one JSON line with the wall time of each call (each call ends with a
device synchronisation) and the step's sizes."""
import argparse
import json
import math
import time

import numpy as np

from . import api
from . import model as M
from . import structure as S


def _time(fn, reps):
    out, best = None, float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        out = fn()
        best = min(best, time.perf_counter() - t0)
    return out, best


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nphot", type=float, default=2e7)
    ap.add_argument("--angles", default="20,45,80")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--nphi", type=int, default=45)
    ap.add_argument("--nr", type=int, default=2)
    ap.add_argument("--npix", type=int, default=500)
    ap.add_argument("--nint", type=int, default=1000)
    a = ap.parse_args()
    ctx = api.Context(0)
    m = M.disk_model(ctx, nrad=200, ntheta=120, nlam=200, mdust=1e-3, ngrains=20)
    ctx.set_model(m)
    n, res = ctx.mcradiation(int(a.nphot), precision="mixed", randomwalk=True, factRW=10.0, maxinteract=100000)
    T, dT, _ = ctx.finalize_t()
    out = {"deck": "precision disk, nr 200 x ntheta 120, nlam 200, 20 grains", "packets": int(n)}

    (Td, _, counts), t = _time(lambda: ctx.diffuse(res["Ni"], dT, T), a.reps)
    out["diffuse"] = {"s": t, "selected": counts[0], "unknowns": counts[1], "solved": counts[2],
                      "failed_passes": counts[3]}

    st = S.initial_state(m)
    Temp = np.maximum(Td, 2.7)
    zones = [(0.5, 100.0, 0.05 * math.sqrt(2.0), 1.0, 1.125, 1.0, 0)]
    _, t = _time(lambda: ctx.disk_structure(m.R, m.Theta, m.V, 2.5 * M.MSUN, zones, Temp, st["dens"], st["dens0"],
                                            st["gasdens"], st["w"], st["w0"]), a.reps)
    out["disk_structure"] = {"s": t, "columns": (m.nr - 1) * (m.ncomp + 1), "cells": m.ncell}

    from .outputs import spectrum_wavelengths
    lam_obs = spectrum_wavelengths(m.lam, m.lam[0], m.lam[-1])
    spectra = []
    for ang in [float(x) for x in a.angles.split(",") if x]:
        (flux, info), t = _time(lambda: ctx.trace_spectrum(Td, lam_obs, math.radians(ang), nphi=a.nphi, nr=a.nr),
                                a.reps)
        spectra.append({"angle_deg": ang, "s": t, "wavelengths": int(lam_obs.size), "image_radii": info[0],
                        "rays_per_wavelength": info[0] * a.nphi, "bad_rays": info[1],
                        "rays_per_s": info[0] * a.nphi * lam_obs.size / t})
    out["trace_spectrum"] = spectra
    lam_img = (m.lam[0] + m.lam[-1]) / 2.0
    images = []
    for ang in [float(x) for x in a.angles.split(",") if x]:
        r, t = _time(lambda: ctx.trace_image(Td, lam_img, math.radians(ang), npixel=a.npix, nint=a.nint,
                                             nphi=a.nphi, nr=a.nr), a.reps)
        pts = (r["info"][0] - 1) * a.nphi * a.nint
        images.append({"angle_deg": ang, "s": t, "lam": lam_img, "pixels": a.npix * a.npix, "image_radii": r["info"][0],
                       "points": pts, "points_per_s": pts / t, "sum_over_flux": float(r["image"].sum() / r["flux"])})
    out["trace_image"] = images
    print(json.dumps(out))
    ctx.close()


if __name__ == "__main__":
    main()
