"""The full disk model: the learned-opacities disk iterated to hydrostatic
equilibrium with settled grains, then observed with ray-traced spectra and
images, on one GPU.

    python -m mcmax_b200.full_model [--nphot 1e9] [--passes 5] [--nrad 300] [--ntheta 200] [--nlam 300]
                                    [--alpha 1e-4] [--angles 20,45,80] [--npix 512] [--nint 1000]
                                    [--image-lam 1,10,100] [--scatter-nphot 1000] [--scatter-nstar 1000]
                                    [--check] [--floor] [--out DIR]

Deck: the learned-opacities disk (three compositions of 50 log size bins
from 0.01 to 1000 micron each, MRN within a composition, porosity and
fmax per composition; Mdust 1e-3 Msun, Rin 0.5 AU, Rout 100 AU, H/R 0.05
at 1 AU with flaring 1.125) on nr x ntheta cells and nlam wavelengths, the
zone's vertical structure not fixed: hydrostatic equilibrium
(DiskStructure) with FixedMPSettling at alpha recomputed before every
structure pass (DiskStructure.f:108, MPSettling.f:132-168).  Opacities
from the surrogate network (the DHS kernels outside its box); packet loop
in mixed precision with the random walk (factRW 10) and the overflow
roulette at maxinteract 1e5.

Loop (Main.f:202-792, mcmax_b200.structure.iterate): the optically thin
start (three structure passes), then --passes structure passes, each after
a packet run of --nphot packets with its own Philox key, and a last packet
run on the final structure; every run is followed by the post-run
temperatures and Diffuse.  Then for every inclination the ray-traced
spectrum (the 'SPECTRUM' observation: 45 angles, 2 points per radial
cell, at the model's wavelengths) and an --npix square image at each
--image-lam (the 'IMAGE' observation, field of view the grid's diameter).
Both carry the scattered light of TraceMono's field: per wavelength
--scatter-nstar packets of single-scattered starlight and --scatter-nphot
Monte Carlo packets, five exit rays per cell (an observation's defaults,
Telescope.f:606-619).

--check runs the same pipeline again in the FP64 form with the DHS
opacities (the FP64 GPU oracle of the mixed form) and reports the
agreement: final per-cell temperatures of the cells with at least 1e3
absorption events in the last packet run (within 1 %), the ray-traced
spectra (within 2 % where the flux is above 1e-6 of its peak) and the
images (total flux, and the pixels above 1e-3 of the peak within 5 %).
--floor runs the mixed pipeline once more with another seed and reports
the same statistics against the first run: the Monte Carlo noise floor of
the comparison, structure feedback included.

Prints one JSON line: the timings of every stage (device-synchronised
wall clock per call), the packet rate of every packet run, the structure
history (errT per pass) and, with --check, the agreement.  --out writes
denstemp.dat, spectrum<angle>.dat and ImageAI_*.fits (Jy per pixel at
100 pc) of the mixed-precision model."""
import argparse
import json
import math
import os
import time

import numpy as np

from . import api
from . import model as M
from . import outputs
from . import structure as S

RUN = dict(randomwalk=True, factRW=10.0, maxinteract=100_000)


def _surrogate_params():
    from . import surrogate as SU
    params, _ = SU.load(os.path.join(os.path.dirname(__file__), "data", "surrogate_nf20.npz"))
    return params


def _scatter(a, seed):
    return dict(nphot=a.scatter_nphot, nphot_star=a.scatter_nstar, seed=seed, nexits=5)


def pipeline(ctx, a, precision, opacity, seed, log=None):
    """One full model: returns dict(model, T, Nabs, history, passes
    (packets, seconds per packet run), timings, spectra {angle: flux},
    images {(angle, lam): image})."""
    t = {}
    t0 = time.perf_counter()
    params = _surrogate_params() if opacity == "surrogate" else None
    m, t_opac, served = M.learned_disk_model(ctx, opacity=opacity, params=params, nrad=a.nrad, ntheta=a.ntheta,
                                             nlam=a.nlam, mdust=a.mdust, alpha=a.alpha, settle=False)
    t["opacity_s"] = t_opac
    t["model_s"] = time.perf_counter() - t0
    zones = [(0.5, 100.0, 0.05 * math.sqrt(2.0), 1.0, 1.125, 1.0, 0)]
    fixed = dict(rho=m.rho_grain, rv=m.rv, alpha=a.alpha)
    passes = []
    clock = [time.perf_counter()]

    def on_pass(n, res, T):
        now = time.perf_counter()
        passes.append(dict(packets=int(n), run_s=now - clock[0], device_ms=float(res.get("device_ms", 0.0))))
        if log:
            log("%s packet run %d: %d packets, %.1f s" % (precision, len(passes), n, now - clock[0]))
        clock[0] = now

    orig = ctx.disk_structure

    def timed_structure(*args, **kw):
        s0 = time.perf_counter()
        out = orig(*args, **kw)
        dt = time.perf_counter() - s0
        t["structure_s"] = t.get("structure_s", 0.0) + dt
        clock[0] += dt
        return out

    ctx.disk_structure = timed_structure
    try:
        t1 = time.perf_counter()
        out = S.iterate(ctx, m, zones, 2.5 * M.MSUN, a.nphot, run=dict(RUN, seed=seed), maxiter=a.passes - 1,
                        epsiter=0.0, precision=precision, thin=True, fixed=fixed, on_pass=on_pass)
        t["loop_s"] = time.perf_counter() - t1
    finally:
        ctx.disk_structure = orig
    T = out["T"]
    ctx.set_model(m)
    spectra, images = {}, {}
    t2 = time.perf_counter()
    for ang in a.angle_list:
        spectra[ang], _ = ctx.trace_spectrum(T, m.lam, math.radians(ang), nphi=45, nr=2, scatter=_scatter(a, seed))
    t["spectra_s"] = time.perf_counter() - t2
    t3 = time.perf_counter()
    for ang in a.angle_list:
        for lam in a.lam_list:
            images[(ang, lam)] = ctx.trace_image(T, lam, math.radians(ang), npixel=a.npix, nint=a.nint,
                                                 scatter=_scatter(a, seed))["image"]
    t["images_s"] = time.perf_counter() - t3
    t["total_s"] = time.perf_counter() - t0
    return dict(model=m, T=T, Nabs=np.asarray(out["result"]["Nabs"]), history=out["history"], passes=passes,
                timings=t, spectra=spectra, images=images, served=served)


def agreement(ref, other):
    """other against ref (the FP64 + DHS pipeline): see the module text"""
    m = ref["model"]
    nc = m.nt - 1
    sel = (ref["Nabs"] >= 1000) & (np.arange(m.ncell) >= nc) & (ref["T"] > 0)
    rel = np.abs(other["T"][sel] / ref["T"][sel] - 1)
    out = {"cells_nabs_ge_1e3": int(sel.sum()), "T_within_1pct": float(np.mean(rel < 0.01)),
           "T_median_rel": float(np.median(rel)), "T_p95_rel": float(np.percentile(rel, 95))}
    sp = {}
    for ang, f in ref["spectra"].items():
        g = other["spectra"][ang]
        ok = f > 1e-6 * f.max()
        r = np.abs(g[ok] / f[ok] - 1)
        sp[str(ang)] = {"wavelengths": int(ok.sum()), "within_2pct": float(np.mean(r < 0.02)),
                        "median_rel": float(np.median(r)), "max_rel": float(r.max())}
    out["spectra"] = sp
    im = {}
    for key, f in ref["images"].items():
        g = other["images"][key]
        ok = f > 1e-3 * f.max()
        r = np.abs(g[ok] / f[ok] - 1)
        im["%g_deg_%g_um" % key] = {"total_flux_ratio": float(g.sum() / f.sum()), "bright_pixels": int(ok.sum()),
                                    "bright_within_5pct": float(np.mean(r < 0.05)),
                                    "bright_median_rel": float(np.median(r))}
    out["images"] = im
    return out


def _summary(p):
    pk = sum(x["packets"] for x in p["passes"])
    run_s = sum(x["run_s"] for x in p["passes"])
    return {"timings_s": p["timings"], "packet_runs": p["passes"], "packets": pk,
            "packets_per_s_loop": pk / run_s if run_s > 0 else None,
            "errT": [h["errT"] for h in p["history"]], "bins_served_by_network": p["served"]}


def write_outputs(outdir, p, distance_pc=100.0):
    os.makedirs(outdir, exist_ok=True)
    m = p["model"]
    files = [os.path.join(outdir, "denstemp.dat")]
    outputs.write_denstemp(files[0], m, p["T"])
    for ang, f in p["spectra"].items():
        files.append(outputs.write_spectrum(outdir, ang, m.lam, f, m.lam, m.Fstar, distance_pc))
    dcm = distance_pc * outputs.PARSEC
    rmax = float(m.R[-1])
    for (ang, lam), im in p["images"].items():
        path = os.path.join(outdir, outputs.image_name("AI", math.radians(ang), lam, rmax))
        files.append(outputs.write_image_fits(path, im * 1e23 / dcm ** 2, rmax))
    return files


def parse_args(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--nphot", type=float, default=1e9, help="packets per packet run")
    ap.add_argument("--passes", type=int, default=5, help="structure passes after the thin start")
    ap.add_argument("--nrad", type=int, default=300)
    ap.add_argument("--ntheta", type=int, default=200)
    ap.add_argument("--nlam", type=int, default=300)
    ap.add_argument("--mdust", type=float, default=1e-3)
    ap.add_argument("--alpha", type=float, default=1e-4)
    ap.add_argument("--angles", default="20,45,80")
    ap.add_argument("--npix", type=int, default=512)
    ap.add_argument("--nint", type=int, default=1000)
    ap.add_argument("--image-lam", default="1,10,100", help="image wavelengths, micron")
    ap.add_argument("--scatter-nphot", type=int, default=1000, help="scattered-light Monte Carlo packets per field")
    ap.add_argument("--scatter-nstar", type=int, default=1000, help="single-scattered starlight packets per field")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--check", action="store_true", help="also the FP64 + DHS pipeline, and the agreement")
    ap.add_argument("--floor", action="store_true", help="also the mixed pipeline with another seed (noise floor)")
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    a.nphot = int(a.nphot)
    a.angle_list = [float(x) for x in a.angles.split(",") if x]
    a.lam_list = [float(x) for x in a.image_lam.split(",") if x]
    if a.passes < 1:
        ap.error("--passes must be at least 1")
    return a


def main(argv=None):
    a = parse_args(argv)
    ctx = api.Context(0)
    log = lambda s: print(s, flush=True)
    res = {"workload": "full disk model: learned opacities, hydrostatic structure with settling, ray-traced "
                       "spectra and images",
           "config": {"nrad": a.nrad, "ntheta": a.ntheta, "nlam": a.nlam, "ngrains": 150, "mdust": a.mdust,
                      "alpha": a.alpha, "packets_per_run": a.nphot, "structure_passes": a.passes,
                      "packet_runs": a.passes + 1, "angles_deg": a.angle_list, "image_lam_um": a.lam_list,
                      "npix": a.npix, "nint": a.nint, "scatter_nphot": a.scatter_nphot,
                      "scatter_nstar": a.scatter_nstar}}
    mixed = pipeline(ctx, a, "mixed", "surrogate", a.seed, log)
    res["mixed_surrogate"] = _summary(mixed)
    if a.out:
        res["files"] = write_outputs(a.out, mixed)
    if a.check:
        ref = pipeline(ctx, a, "fp64", "dhs", a.seed + 1000, log)
        res["fp64_dhs"] = _summary(ref)
        res["agreement"] = agreement(ref, mixed)
        res["speedup_loop"] = res["mixed_surrogate"]["packets_per_s_loop"] / res["fp64_dhs"]["packets_per_s_loop"]
        res["speedup_total"] = ref["timings"]["total_s"] / mixed["timings"]["total_s"]
    if a.floor:
        again = pipeline(ctx, a, "mixed", "surrogate", a.seed + 2000, log)
        res["noise_floor"] = agreement(mixed, again)
    ctx.close()
    print(json.dumps(res))
    return res


if __name__ == "__main__":
    main()
