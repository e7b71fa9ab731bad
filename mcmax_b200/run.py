"""Command-line run of the packet loop on an MCMax input deck, writing the
reference's result files:

    python -m mcmax_b200.run input.in Nphot [observation files] [-o outdir] [-s key=value]...
                             [--precision mixed|fp64|exact] [--opacity dhs|surrogate]
                             [--spectrum DEG]...

The arguments follow the reference's command line (Main.f:60-72 for -o,
Init.f:462-478 for -s): the deck, the packet count, an output directory
(created if missing) and keyword overrides applied after the deck.  One
pass of MCRadiation with the deck's run keywords (randomwalk, factrw,
maxinteract, nruns, idum), the post-Monte-Carlo temperatures
(Main.f:498-549), the diffusion step for poorly sampled thick cells when
nphotdiffuse > 0 or dtdiffuse < 1 (Main.f:561-563, on by default); when a
zone has no fixed structure (zoneN:fix, false by default) these passes
repeat with the hydrostatic vertical structure rebuilt in between
(mcmax_b200.structure) until the temperatures converge; then
denstemp.dat (format 5, InputOutput.f:6-227) and
the MCSpec<angle>.dat files (MCRadiation.f:738-762) in the output
directory.  --opacity surrogate serves the grain bins inside the network's
training box from the committed surrogate weights."""
import argparse
import math
import os
import sys

from . import model as M
from . import outputs


def _surrogate_parts(ctx):
    from . import surrogate as S
    params, _ = S.load(os.path.join(os.path.dirname(__file__), "data", "surrogate_nf20.npz"))
    return lambda parts: S.compute_part_surrogate(ctx, parts, params)[0]


def fixed_radii(zones, rin, rout):
    """zone edges strictly inside the grid, each once, sorted (D%Rfix,
    Init.f:1511-1517)"""
    out = []
    for z in zones:
        for r in (z[0], z[1]):
            if rin < r < rout and r not in out:
                out.append(r)
    return sorted(out)


def scatter_opts(ob, seed):
    """the scattered-light settings of an observation (Telescope.f:606-619,
    943-973): its nphot Monte Carlo and nphotstar starlight packets per
    field and nexits exit rays, the field keys from the run's seed"""
    return dict(nphot=int(ob.get("nphot", 1000)), nphot_star=int(ob.get("nphotstar", 1000)), seed=int(seed),
                nexits=int(ob.get("nexits", 5)))


def observe_image(ctx, m, T, ob, outdir, rfix=(), seed=42, posangle=0.0):
    """An IMAGE observation (Telescope.f:162-182) without convolution,
    noise or opening: the rays traced at the observation's wavelength
    (mcg_trace_image), the radial profile RImage_*.dat and, per field of
    view, the rectangular image ImageAI_*.fits in Jy/pixel and AU
    (scaletype 1) or mJy/arcsec^2 and arcsec (scaletype 2), with no
    interstellar extinction.  Returns the files written."""
    from .outputs import PARSEC
    angle = (math.pi * ob["inc"]) / 180.0
    lam0 = ob["lam1"]
    dcm = m.distance * PARSEC
    fovs = ob["fov"] or [2.0 * float(m.R[-1])]
    scaletype = int(ob.get("scaletype", 1))
    files = []
    for n, fov in enumerate(fovs):
        if scaletype == 2:
            fov = fov * dcm / PARSEC
            rscale, zscale = PARSEC / dcm, 1e3 * ((ob["npix"] / fov) * dcm / PARSEC) ** 2
        else:
            rscale, zscale = 1.0, 1.0
        r = ctx.trace_image(T, lam0, angle, npixel=ob["npix"], nint=ob["nint"], Rmax=fov / 2.0, pa=posangle,
                            nphi=ob["nphi"], nr=ob["nrad"], Rfix=rfix, seed=seed + n,
                            scatter=scatter_opts(ob, seed + n))
        if n == 0:
            files.append(outputs.write_rimage(os.path.join(outdir, outputs.rimage_name(angle, lam0, ob["flag"])),
                                              r["R"], r["rphi"], rscale, zscale, dcm, fov, ob["npix"],
                                              polarised=int(m.scat_how) == 2))
        im = r["image"] * 1e23 * zscale / dcm ** 2
        files.append(outputs.write_image_fits(
            os.path.join(outdir, outputs.image_name("AI", angle, lam0, fov / 2.0, ob["flag"])), im, fov / 2.0,
            rscale, scaletype))
    return files


def observe_ifu(ctx, m, T, ob, outdir, rfix=(), seed=42, posangle=0.0):
    """An IFU observation (Telescope.f:184-199): the image rays placed with
    the tau = 0.1 radius at 0.55 micron, then per wavelength of the
    observation (as a SPECTRUM's) and per field of view a rectangular image
    ImageAI_*.fits (mcg_trace_image with lam_path 0.55).  As in the
    reference, the fields of view of scaletype 2 are not converted from
    arcsec before they set the image size, only rscale and zscale change.
    Returns the files written."""
    from .outputs import PARSEC
    angle = (math.pi * ob["inc"]) / 180.0
    dcm = m.distance * PARSEC
    fovs = ob["fov"] or [2.0 * float(m.R[-1])]
    scaletype = int(ob.get("scaletype", 1))
    lam_obs = outputs.spectrum_wavelengths(m.lam, ob["lam1"], ob["lam2"], ob["nlam"], ob["lamfile"] or None)
    files = []
    n = 0
    for lam0 in lam_obs:
        for fov in fovs:
            if scaletype == 2:
                rscale, zscale = PARSEC / dcm, 1e3 * ((ob["npix"] / fov) * dcm / PARSEC) ** 2
            else:
                rscale, zscale = 1.0, 1.0
            r = ctx.trace_image(T, lam0, angle, npixel=ob["npix"], nint=ob["nint"], Rmax=fov / 2.0, pa=posangle,
                                nphi=ob["nphi"], nr=ob["nrad"], Rfix=rfix, seed=seed + n, lam_path=0.55,
                                scatter=scatter_opts(ob, seed + n))
            n += 1
            im = r["image"] * 1e23 * zscale / dcm ** 2
            files.append(outputs.write_image_fits(
                os.path.join(outdir, outputs.image_name("AI", angle, lam0, fov / 2.0, ob["flag"])), im, fov / 2.0,
                rscale, scaletype))
    return files


def observe_visibility(ctx, m, T, ob, outdir, rfix=(), seed=42, posangle=0.0, vis_norm_fov=True):
    """A VISIBILITY observation (Telescope.f:200-245): the image rays placed
    at 0.55 micron, then per wavelength (as a SPECTRUM's) the flux and, per
    baseline, the visibility and phase of the ray image (outputs.visibility;
    the rays come from mcg_trace_image with a one-pixel image).  Writes
    visibility<angle>.dat; returns its path."""
    from .outputs import PARSEC
    angle = (math.pi * ob["inc"]) / 180.0
    dcm = m.distance * PARSEC
    lam_obs = outputs.spectrum_wavelengths(m.lam, ob["lam1"], ob["lam2"], ob["nlam"], ob["lamfile"] or None)
    b, th = list(ob["b"]), list(ob["theta"])
    spec, V, ph = [], [], []
    for n, lam0 in enumerate(lam_obs):
        r = ctx.trace_image(T, lam0, angle, npixel=1, nint=1, nphi=ob["nphi"], nr=ob["nrad"], Rfix=rfix,
                            seed=seed + n, lam_path=0.55, scatter=scatter_opts(ob, seed + n))
        spec.append(1e23 * r["flux"] / dcm ** 2)
        vp = [outputs.visibility(r["R"], r["rphi"], bk, math.pi * tk / 180.0, lam0, dcm, ob["d"], posangle,
                                 vis_norm_fov) for bk, tk in zip(b, th)]
        V.append([x[0] for x in vp])
        ph.append([x[1] for x in vp])
    return outputs.write_visibility(outdir, ob["inc"], lam_obs, spec, b, th, V, ph, ob["flag"])


def observe_basevis(ctx, m, T, ob, outdir, rfix=(), seed=42, posangle=0.0, vis_norm_fov=True):
    """A BASEVIS observation (Telescope.f:246-291): the image rays placed at
    lam1, then for each wavelength lamN (traced again only when it differs
    from the one before) the visibility and phase on 100 baselines from
    base1 to base2, at the baseline angle angleN of that wavelength.
    Writes basevis<angle>.dat; returns its path."""
    from .outputs import PARSEC
    angle = (math.pi * ob["inc"]) / 180.0
    dcm = m.distance * PARSEC
    lams = list(ob.get("lams") or [ob["lam1"]])
    b = list(ob["b"]) + [0.0] * max(0, 2 - len(ob["b"]))
    th = list(ob["theta"]) + [0.0] * max(0, len(lams) - len(ob["theta"]))
    base = [b[0] + (b[1] - b[0]) * ((k - 1.0) / 99.0) for k in range(1, 101)]
    V, ph = [], []
    r = None
    for j, lam0 in enumerate(lams):
        if j == 0 or lam0 != lams[j - 1]:
            r = ctx.trace_image(T, lam0, angle, npixel=1, nint=1, nphi=ob["nphi"], nr=ob["nrad"], Rfix=rfix,
                                seed=seed + j, lam_path=ob["lam1"], scatter=scatter_opts(ob, seed + j))
        vp = [outputs.visibility(r["R"], r["rphi"], bk, math.pi * th[j] / 180.0, lam0, dcm, ob["d"], posangle,
                                 vis_norm_fov) for bk in base]
        V.append([x[0] for x in vp])
        ph.append([x[1] for x in vp])
    return outputs.write_basevis(outdir, ob["inc"], base, lams, th[:len(lams)], 1e23 * r["flux"] / dcm ** 2, V, ph,
                                 ob["flag"])


def run_deck(ctx, deck, nphot, outdir=".", overrides=(), precision="mixed", opacity="dhs", compute_parts=None,
             spectra=(), spectrum_nphi=45, spectrum_nr=2, observations=()):
    """Build the deck's model, run the packet loop and the diffusion step
    and write the result files; for each inclination in `spectra` [deg]
    also the ray-traced spectrum (mcg_trace_spectrum) as
    spectrum<angle>.dat.  Returns dict(model, run, nphot, result, T,
    diffused (the counts of mcg_diffuse, or None), structure, files).
    observations: MCMax observation files; their SPECTRUM observations are
    ray-traced the same way, their IMAGE observations give RImage_*.dat
    and ImageAI_*.fits (observe_image), IFU observations one ImageAI_*.fits
    per wavelength (observe_ifu); other kinds are skipped and listed in
    'skipped'."""
    if compute_parts is None and opacity == "surrogate":
        compute_parts = _surrogate_parts(ctx)
    elif opacity not in ("dhs", "surrogate"):
        raise ValueError("opacity: 'dhs' or 'surrogate'")
    m, run = M.deck_model(ctx, deck, overrides, compute_parts=compute_parts)
    rad = {k: run[k] for k in ("seed", "randomwalk", "factRW", "maxinteract", "maxruntime", "nruns")}
    diffused = structure = None
    if run.get("iterate", any(not z[6] for z in run["zones"])):
        # a zone without a fixed structure, or iter=.true.: structure
        # iterations (Init.f:563,1519) from the optically thin structure
        from . import structure as S
        structure = S.iterate(ctx, m, run["zones"], run["Mstar"], nphot, run=rad, maxiter=run["maxiter"],
                              epsiter=run["epsiter"], nphotdiffuse=run["nphotdiffuse"], dtdiffuse=run["dtdiffuse"],
                              precision=precision, thin=True, settling=run.get("settling"), fixed=run.get("fixed"))
        T, n, res = structure["T"], structure["nphot"], structure["result"]
    else:
        if run.get("thin_start"):
            # a power-law density: its vertical structure at the optically
            # thin temperatures, then one pass (Init.f:3924-3960)
            from . import structure as S
            S.thin_start(ctx, m, run["zones"], run["Mstar"], settling=run.get("settling"), fixed=run.get("fixed"))
        ctx.set_model(m)
        n, res = ctx.mcradiation(int(nphot), precision=precision, **rad)
        T, dT, dE = ctx.finalize_t()
        if run["nphotdiffuse"] > 0 or run["dtdiffuse"] < 1.0:
            T, _, diffused = ctx.diffuse(res["Ni"], dT, T, run["nphotdiffuse"], run["dtdiffuse"], run["factRW"])
    os.makedirs(outdir, exist_ok=True)
    if run.get("outputfits"):
        files = [outputs.write_denstemp_fits(os.path.join(outdir, "denstemp.fits.gz"), m, T)]
    else:
        files = [os.path.join(outdir, "denstemp.dat")]
        outputs.write_denstemp(files[0], m, T)
    names = outputs.write_mcspec(outdir, m, res, distance_pc=m.distance)
    files += [os.path.join(outdir, x) for x in names + ["MCSpec.dat"]]
    todo = [dict(inc=a, lam1=m.lam[0], lam2=m.lam[-1], nlam=-1, lamfile="", nphi=spectrum_nphi, nrad=spectrum_nr,
                 flag="") for a in spectra]
    skipped, images = [], []
    for path in observations:
        for ob in outputs.read_observations(path, m.lam, run.get("incangle", 45.0), rout=m.R[-1],
                                            vis_norm_fov=run.get("vis_norm_fov", True)):
            {"SPECTRUM": todo, "IMAGE": images, "IFU": images, "VISIBILITY": images,
             "BASEVIS": images}.get(ob["kind"], skipped).append(ob)
    rfix = fixed_radii(run["zones"], m.R[1], m.R[-1])
    for ob in todo:
        lam_obs = outputs.spectrum_wavelengths(m.lam, ob["lam1"], ob["lam2"], ob["nlam"], ob["lamfile"] or None)
        flux, _ = ctx.trace_spectrum(T, lam_obs, math.radians(ob["inc"]), nphi=ob["nphi"], nr=ob["nrad"], Rfix=rfix,
                                     scatter=scatter_opts(ob, run["seed"]))
        files.append(outputs.write_spectrum(outdir, ob["inc"], lam_obs, flux, m.lam, m.Fstar, m.distance,
                                            flag=ob["flag"], polarised=int(m.scat_how) == 2))
    for ob in images:
        if ob["kind"] == "BASEVIS":
            files.append(observe_basevis(ctx, m, T, ob, outdir, rfix, seed=run["seed"],
                                         posangle=run.get("posangle", 0.0),
                                         vis_norm_fov=ob.get("vis_norm_fov", True)))
            continue
        if ob["kind"] == "VISIBILITY":
            files.append(observe_visibility(ctx, m, T, ob, outdir, rfix, seed=run["seed"],
                                            posangle=run.get("posangle", 0.0),
                                            vis_norm_fov=ob.get("vis_norm_fov", True)))
            continue
        observe = observe_ifu if ob["kind"] == "IFU" else observe_image
        files += observe(ctx, m, T, ob, outdir, rfix, seed=run["seed"], posangle=run.get("posangle", 0.0))
    return dict(model=m, run=run, nphot=n, result=res, T=T, diffused=diffused, structure=structure, files=files,
                skipped=[ob["kind"] for ob in skipped])


def parse_args(argv):
    ap = argparse.ArgumentParser(prog="python -m mcmax_b200.run", description=__doc__.split("\n\n")[0])
    ap.add_argument("deck")
    ap.add_argument("nphot", type=lambda s: int(float(s)))
    ap.add_argument("observations", nargs="*", help="MCMax observation files (SPECTRUM and IMAGE observations are traced)")
    ap.add_argument("-o", dest="outdir", default=".")
    ap.add_argument("-s", dest="overrides", action="append", default=[], metavar="key=value")
    ap.add_argument("--precision", choices=("mixed", "fp64", "exact"), default="mixed")
    ap.add_argument("--opacity", choices=("dhs", "surrogate"), default="dhs")
    ap.add_argument("--spectrum", dest="spectra", action="append", type=float, default=[], metavar="DEG",
                    help="write the ray-traced spectrum at this inclination (repeatable)")
    ap.add_argument("--spectrum-nphi", type=int, default=45)
    ap.add_argument("--spectrum-nr", type=int, default=2)
    ap.add_argument("--device", type=int, default=0)
    return ap.parse_args(argv)


def main(argv=None, context=None):
    a = parse_args(sys.argv[1:] if argv is None else argv)
    if context is None:
        from .api import Context
        context = Context
    ctx = context(a.device)
    try:
        r = run_deck(ctx, a.deck, a.nphot, a.outdir, a.overrides, a.precision, a.opacity, spectra=a.spectra,
                     spectrum_nphi=a.spectrum_nphi, spectrum_nr=a.spectrum_nr, observations=a.observations)
    finally:
        ctx.close()
    print("packets %d, %d cells, T %.1f-%.1f K, wrote %s" % (r["nphot"], r["T"].size, r["T"].min(), r["T"].max(),
                                                             ", ".join(os.path.basename(f) for f in r["files"][:2])
                                                             + ", ..."))
    return r


if __name__ == "__main__":
    main()
