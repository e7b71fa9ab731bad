"""The reference's ASCII output files, written from the library's results so
that MCMax's own readers and plotting scripts take them unchanged.

    write_denstemp(path, model, T)        denstemp.dat (outputstruct,
                                          InputOutput.f:6-227, format 5 with
                                          DENS, TEMP, COMP, GASDENS, DENS0 as
                                          Main.f:605 writes it)
    read_denstemp(path)                   the same file back
    write_denstemp_fits(path, model, T)   denstemp.fits.gz, the same arrays as
                                          FITS images (outputstruct_fits,
                                          InputOutput.f:230-574)
    read_denstemp_fits(path)              the same file back
    write_mcspec(outdir, model, result)   MCSpec<angle>.dat per inclination
                                          bin and MCSpec.dat
                                          (MCRadiation.f:738-762)
    spectrum_wavelengths(lam, lam1, lam2) the wavelengths of a ray-traced
                                          spectrum (Telescope.f:40-52)
    write_spectrum(outdir, angle, ...)    spectrum<angle>.dat of a ray-traced
                                          spectrum (Telescope.f:140-160)

Cells are written for ir = 1..nR-1 (the star cell is left out) and it =
1..nTheta-1, radius and angle at the cell middles (D%R_av in cm, D%theta_av
in radians from the pole).  Numbers are written in free format, one or a
row per line, as list-directed Fortran output is read back.
"""
import math
import os

import numpy as np

from . import model as M

# single-precision literal widened to real*8, as Modules.f:9 holds it
PARSEC = float(np.float32(3.08568025e18))


def _r_av_cm(R):
    R = np.asarray(R, float)
    return M.AU * 10.0 ** ((np.log10(R[:-1]) + np.log10(R[1:])) / 2.0)


def _num(x):
    return " %.16E" % float(x)


def write_denstemp(path, model, T, dens0=None, gas2dust=100.0):
    """denstemp.dat of a model and its cell temperatures T (ncell, the
    library's cell order c = i*(nt-1) + (j-1)).  dens0: the dust density
    before settling (defaults to the model's density); the gas density is
    written as dens0 * gas2dust (C%gasdens*gas2dust)."""
    nr, nc = model.nr, model.nt - 1
    ng = model.ncomp
    dens = np.asarray(model.dens, float).reshape(nr, nc)
    T = np.asarray(T, float).reshape(nr, nc)
    comp = np.asarray(model.comp_w, float).reshape(nr, nc, ng)
    d0 = dens if dens0 is None else np.asarray(dens0, float).reshape(nr, nc)
    r_av = _r_av_cm(model.R)
    th = M.theta_centres(nc)
    with open(path, "w") as f:
        f.write("# Format number\n")
        f.write("%6d\n" % 5)
        f.write("# NR, NT, NGRAINS, NGRAINS2\n")
        f.write("%6d%6d%6d%6d\n" % (nr - 1, nc, ng, 1))
        f.write("# Spherical radius grid [cm] (middle of cell)\n")
        for i in range(1, nr):
            f.write(_num(r_av[i]) + "\n")
        f.write("# Theta grid [rad, from pole] (middle of cell)\n")
        for j in range(nc):
            f.write(_num(th[j]) + "\n")
        blocks = (("# Density array (for ir=0,nr-1 do for it=0,nt-1 do ...)", dens),
                  ("# Temperature array (for ir=0,nr-1 do for it=0,nt-1 do ...)", T))
        for title, a in blocks:
            f.write(title + "\n")
            for i in range(1, nr):
                for j in range(nc):
                    f.write(_num(a[i, j]) + "\n")
        f.write("# Composition array (for ir=0,nr-1 do for it=0,nt-1 do ...)\n")
        for i in range(1, nr):
            for j in range(nc):
                f.write("".join(_num(v) for v in comp[i, j]) + "\n")
        f.write("# Gas density array (for ir=0,nr-1 do for it=0,nt-1 do ...)\n")
        for i in range(1, nr):
            for j in range(nc):
                f.write(_num(d0[i, j] * gas2dust) + "\n")
        f.write("# Density0 array (for ir=0,nr-1 do for it=0,nt-1 do ...)\n")
        for i in range(1, nr):
            for j in range(nc):
                f.write(_num(d0[i, j]) + "\n")


def read_denstemp(path):
    """dict with r_av, theta_av, dens, T, comp, gasdens, dens0 ((nr-1, nt-1)
    arrays) from a format-5 denstemp.dat"""
    with open(path) as f:
        lines = [ln for ln in f.read().splitlines() if ln.strip() and not ln.lstrip().startswith("#")]
    fmt = int(lines[0])
    if fmt != 5:
        raise ValueError("denstemp format %d: only format 5 is read" % fmt)
    nr, nt, ng, ng2 = (int(x) for x in lines[1].split())
    k = 2
    r_av = np.array([float(x) for x in lines[k:k + nr]])
    k += nr
    th = np.array([float(x) for x in lines[k:k + nt]])
    k += nt

    def block(width=1):
        nonlocal k
        rows = [[float(x) for x in ln.split()] for ln in lines[k:k + nr * nt]]
        k += nr * nt
        a = np.array(rows)
        return a.reshape(nr, nt, width) if width > 1 else a.reshape(nr, nt)

    dens = block()
    T = block()
    comp = block(ng)
    gas = block()
    dens0 = block()
    return dict(r_av=r_av, theta_av=th, dens=dens, T=T, comp=comp, gasdens=gas, dens0=dens0, ngrains=ng)


def write_denstemp_fits(path, model, T, dens0=None, gas2dust=100.0, rin=None, rout=None, nlam=None):
    """denstemp.fits(.gz) as outputstruct_fits writes it (InputOutput.f:230-
    574) for DENS, TEMP, COMP, GASDENS, DENS0: a primary image (nR-1) x
    (nTheta-1) x 2 of the cell-centre radius [AU] and angle, with the
    keywords RIN, ROUT, NR, NTHETA, NGRAINS, NGRAINS2, NLAM, NHDU and
    'HDU n' naming the extensions, then one image per quantity (COMP: w and
    wopac, (nR-1) x (nTheta-1) x ngrains x 2).  A name ending in .fits gets
    .gz as in the reference."""
    from . import particle_fits as PF
    if path.endswith(".fits"):
        path = path + ".gz"
    nr, nc, ng = model.nr, model.nt - 1, model.ncomp
    dens = np.asarray(model.dens, float).reshape(nr, nc)[1:]
    T = np.asarray(T, float).reshape(nr, nc)[1:]
    comp = np.asarray(model.comp_w, float).reshape(nr, nc, ng)[1:]
    d0 = dens if dens0 is None else np.asarray(dens0, float).reshape(nr, nc)[1:]
    r_av = _r_av_cm(model.R)[1:] / M.AU
    th = M.theta_centres(nc)
    vars_ = ["DENS", "TEMP", "COMP", "GASDENS", "DENS0"]
    cards = [PF._card("SIMPLE", True, "file does conform to FITS standard"),
             PF._card("BITPIX", -64, "number of bits per data pixel"), PF._card("NAXIS", 3, "number of data axes"),
             PF._card("NAXIS1", nr - 1, "length of data axis 1"), PF._card("NAXIS2", nc, "length of data axis 2"),
             PF._card("NAXIS3", 2, "length of data axis 3"),
             PF._card("EXTEND", True, "FITS dataset may contain extensions"),
             PF._card("Rin", float(model.R[1] if rin is None else rin), "[AU]"),
             PF._card("Rout", float(model.R[-1] if rout is None else rout), "[AU]"),
             PF._card("nR", nr - 1), PF._card("nTheta", nc), PF._card("ngrains", ng), PF._card("ngrains2", 1),
             PF._card("nlam", int(model.nlam if nlam is None else nlam)), PF._card("nHDU", len(vars_))]
    cards += [PF._card("HDU%2d" % (i + 1), v) for i, v in enumerate(vars_)]
    grid = np.stack([np.broadcast_to(r_av[None, :], (nc, nr - 1)), np.broadcast_to(th[:, None], (nc, nr - 1))])
    raw = PF._header(cards) + PF._data(grid)
    comp4 = np.stack([comp.transpose(2, 1, 0), np.ones((ng, nc, nr - 1))])      # (2, ng, nc, nr-1)
    blocks = {"DENS": dens.T, "TEMP": T.T, "COMP": comp4, "GASDENS": (d0 * gas2dust).T, "DENS0": d0.T}
    for v in vars_:
        a = blocks[v]
        ext = [PF._card("XTENSION", "IMAGE", "IMAGE extension"), PF._card("BITPIX", -64),
               PF._card("NAXIS", a.ndim)]
        ext += [PF._card("NAXIS%d" % (k + 1), a.shape[a.ndim - 1 - k]) for k in range(a.ndim)]
        ext += [PF._card("PCOUNT", 0), PF._card("GCOUNT", 1)]
        raw += PF._header(ext) + PF._data(a)
    import gzip
    with open(path, "wb") as f:
        f.write(gzip.compress(raw) if path.endswith(".gz") else raw)
    return path


def read_denstemp_fits(path):
    """dict as read_denstemp from a denstemp.fits(.gz) file"""
    from . import particle_fits as PF
    hdus = PF._read_hdus(PF._open(path))
    hdr, grid = hdus[0]
    names = [str(hdr.get("HDU%2d" % (i + 1), "")).strip() for i in range(int(hdr.get("NHDU", len(hdus) - 1)))]
    out = dict(r_av=grid[0, 0, :] * M.AU, theta_av=grid[1, :, 0], ngrains=int(hdr["NGRAINS"]))
    key = {"DENS": "dens", "TEMP": "T", "GASDENS": "gasdens", "DENS0": "dens0"}
    for name, (h, a) in zip(names, hdus[1:]):
        if name == "COMP":
            out["comp"] = a[0].transpose(2, 1, 0)
        elif name in key:
            out[key[name]] = a.T
    return out


def mcspec_name(j, nangle=30):
    """file name of inclination bin j = 1..nangle (MCRadiation.f:741-743):
    the bin's angle written as one digit of tens and f3.1 of the rest"""
    angle = 180.0 * math.acos((j - 0.5) / nangle) / math.pi
    tens = int(angle / 10.0)
    return "MCSpec%d%3.1f.dat" % (tens, angle - 10.0 * tens)


def write_mcspec(outdir, model, result, distance_pc=100.0, nangle=30):
    """MCSpec<angle>.dat for the nangle inclination bins and MCSpec.dat.

    Columns (MCRadiation.f:752-753): wavelength [micron], flux density
    [Jy] spec/d^2, its Monte Carlo error spec/sqrt(ispec)/d^2, the scattered
    part scatspec/d^2, a scattered-packet count, and the stellar flux
    1e23 Fstar/d^2; no interstellar extinction.  The library counts
    escaping packets per bin (ispec) but not the scattered ones separately,
    so the fifth column is 0.  It does not fill the narrow observer bin 0
    (MCRadiation.f:610-612), so MCSpec.dat holds zeros."""
    os.makedirs(outdir, exist_ok=True)
    d2 = (distance_pc * PARSEC) ** 2
    spec = np.asarray(result["spec"], float).reshape(model.nlam, nangle + 1)
    scat = np.asarray(result["scatspec"], float).reshape(model.nlam, nangle + 1)
    ispec = np.asarray(result["ispec"]).reshape(model.nlam, nangle + 1)
    names = []
    for j in range(1, nangle + 1):
        name = mcspec_name(j, nangle)
        names.append(name)
        with open(os.path.join(outdir, name), "w") as f:
            for i in range(model.nlam):
                n = int(ispec[i, j])
                dspec = spec[i, j] / math.sqrt(n) if n > 0 else 0.0
                f.write("%s%s%s%s %d%s\n" % (_num(model.lam[i]), _num(spec[i, j] / d2), _num(dspec / d2),
                                            _num(scat[i, j] / d2), 0, _num(1e23 * model.Fstar[i] / d2)))
    with open(os.path.join(outdir, "MCSpec.dat"), "w") as f:
        for i in range(model.nlam):
            f.write("%s%s\n" % (_num(model.lam[i]), _num(spec[i, 0] / d2)))
    return names


def spectrum_wavelengths(lam, lam1, lam2, nlam=-1, lamfile=None):
    """The wavelengths of a spectrum observation (Telescope.f:40-71): from
    lamfile when given (one per line); else with nlam < 0, lam1, the model's
    wavelengths strictly between lam1 and lam2, and lam2; else nlam
    log-spaced points (at most the model's count)."""
    lam = np.asarray(lam, float)
    if lamfile:
        out = []
        with open(lamfile) as f:
            for line in f:
                try:
                    out.append(float(line.split()[0].replace("d", "e").replace("D", "E")))
                except (ValueError, IndexError):
                    continue
        return np.array(out)
    if nlam < 0:
        return np.concatenate([[lam1], lam[(lam > lam1) & (lam < lam2)], [lam2]])
    n = min(int(nlam), lam.size)
    if n == 1:
        return np.array([lam1])
    return 10.0 ** (math.log10(lam1) + math.log10(lam2 / lam1) * np.arange(n) / (n - 1))


def read_observations(path, lam, incangle=45.0, rout=None, vis_norm_fov=True):
    """The observations of an MCMax observation file (Telescope.f:583-1100):
    keywords before the first type= line set the defaults, each type= line
    starts an observation whose own keywords follow.  Returns a list of
    dicts with kind, inc [deg], lam1, lam2, nlam, lamfile, nphi, nrad, flag,
    npix, nint, fov (list, AU or arcsec), scaletype, the VISIBILITY
    baselines b [m] and theta [deg] (default one of 100 m at 0), d (the
    telescope diameter, m), the scattered-light packets nphot and nphotstar
    and the exit rays nexits (and the other keywords as given, lower-case).
    Defaults: inc from the deck's incangle, lam1/lam2 the model's range,
    nphi 45, nrad 2, npix 500, nint 1000, fov twice the grid's outer radius
    `rout`, scaletype 1, nphot 1000, nphotstar 1000, nexits 5
    (Telescope.f:602-619), and vis_norm_fov from the input deck's
    (Telescope.f:657), which the file can set for all observations or one
    (Telescope.f:1023, 1176).  An IMAGE observation's lam1 is
    the default-level `lam`, else the middle of the wavelength range
    (Telescope.f:591,710-712); a `lam` among an observation's own keywords
    sets its lam1."""
    lam = np.asarray(lam, float)
    default = dict(inc=float(incangle), lam1=float(lam[0]), lam2=float(lam[-1]), nlam=-1, lamfile="", nphi=45,
                   nrad=2, flag="", npix=500, nint=1000, fov=[] if rout is None else [2.0 * float(rout)],
                   scaletype=1, b=[100.0], theta=[0.0], d=-1.0, nphot=1000, nphotstar=1000, nexits=5,
                   vis_norm_fov=bool(vis_norm_fov))
    deflam = (float(lam[0]) + float(lam[-1])) / 2.0
    obs, cur = [], default
    base = os.path.dirname(os.path.abspath(path))
    num = lambda v: float(v.replace("d", "e").replace("D", "E"))
    with open(path) as f:
        for line in f:
            t = line.strip()
            if not t or t.startswith("*") or "=" not in t:
                continue
            key, val = t.split("=", 1)
            key = key.strip().lower()
            val = val.strip()
            if val[:1] in ("'", '"'):
                val = val[1:-1] if len(val) > 1 and val[-1] == val[0] else val[1:]
            if key == "type":
                cur = dict(default, kind=val.upper(), fov=list(default["fov"]), b=list(default["b"]),
                           theta=list(default["theta"]))
                if cur["kind"] in ("IMAGE", "BASEVIS"):
                    cur["lam1"] = deflam
                obs.append(cur)
                continue
            if key in ("nphi", "nrad", "nlam", "npix", "nint", "scaletype", "nphot", "nphotstar", "nexits"):
                cur[key] = int(num(val))
            elif cur is not default and cur["kind"] == "BASEVIS" and key[:3] == "lam" and key[3:].isdigit():
                # lamN: the wavelengths of a BASEVIS observation (Telescope.f:1129-1133)
                i = int(key[3:])
                lams = cur.setdefault("lams", [])
                while len(lams) < i:
                    lams.append(0.0)
                lams[i - 1] = num(val)
                if i == 1:
                    cur["lam1"] = lams[0]
            elif key == "lam" and cur is default:
                deflam = num(val)
            elif key in ("inc", "lam1", "lam2", "lam"):
                cur["lam1" if key == "lam" else key] = num(val)
            elif cur is not default and cur["kind"] in ("VISIBILITY", "BASEVIS") and (
                    (key[:4] == "base" and key[4:].isdigit()) or (key[:5] == "angle" and key[5:].isdigit())):
                # baseN [m] and angleN [deg] of the baselines (Telescope.f:1067-1127)
                i = int(key[4:] if key[:4] == "base" else key[5:])
                while len(cur["b"]) < i:
                    cur["b"].append(0.0)
                    cur["theta"].append(0.0)
                cur["b" if key[:4] == "base" else "theta"][i - 1] = num(val)
            elif key == "d":
                cur["d"] = num(val)
            elif key == "vis_norm_fov":
                cur[key] = val.strip().strip(".").lower() in ("true", "t")
            elif key[:3] == "fov":
                i = int(key[3:]) if len(key) > 3 else 1
                while len(cur["fov"]) < i:
                    cur["fov"].append(None)
                cur["fov"][i - 1] = num(val)
            elif key == "lamfile":
                cur[key] = val if os.path.isabs(val) else os.path.join(base, val)
            else:
                cur[key] = val
    for ob in obs:
        ob["fov"] = [x for x in ob["fov"] if x is not None]
    return obs


def _arrinterpol_log(x, xarr, yarr):
    """arrinterpol(..., log=1) as Subroutines.f:2506-2535 evaluates it: at
    or beyond either end it returns the end's abscissa, and inside, its scan
    keeps the last interval, so the value is the power law through the
    grid's last two points"""
    n = len(xarr)
    if x <= xarr[0]:
        return float(xarr[0])
    if x >= xarr[n - 1]:
        return float(xarr[n - 1])
    x1, x2, y1, y2 = xarr[n - 2], xarr[n - 1], yarr[n - 2], yarr[n - 1]
    p = math.log10(y2 / y1) / math.log10(x2 / x1)
    return y1 * (x / x1) ** p


def spectrum_name(angle_deg, flag=""):
    """spectrum<angle><flag>.dat: the angle as one digit of tens and f3.1
    of the rest (Telescope.f:143-144)"""
    tens = int(angle_deg / 10.0)
    return "spectrum%d%3.1f%s.dat" % (tens, angle_deg - 10.0 * tens, flag)


def write_spectrum(outdir, angle_deg, lam_obs, flux, lam, Fstar, distance_pc=100.0, scatflux=None, flag="",
                   star_column="reference", polarised=False):
    """spectrum<angle>.dat of a ray-traced spectrum (Telescope.f:140-160):
    wavelength [micron], flux [Jy], its scattered part [Jy], the star [Jy],
    with no interstellar extinction (Av = 0); with polarised (scattering
    with the full Mueller matrix) a fifth column, the Q flux [Jy], zero
    here: the traced flux carries no polarisation.  star_column "reference"
    writes the star as the reference's arrinterpol gives it (see
    _arrinterpol_log); "interpolated" writes the log-log interpolation of
    the stellar spectrum instead.  Returns the path."""
    os.makedirs(outdir, exist_ok=True)
    d2 = (distance_pc * PARSEC) ** 2
    lam = np.asarray(lam, float)
    Fstar = np.asarray(Fstar, float)
    scat = np.zeros(len(lam_obs)) if scatflux is None else np.asarray(scatflux, float)
    path = os.path.join(outdir, spectrum_name(angle_deg, flag))
    with open(path, "w") as f:
        for j, l0 in enumerate(lam_obs):
            if star_column == "reference":
                fs = _arrinterpol_log(l0, lam, Fstar)
            else:
                fs = float(np.exp(np.interp(np.log(l0), np.log(lam), np.log(Fstar))))
            f.write("%s%s%s%s%s\n" % (_num(l0), _num(1e23 * flux[j] / d2), _num(1e23 * scat[j] / d2),
                                      _num(1e23 * fs / d2), _num(0.0) if polarised else ""))
    return path


def _fortran_f(x, w, d):
    """Fortran fw.d: asterisks when the number does not fit"""
    t = "%*.*f" % (w, d, x)
    return "*" * w if len(t) > w else t


def _fortran_i1(n):
    return str(n) if 0 <= n <= 9 else "*"


def _angle_tag(angle_rad):
    """i1,f3.1 of the inclination in degrees as FITSImage forms it from the
    angle in radians, tenths of 9.95 and up carried (TraceMono.f:3475-3480)"""
    a = (180.0 * angle_rad) / math.pi
    i10 = int(a / 10.0)
    i1 = a - 10.0 * i10
    if i1 >= 9.95:
        i1 = i1 - 9.95
        i10 = i10 + 1
    return _fortran_i1(i10) + _fortran_f(i1, 3, 1)


def _lam_tag(lam0):
    """4(i1),f4.2 of the wavelength (TraceMono.f:3482-3486)"""
    a = int(lam0 / 10000.0)
    b = int((lam0 - 10000.0 * a) / 1000.0)
    c = int((lam0 - 1000.0 * b - 10000.0 * a) / 100.0)
    d = int((lam0 - 100.0 * c - 1000.0 * b - 10000.0 * a) / 10.0)
    e = lam0 - 10.0 * d - 100.0 * c - 1000.0 * b - 10000.0 * a
    return "".join(_fortran_i1(v) for v in (a, b, c, d)) + _fortran_f(e, 4, 2)


def _fov_tag(Rmax):
    """4(i1),f3.1 of the field of view 2 Rmax with the carries of
    TraceMono.f:3488-3509"""
    r = 2.0 * Rmax
    a = int(r / 10000.0)
    b = int((r - 10000.0 * a) / 1000.0)
    c = int((r - 1000.0 * b - 10000.0 * a) / 100.0)
    d = int((r - 100.0 * c - 1000.0 * b - 10000.0 * a) / 10.0)
    e = r - 10.0 * d - 100.0 * c - 1000.0 * b - 10000.0 * a
    if e >= 9.95:
        d, e = d + 1, e - 9.95
    if d >= 10:
        c, d = c + 1, d - 10
    if c >= 10:
        b, c = b + 1, c - 10
    if b >= 10:
        a, b = a + 1, b - 10
    return "".join(_fortran_i1(v) for v in (a, b, c, d)) + _fortran_f(e, 3, 1)


def image_name(kind, angle_rad, lam0, Rmax, flag=""):
    """Image<kind>_i<angle>_l<lam>_fov<2 Rmax><flag>.fits (TraceMono.f:3511-3512)"""
    return "Image%s_i%s_l%s_fov%s%s.fits" % (kind, _angle_tag(angle_rad), _lam_tag(lam0), _fov_tag(Rmax), flag)


def rimage_name(angle_rad, lam0, flag=""):
    """RImage_i<angle>_l<lam><flag>.dat (TraceMono.f:3399-3400)"""
    return "RImage_i%s_l%s%s.dat" % (_angle_tag(angle_rad), _lam_tag(lam0), flag)


def write_image_fits(path, im, Rmax, rscale=1.0, scaletype=1):
    """an image as FITSImage writes it (TraceMono.f:3446-3570): a primary
    npix x npix BITPIX -64 image whose data stream is im[ix-1, iy-1] with iy
    running fastest, then CTYPE1/2, CRPIX1/2 = 0.5, CRVAL1/2 = -Rmax rscale
    (the corner), CDELT1/2 = 2 Rmax rscale / npix; AU for scaletype 1,
    arcsec for 2.  Returns the path."""
    from . import particle_fits as PF
    im = np.asarray(im, float)
    n = im.shape[0]
    unit = "AU" if scaletype == 1 else "arcsec"
    cards = [PF._card("SIMPLE", True, "file does conform to FITS standard"),
             PF._card("BITPIX", -64, "number of bits per data pixel"), PF._card("NAXIS", 2, "number of data axes"),
             PF._card("NAXIS1", n, "length of data axis 1"), PF._card("NAXIS2", n, "length of data axis 2"),
             PF._card("EXTEND", True, "FITS dataset may contain extensions")]
    if scaletype in (1, 2):
        cards += [PF._card("CTYPE1", "X [%s]" % unit, "X-coordinate"),
                  PF._card("CTYPE2", "Y [%s]" % unit, "Y-coordinate")]
    corner = -Rmax * rscale
    pix = 2.0 * Rmax * rscale / float(np.float32(n))
    cards += [PF._card("CRPIX1", 0.5, "reference pixel: the image corner", 10),
              PF._card("CRPIX2", 0.5, "reference pixel: the image corner", 10),
              PF._card("CRVAL1", corner, "coordinate of the corner", 10),
              PF._card("CRVAL2", corner, "coordinate of the corner", 10)]
    if scaletype in (1, 2):
        cards += [PF._card("CDELT1", pix, "pixel size (%s)" % unit, 10),
                  PF._card("CDELT2", pix, "pixel size (%s)" % unit, 10)]
    if os.path.exists(path):
        os.remove(path)
    with open(path, "wb") as f:
        f.write(PF._header(cards) + PF._data(im))
    return path


def read_image_fits(path):
    """(header dict, image [ix-1, iy-1]) of an image written by write_image_fits"""
    from . import particle_fits as PF
    hdr, a = PF._read_hdus(PF._open(path))[0]
    return hdr, np.asarray(a, float)


def write_rimage(path, R, rphi, rscale, zscale, distance_cm, fov_au, npixel, polarised=False):
    """the radial profile file of RImage (TraceMono.f:3375-3443): per image
    radius R[i] (i < nr-1) the radius x rscale, the flux inside the ring's
    outer edge [Jy at the distance] (the running trapezoid sum over the
    rings) and the intensity at angle column nphi/2 x scaling, scaling =
    zscale 1e23 / d^2 fov^2 AU^2 / npix^2; then the same for the last
    radius with the total flux.  With polarisation (full Mueller matrix) the
    Q, U and polarised columns are written as zeros: the image carries no
    polarisation.  Returns the path."""
    R = np.asarray(R, float)
    rphi = np.asarray(rphi, float)
    nr, nphi = rphi.shape
    d2 = distance_cm ** 2
    scaling = (zscale * 1e23 / d2) * (fov_au ** 2 * M.AU ** 2) / float(npixel ** 2)
    kc = max(nphi // 2, 1) - 1
    flux = 0.0
    lines = []
    for i in range(nr - 1):
        w1 = 2.0 * math.pi * abs(R[i]) * M.AU ** 2 / float(np.float32(nphi))
        w2 = 2.0 * math.pi * abs(R[i + 1]) * M.AU ** 2 / float(np.float32(nphi))
        for k in range(nphi):
            flux = flux + (R[i + 1] - R[i]) * (w1 * rphi[i, k] + w2 * rphi[i + 1, k]) / 2.0
        row = [R[i] * rscale, flux * 1e23 / d2, scaling * rphi[i, kc]]
        if polarised:
            row += [0.0, 0.0, 0.0]
        lines.append(row)
    row = [R[nr - 1] * rscale, flux * 1e23 / d2, scaling * rphi[nr - 1, kc]]
    if polarised:
        row += [0.0]
    lines.append(row)
    with open(path, "w") as f:
        for row in lines:
            f.write("".join(_num(x) for x in row) + "\n")
    return path


def image_phi(nphi):
    """the angles of the image columns, 1e-5 + pi (k - 1/2) / nphi with the
    single-precision k - 0.5 of TraceMono.f:2237"""
    k = np.arange(1, nphi + 1, dtype=np.float32)
    return 1e-5 + (math.pi * (k - np.float32(0.5)).astype(float)) / float(np.float32(nphi))


def _vis_half(R, rphi, phi_c, nphi, theta, k, Rsigma, vis_norm_fov, sign):
    """one half of the image plane (+phi or -phi) of Visibility.f:36-150:
    per ring segment and angle column the closed-form Fourier integral of
    an intensity linear in r and constant in phi; returns (cV, Ftot)"""
    r1 = R[:-1, None]
    r2 = R[1:, None]
    I1 = rphi[:-1]
    I2 = rphi[1:]
    Rs2 = np.float64(Rsigma) ** 2 if Rsigma < 1e150 else np.inf   # 1e200^2 is infinite, as in the reference
    t1 = I1 * np.exp(-r1 ** 2 / (2.0 * Rs2))
    t2 = I2 * np.exp(-r2 ** 2 / (2.0 * Rs2))
    n1, n2 = (t1, t2) if vis_norm_fov else (I1, I2)
    half = 0.5 * math.pi / float(np.float32(nphi))
    phi1 = sign * phi_c[None, :] - half
    phi2 = sign * phi_c[None, :] + half
    c1 = np.cos(theta + phi1)
    b1 = np.sin((phi1 + phi2) / 2.0 + theta)
    a1 = c1 + 2.0 * np.sin((phi1 - phi2) / 2.0) * b1
    cI = 1j
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        far = (np.abs(k * r2) > 0.1) | (np.abs(k * r1) > 0.1)
        ea1, ea2 = np.exp(-cI * k * r1 * a1), np.exp(-cI * k * r2 * a1)
        ec1, ec2 = np.exp(-cI * k * r1 * c1), np.exp(-cI * k * r2 * c1)
        J1f = (-1.0 / (k ** 2 * b1)) * ((ea2 - ea1) / a1 - (ec2 - ec1) / c1)
        J2f = (-1.0 / (cI * k ** 3 * b1)) * ((1.0 + cI * k * a1 * r2) * ea2 / a1 ** 2 - (1.0 + cI * k * c1 * r2) * ec2 / c1 ** 2
                                             - (1.0 + cI * k * a1 * r1) * ea1 / a1 ** 2 + (1.0 + cI * k * c1 * r1) * ec1 / c1 ** 2)
        J1s = ((r2 ** 2 - r1 ** 2) * (a1 - c1) / (2.0 * b1) - (cI * (r2 ** 3 - r1 ** 3) * (a1 ** 2 - c1 ** 2) / (6.0 * b1)) * k
               - ((r2 ** 4 - r1 ** 4) * (a1 ** 3 - c1 ** 3) / (24.0 * b1)) * k ** 2
               + (cI * (r2 ** 5 - r1 ** 5) * (a1 ** 4 - c1 ** 4) / (120.0 * b1)) * k ** 3
               + ((r2 ** 6 - r1 ** 6) * (a1 ** 5 - c1 ** 5) / (720.0 * b1)) * k ** 4
               - (cI * (r2 ** 7 - r1 ** 7) * (a1 ** 6 - c1 ** 6) / (5040.0 * b1)) * k ** 5
               - ((r2 ** 8 - r1 ** 8) * (a1 ** 7 - c1 ** 7) / (40320.0 * b1)) * k ** 6)
        J2s = ((r2 ** 3 - r1 ** 3) * (a1 - c1) / (3.0 * b1) - (cI * (r2 ** 4 - r1 ** 4) * (a1 ** 2 - c1 ** 2) / (8.0 * b1)) * k
               - ((r2 ** 5 - r1 ** 5) * (a1 ** 3 - c1 ** 3) / (30.0 * b1)) * k ** 2
               + (cI * (r2 ** 6 - r1 ** 6) * (a1 ** 4 - c1 ** 4) / (144.0 * b1)) * k ** 3
               + ((r2 ** 7 - r1 ** 7) * (a1 ** 5 - c1 ** 5) / (840.0 * b1)) * k ** 4
               - (cI * (r2 ** 8 - r1 ** 8) * (a1 ** 6 - c1 ** 6) / (5760.0 * b1)) * k ** 5
               - ((r2 ** 9 - r1 ** 9) * (a1 ** 7 - c1 ** 7) / (45360.0 * b1)) * k ** 6)
        J1 = np.where(far, J1f, J1s)
        J2 = np.where(far, J2f, J2s)
        dr = r2 - r1
        cV = t1 * ((1.0 + r1 / dr) * J1 - J2 / dr) + t2 * (J2 - r1 * J1) / dr
        K1 = (r2 ** 2 - r1 ** 2) * (a1 - c1) / (2.0 * b1)
        K2 = (r2 ** 3 - r1 ** 3) * (a1 - c1) / (3.0 * b1)
        F = -(n1 * ((1.0 + r1 / dr) * K1 - K2 / dr)) - n2 * (K2 - r1 * K1) / dr
    keep = np.broadcast_to(r1 != r2, cV.shape)
    return np.sum(np.where(keep, cV, 0.0)), np.sum(np.where(keep, F, 0.0))


def visibility(R, rphi, b, theta_b, lam0, distance_cm, diam=-1.0, pa=0.0, vis_norm_fov=True):
    """Visibility amplitude and phase of the ray image at one baseline
    (Visibility.f:1-163): R the image radii [AU], rphi (nr, nphi) their
    intensities, b the baseline [m], theta_b its angle [rad], lam0
    [micron], the distance [cm], diam the telescope diameter [m] (a
    Gaussian taper of 0.42 lam/D when positive), pa the position angle
    [deg].  The image is linear in r between image radii and constant over
    each angle column, mirrored to -phi; the integrals are the reference's
    closed forms (its series below k r = 0.1), evaluated in complex128
    where the reference uses quad-precision complex, and summed with NumPy
    rather than in the reference's loop order.  Returns (V, phase)."""
    R = np.asarray(R, float)
    rphi = np.asarray(rphi, float)
    nphi = rphi.shape[1]
    dpc = distance_cm / PARSEC
    if abs(theta_b) < math.pi / 360.0:
        theta = math.pi / 2.0 - math.pi / 360.0 + pa * math.pi / 180.0
    else:
        theta = math.pi / 2.0 - theta_b + pa * math.pi / 180.0
    k = 2.0 * math.pi * b / (lam0 * dpc)
    k = k * 1e6 * math.pi / (180.0 * 3600.0)
    if diam > 0.0:
        Rsigma = float(np.float32(0.42)) * lam0 * 1e-6 / diam * 180.0 / math.pi * 3600.0 * dpc
    else:
        Rsigma = 1e200
    phi_c = image_phi(nphi)
    cV1, F1 = _vis_half(R, rphi, phi_c, nphi, theta, k, Rsigma, vis_norm_fov, 1.0)
    cV2, F2 = _vis_half(R, rphi, phi_c, nphi, theta, k, Rsigma, vis_norm_fov, -1.0)
    z = (cV1 + cV2) / (F1 + F2)
    return float(abs(z)), float(math.atan2(z.imag, z.real))


def write_visibility(outdir, angle_deg, lam_obs, spec_jy, b, theta_deg, V, phase, flag=""):
    """visibility<angle><flag>.dat (Telescope.f:214-240): the header naming
    the columns, then per wavelength the wavelength, the flux [Jy], the
    visibilities of each baseline and their phases.  Returns the path."""
    os.makedirs(outdir, exist_ok=True)
    tens = int(angle_deg / 10.0)
    path = os.path.join(outdir, "visibility%d%3.1f%s.dat" % (tens, angle_deg - 10.0 * tens, flag))
    nb = len(b)
    with open(path, "w") as f:
        f.write("# column   1: wavelength\n# column   2: full disk\n")
        for kk in range(nb):
            f.write("# column %3d and %3d: vis and phase for: baseline %10.3f, angle %10.3f\n"
                    % (kk + 3, kk + 3 + nb, b[kk], theta_deg[kk]))
        for j, l0 in enumerate(lam_obs):
            f.write("".join(_num(x) for x in [l0, spec_jy[j]] + list(V[j]) + list(phase[j])) + "\n")
    return path


def write_basevis(outdir, angle_deg, base, lams, theta_deg, flux_jy, V, phase, flag=""):
    """basevis<angle><flag>.dat (Telescope.f:246-291): the header naming the
    columns, then per baseline [m] the flux of the last wavelength [Jy] and
    the visibilities and phases at each wavelength.  Returns the path."""
    os.makedirs(outdir, exist_ok=True)
    tens = int(angle_deg / 10.0)
    path = os.path.join(outdir, "basevis%d%3.1f%s.dat" % (tens, angle_deg - 10.0 * tens, flag))
    nl = len(lams)
    with open(path, "w") as f:
        f.write("# column   1: baseline\n# column   2: full disk (only last wavelength)\n")
        for j in range(nl):
            f.write("# column %3d and %3d: vis and phase for wavelength %10.3f, angle %10.3f\n"
                    % (j + 3, j + 3 + nl, lams[j], theta_deg[j]))
        for k, b in enumerate(base):
            f.write("".join(_num(x) for x in [b, flux_jy] + [V[j][k] for j in range(nl)]
                            + [phase[j][k] for j in range(nl)]) + "\n")
    return path
