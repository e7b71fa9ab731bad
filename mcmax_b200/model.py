"""Host-side model set-up: the parts of Init.f that build what the packet loop
reads, plus the keyword-deck surface.

    parse_deck            key=value decks, lower-cased keys, '*' comments,
                          quotes stripped, -s overrides (Init.f:462-498)
    readrefind            .lnk refractive-index regridding (readrefindCP,
                          ComputePart.f:1102-1172, log-log interpolation and
                          the dielectric long-wavelength extrapolation)
    wavelength_grid       Init.f:2580-2614 (log grid, nu, dnu)
    spatial_grid          Init.f:2779-2930 (radial log grid with the star cell
                          i = 0, cos-theta edges from the midpoint rule)
    zones_density         Init.f:3054-3139 ('ZONES' density, one or more zones)
    mrn_abundances        MRN.f:21-201 (gsd_MRN mass fractions of size bins)
    grain_bins            Init.f:1323-1420 (computepartNN:ngrains -> log bins)

The radial/theta regridding MCMax applies during its first iterations
(RegridR, RegridTheta) is outside the packet loop and not restated: models
here use the plain log radial grid.
"""
import math
import os
import shlex

import numpy as np

from . import api
from ._ffi import TT, NANG

# Modules.f:4-10 declares these real*8 but writes them as default-real
# (single-precision) literals, so the reference computes with the float
# nearest each decimal value, widened to double
AU = float(np.float32(1.49598e13))
RSUN = float(np.float32(6.9599e10))
MSUN = float(np.float32(1.98892e33))
LSUN = float(np.float32(3.846e33))
CLIGHT_MICRON = 2.9979e14


# ---------------------------------------------------------------- keyword deck
def parse_deck(text, overrides=()):
    """Parse an MCMax input deck.  Returns {key: value-string}; `overrides`
    are 'key=value' strings applied after the file (the -s switches)."""
    out = {}

    def take(line):
        line = line.split("*", 1)[0] if line.lstrip().startswith("*") else line
        if "=" not in line:
            return
        key, val = line.split("=", 1)
        key = key.strip().lower()
        val = val.strip()
        if val[:1] in ("'", '"'):
            q = val[0]
            val = val[1:].split(q, 1)[0]
        else:
            val = val.split()[0] if val.split() else ""
        if key:
            out[key] = val

    for line in text.splitlines():
        if line.strip().startswith("*") or not line.strip():
            continue
        take(line)
    for ov in overrides:
        take(ov)
    return out


def deck_value(d, key, default, cast=float):
    if key not in d:
        return default
    v = d[key]
    if cast is bool:
        return v.strip(".").lower() in ("true", "t", "1", "yes")
    if cast is float:
        return float(v.lower().replace("d", "e"))
    return cast(v)


# ---------------------------------------------------------------- refractive index
def read_lnk(path):
    rows = []
    with open(path) as f:
        for line in f:
            s = line.strip()
            if not s or s[0] in "#*!":
                continue
            parts = s.replace("D", "E").replace("d", "e").split()
            try:
                rows.append([float(x) for x in parts[:3]])
            except ValueError:
                continue
    return np.array(rows)


def readrefind(path_or_table, grid, loglog=False):
    """Regrid (lam, n, k) onto `grid` (ComputePart.f:1102-1172)."""
    tab = read_lnk(path_or_table) if isinstance(path_or_table, str) else np.asarray(path_or_table, float)
    grid = np.asarray(grid, float)
    n = grid.size
    e1 = np.zeros(n)
    e2 = np.zeros(n)
    i = 0
    x0, y01, y02 = tab[0]
    y02 = max(y02, 1e-8)
    while i < n and x0 >= grid[i]:
        e1[i], e2[i] = y01, y02
        i += 1
    for x1, y11, y12 in tab[1:]:
        if i >= n:
            break
        y12 = max(y12, 1e-8)
        while i < n and grid[i] <= x1 and grid[i] > x0:
            e1[i] = 10 ** (math.log10(y11) + math.log10(grid[i] / x1) * math.log10(y01 / y11) / math.log10(x0 / x1))
            e2[i] = 10 ** (math.log10(y12) + math.log10(grid[i] / x1) * math.log10(y02 / y12) / math.log10(x0 / x1))
            i += 1
        x0, y01, y02 = x1, y11, y12
    if i < n:
        if loglog and i >= 2:
            for j in range(i, n):
                r = math.log10(grid[i - 2] / grid[j]) / math.log10(grid[i - 2] / grid[i - 1])
                e1[j] = 10 ** (math.log10(e1[i - 2]) + math.log10(e1[i - 1] / e1[i - 2]) * r)
                e2[j] = 10 ** (math.log10(e2[i - 2]) + math.log10(e2[i - 1] / e2[i - 2]) * r)
        else:
            for j in range(i, n):
                e1[j] = e1[i - 1]
                e2[j] = e2[i - 1] * grid[i - 1] / grid[j]
    return e1, e2


def read_particle_file(path):
    """Particle file of ComputePart's 'FILE' standard (ComputePart.f:65-92):
    ns, nf, then per material a .lnk path line and a 'frac rho' line."""
    lines = []
    with open(path) as f:
        for line in f:
            s = line.strip()
            if s and not s.startswith("*"):
                lines.append(s)
    ns = int(lines[0].split()[0])
    nf = int(lines[1].split()[0])
    mats = []
    k = 2
    base = os.path.dirname(os.path.abspath(path))
    while k + 1 < len(lines):
        name = shlex.split(lines[k])[0]
        if not os.path.isabs(name):
            name = os.path.join(base, name)
        fr, rh = [float(x.replace("d", "e").replace("D", "E")) for x in lines[k + 1].split()[:2]]
        mats.append((name, fr, rh))
        k += 2
    return ns, nf, mats


# ---------------------------------------------------------------- grids
def wavelength_grid(lam1, lam2, nlam):
    i = np.arange(nlam)
    lam = 10.0 ** (math.log10(lam1) + (math.log10(lam2) - math.log10(lam1)) * i / (nlam - 1))
    nu = CLIGHT_MICRON / lam
    return lam, nu


def theta_centres(ntheta):
    """cell-centre angles theta_av (radians, j = 1..ntheta, pole to
    midplane) of the theta grid of Init.f:2779-2890 (no refinement)"""
    nT = ntheta + 1
    th = []
    k = nT // 2
    for j in range(1, k + 1):
        th.append((j - 1) / (k - 1))
        th.append(math.cos(0.5 * math.pi * j / (k + 1)))
    i = len(th)
    if i < nT:
        for j in range(i + 1, nT + 1):
            th.append((j - i + 1) / (nT - i + 1))
    th = sorted(th)[:nT]
    return np.array([math.acos((th[nT - i] + th[nT - i - 1]) / 2.0) for i in range(1, nT)])


def spatial_grid(rstar_cm, rin, rout, nrad, ntheta):
    """Edges R[0..nR] (AU, R[0] = Rstar) and cos-theta edges Theta[0..nTheta-1]
    following Init.f:2779-2890 without refinement (ntspan = ntlev = 0)."""
    nR = nrad + 1
    nT = ntheta + 1
    th = []
    k = nT // 2
    for j in range(1, k + 1):
        th.append((j - 1) / (k - 1))
        th.append(math.cos(0.5 * math.pi * j / (k + 1)))
    i = len(th)
    if i < nT:
        for j in range(i + 1, nT + 1):
            th.append((j - i + 1) / (nT - i + 1))
    th = sorted(th)[:nT]
    theta_av = [math.acos((th[nT - i] + th[nT - i - 1]) / 2.0) for i in range(1, nT)]
    R = np.zeros(nR + 1)
    R[0] = rstar_cm / AU
    ii = np.arange(nR)
    R[1:] = 10.0 ** (math.log10(rin) + (math.log10(rout) - math.log10(rin)) * ii / (nR - 1))
    Theta = np.zeros(nT)
    thet = np.zeros(nT)
    Theta[0] = 1.0
    thet[0] = 0.0
    for i in range(2, nT):
        thet[i - 1] = (theta_av[i - 2] + theta_av[i - 1]) / 2.0
        Theta[i - 1] = math.cos(thet[i - 1])
    Theta[nT - 1] = 0.0
    thet[nT - 1] = math.pi / 2.0
    SinTheta = np.sin(thet)
    return R, Theta, thet, SinTheta


def grid_from_centres(rstar_cm, rin, rout, r_av_cm, theta_av):
    """Edges rebuilt from the cell centres of a density file
    (Init.f:2727-2752 for the radii, Init.f:2876-2889 for theta): R[1] = rin,
    each next edge the mirror of the previous one about the centre in log r
    (or the midpoint of the two centres when that falls outside them),
    R[nR] = rout; theta edges halfway between the centre angles.  Returns
    (R, Theta, thet, SinTheta) as spatial_grid."""
    r_av = np.asarray(r_av_cm, float) / AU
    n = r_av.size
    R = np.zeros(n + 2)
    R[0] = rstar_cm / AU
    R[1] = rin
    for i in range(2, n + 1):
        R[i] = 10.0 ** (2.0 * math.log10(r_av[i - 2]) - math.log10(R[i - 1]))
        if r_av[i - 1] < R[i] or r_av[i - 2] > R[i]:
            R[i] = (r_av[i - 2] + r_av[i - 1]) / 2.0
    R[n + 1] = rout
    R[1:n + 1] = np.sort(R[1:n + 1])
    ta = np.asarray(theta_av, float)
    nT = ta.size + 1
    Theta = np.zeros(nT)
    thet = np.zeros(nT)
    Theta[0] = 1.0
    for i in range(2, nT):
        thet[i - 1] = (ta[i - 2] + ta[i - 1]) / 2.0
        Theta[i - 1] = math.cos((ta[i - 2] + ta[i - 1]) / 2.0)
    Theta[nT - 1] = 0.0
    thet[nT - 1] = math.pi / 2.0
    return R, Theta, thet, np.sin(thet)


def cell_volumes(R, Theta):
    R = np.asarray(R, float)
    Theta = np.asarray(Theta, float)
    return (4.0 * math.pi / 3.0) * (R[1:, None] ** 3 - R[:-1, None] ** 3) * (Theta[None, :-1] - Theta[None, 1:]) \
        * AU ** 3


def zones_density(R, Theta, thet, zones):
    """'ZONES' dust density (Init.f:3054-3139).  zones: list of dicts with
    rin, rout, mdust (Msun), denspow, sh, rsh, shpow.  Each cell averages the
    zone profile over 10 sub-angles; cell i = 0 gets 1e-60
    (Init.f:2932-2938)."""
    nR = R.size - 1
    nc = Theta.size - 1
    V = cell_volumes(R, Theta)
    R_av = AU * 10.0 ** ((np.log10(R[:-1]) + np.log10(R[1:])) / 2.0)
    thet = np.asarray(thet, float)
    dens = np.full((nR, nc), 1e-60)
    total = np.zeros((nR, nc))
    for z in zones:
        inside = (R_av >= z["rin"] * AU) & (R_av <= z["rout"] * AU)
        inside[0] = False
        acc = np.zeros((nR, nc))
        for jj in range(1, 11):
            theta = thet[:-1] + (thet[1:] - thet[:-1]) * jj / 11.0
            r = R_av[:, None] * np.sin(theta)[None, :] / AU
            zz = R_av[:, None] * np.cos(theta)[None, :] / AU
            hr = z["sh"] * (r / z["rsh"]) ** z["shpow"]
            f1 = r ** (-z["denspow"])
            f2 = np.exp(-(zz / hr) ** 2)
            acc = acc + f1 * f2 / hr / 10.0
        zd = np.where(inside[:, None], acc, 0.0)
        tot = (zd * V).sum()
        zd *= z["mdust"] * MSUN / tot
        total += zd
    dens[1:] = 1e-60 + total[1:]
    return dens, V

ANALYTIC_DENSITIES = ("PASCUCCI", "MIN", "PARAMETERIZED", "PINTE", "SHELL", "WEDGE", "MASSLOSS", "INFALL",
                      "MEIXNER")
# radial power laws whose vertical structure the reference builds from the
# optically thin temperatures before the first pass (Init.f:3924-3960)
THIN_START_DENSITIES = ("POW", "DOUBLEPOW", "SIMILARITY", "DOUBLEPOWSIM", "SURFFILE")


def regridlog(path, grid):
    """A two-column table (x, y) on the grid as regridlog reads it
    (Subroutines.f:82-123): grid points up to the first x take its y,
    points inside the table the log-log interpolation of their interval
    (an entry y <= 0 read as 1e-50 of the one before), points beyond it
    the last value times grid(last)/grid (1/x); values that are still <= 0
    become 1e-60 of the last entry read.  Lines before the first readable
    pair are skipped."""
    grid = np.asarray(grid, float)
    n = grid.size
    pairs = []
    with open(path) as f:
        for line in f:
            t = line.replace("d", "e").replace("D", "E").split()
            try:
                pairs.append((float(t[0]), float(t[1])))
            except (IndexError, ValueError):
                if pairs:
                    raise ValueError("%s: unreadable line %r" % (path, line))
    if not pairs:
        raise ValueError("%s: no (x, y) pairs" % path)
    y = np.zeros(n)
    x0, y0 = pairs[0]
    i = 0
    while i < n and x0 >= grid[i]:
        y[i] = y0
        i += 1
    for x1, y1 in pairs[1:]:
        if i >= n:
            break
        if y1 <= 0.0:
            y1 = y0 * 1e-50
        while i < n and x0 < grid[i] <= x1:
            y[i] = 10.0 ** (math.log10(y1) + math.log10(grid[i] / x1) * math.log10(y0 / y1) / math.log10(x0 / x1))
            i += 1
        x0, y0 = x1, y1
    if i == 0:
        raise ValueError("%s: the table starts beyond the grid" % path)
    for j in range(i, n):
        y[j] = y[i - 1] * grid[i - 1] / grid[j]
    return np.where(y <= 0.0, y0 * 1e-60, y)


def surface_density(R, Theta, path, gaspath=None, gas2dust=100.0, mtot=None):
    """'SURFFILE' densities (Init.f:2966-3003): the file's surface density
    regridded on the cell centres (regridlog), spread evenly over each
    ring, dens = Sigma (R_i+1^2 - R_i^2) / V in the reference's mixed units
    (radii in AU, volumes in cm^3), then scaled to mtot [g] when mdust was
    given, else kept (Init.f:3242-3264).  gaspath: the gas surface density,
    gasdens = Sigma_gas pi (R_i+1^2 - R_i^2) AU^2 / V / (nTheta - 1) /
    gas2dust, not scaled.  Returns (dens, V, gasdens or None)."""
    R = np.asarray(R, float)
    nR, nc = R.size - 1, np.asarray(Theta).size - 1
    V = cell_volumes(R, Theta)
    R_av = 10.0 ** ((np.log10(R[:-1]) + np.log10(R[1:])) / 2.0)
    ring = (R[2:] ** 2 - R[1:-1] ** 2)[:, None]
    dens = np.full((nR, nc), 1e-60)
    dens[1:] = regridlog(path, R_av[1:])[:, None] * ring / V[1:]
    mass = float((dens[1:] * V[1:]).sum())
    dens[1:] = dens[1:] * ((mass if mtot is None else mtot) / mass)
    gas = None
    if gaspath:
        gas = np.full((nR, nc), 1e-60)
        gas[1:] = regridlog(gaspath, R_av[1:])[:, None] * math.pi * ring * AU ** 2 / V[1:] / float(
            np.float32(nc)) / gas2dust
    return np.maximum(dens, 1e-60), V, gas


def analytic_density(denstype, R, Theta, thet, p, lam=None, kext=None):
    """The closed-form dust densities of Init.f:3142-3240 that need no
    initial structure iteration: PASCUCCI (the radiative-transfer benchmark
    disk, scaled to the midplane optical depth tau550 at 0.55 micron,
    Init.f:3992-4026), MIN and PINTE (Gaussian vertical profile of scale
    height sh1AU r^shpow; PINTE cut at r = Rexp), PARAMETERIZED (the same,
    averaged over 10 sub-angles), SHELL ((AU/R)^denspow) and WEDGE (the
    cells within wedgeopen degrees of the midplane, 10 sub-angles), MASSLOSS
    (a wind Mdot / (gas2dust 4 pi R^2 v(R)), v = vexp2 (1 - (1 - (vexp1 /
    vexp2)^(1/bexp)) Rstar / R)^bexp), INFALL (rotating infall of
    Minfall onto radius rexp around Mstar) and MEIXNER (meixa..meixf,
    meixrsw, meixrin, timeshift).  r and z
    are taken at the cell centre (R_av, theta_av); cell i = 0 is empty.
    Also the radial power laws of THIN_START_DENSITIES (POW, DOUBLEPOW,
    SIMILARITY, DOUBLEPOWSIM, with denspow2, rpow2, rpow3, rexp,
    gamma_exp), whose vertical structure the caller then builds
    (structure.thin_start).

    p: dict of the deck's rin, rout [AU], denspow, shpow, sh1au, rexp,
    tau550, wedgeopen, and mtot [g] with mdustscale (mdust given).  lam,
    kext (ngrains, nlam) are needed for PASCUCCI: its tau550 uses the sum
    of the grains' Kext at 0.55 micron, unweighted, as the reference forms
    it.  Then the mass normalisation of Init.f:3242-3264: the densities are
    scaled to mtot when mdust was given (never for PASCUCCI), else kept.
    Densities below 1e-60 are raised to 1e-60, the floor the 'ZONES' cells
    start from.  Returns (dens (nR, ncells per ring), V)."""
    nR = R.size - 1
    nc = Theta.size - 1
    V = cell_volumes(R, Theta)
    R_av = AU * 10.0 ** ((np.log10(R[:-1]) + np.log10(R[1:])) / 2.0)
    Theta = np.asarray(Theta, float)
    thet = np.asarray(thet, float)
    theta_av = np.arccos((Theta[:-1] + Theta[1:]) / 2.0)
    r = R_av[:, None] * np.sin(theta_av)[None, :] / AU
    z = R_av[:, None] * np.cos(theta_av)[None, :] / AU
    rin, rout = p["rin"], p["rout"]
    mtot = p["mtot"]
    mdustscale = p["mdustscale"]
    with np.errstate(over="ignore", under="ignore", divide="ignore"):
        if denstype == "PASCUCCI":
            # Init.f:3992-4026: the tau550 form replaces the mass-scaled one
            l55 = float(np.float32(0.55))
            lam = np.asarray(lam, float)
            il1, w1, w2 = 0, 1.0, 0.0
            for i in range(lam.size - 1):
                if lam[i] <= l55 <= lam[i + 1]:
                    il1 = i
                    w1 = (lam[i + 1] - l55) / (lam[i + 1] - lam[i])
                    w2 = (l55 - lam[i]) / (lam[i + 1] - lam[i])
            kext = np.atleast_2d(np.asarray(kext, float))
            k550 = 0.0
            for row in kext:
                k550 = k550 + row[il1] * w1 + row[il1 + 1] * w2
            rd, zd = rout / 2.0, rout / 8.0
            scale = p["tau550"] / (rd * math.log(rout / rin) * k550)
            hr = zd * (r / rd) ** 1.125
            dens = (r / rd) ** (-1.0) * np.exp(-(math.pi / 4.0) * (z / hr) ** 2) * scale / AU
            mdustscale = False
        elif denstype in ("MIN", "PINTE"):
            hr = p["sh1au"] * r ** p["shpow"]
            scale = mtot / (AU ** 3 * 2.0 * math.pi * p["sh1au"] * math.sqrt(math.pi) * (rout - rin))
            dens = scale * r ** (-p["denspow"]) * np.exp(-(z / hr) ** 2) * r ** (-p["shpow"])
            if denstype == "PINTE":
                dens = np.where(r < p["rexp"], dens, 1e-60)
        elif denstype == "PARAMETERIZED":
            scale = mtot / (AU ** 3 * 2.0 * math.pi * p["sh1au"] * math.sqrt(math.pi) * (rout - rin))
            dens = np.zeros((nR, nc))
            for jj in range(1, 11):
                theta = thet[:-1] + (thet[1:] - thet[:-1]) * jj / 11.0
                rr = R_av[:, None] * np.sin(theta)[None, :] / AU
                zz = R_av[:, None] * np.cos(theta)[None, :] / AU
                hr = p["sh1au"] * rr ** p["shpow"]
                dens = dens + scale * rr ** (-p["denspow"]) * np.exp(-(zz / hr) ** 2) / hr / 10.0
        elif denstype == "SHELL":
            dens = np.broadcast_to(((AU / R_av) ** p["denspow"])[:, None], (nR, nc)).copy()
        elif denstype == "MASSLOSS":
            # a stationary wind with a beta velocity law; the 1. literals
            # are exact in single precision
            v2, v1 = p["vexp2"], p["vexp1"]
            vexp = v2 * (1.0 - (1.0 - (v1 / v2) ** (1.0 / p["bexp"])) * p["rstar_cm"] / R_av) ** p["bexp"]
            d1 = p["mdot"] / (p["gas2dust"] * 4.0 * math.pi * R_av ** 2 * vexp)
            dens = np.broadcast_to(d1[:, None], (nR, nc)).copy()
            mdustscale = False
        elif denstype == "MEIXNER":
            # the axisymmetric superwind shell of Meixner et al. (2002) as
            # Init.f:3226-3238 writes it, r shifted by timeshift vexp1
            ra = R_av / AU
            rr = ra - p["timeshift"] * p["vexp1"] * 0.210944839e-5
            rin_m, rsw = p["meixrin"], p["meixrsw"]
            st, ct = np.sin(theta_av)[None, :], np.cos(theta_av)[None, :]
            rc = rr[:, None]
            dens = ((rc / rin_m) ** (-p["meixb"] * (1.0 + p["meixc"] * st ** p["meixf"]
                                                     * np.exp(-(rc / rsw) ** p["meixd"] + (rin_m / rsw) ** p["meixd"]))))
            dens = dens * (1.0 + p["meixa"] * (1.0 - ct) ** p["meixf"]
                           * np.exp(-(rc / rsw) ** p["meixe"] + (rin_m / rsw) ** p["meixe"]))
            dens = dens * (rc / ra[:, None]) ** 2
            dens = np.where(rc > rin_m, dens, 1e-60)
        elif denstype == "INFALL":
            # rotating infall onto a disk of radius rexp: mu0 of each
            # streamline by solve_mu0's scan of 1000 values (Init.f:5747-5764)
            mu1 = (np.arange(1000, dtype=np.float32) / np.float32(999)).astype(float)
            dens = np.zeros((nR, nc))
            Gc = 6.67300e-8
            for i in range(1, nR):
                rr = R_av[i] / (AU * p["rexp"])
                for j in range(nc):
                    mu = math.cos(theta_av[j])
                    d = np.abs((1.0 - mu1 ** 2) - rr * (1.0 - mu / mu1))
                    d = np.where(np.isnan(d), np.inf, d)
                    k = int(np.argmin(d)) if np.min(d) < 1e200 else None
                    mu0 = mu1[k] if k is not None else 0.0
                    dens[i, j] = ((p["minfall"] / (4.0 * math.pi * math.sqrt(Gc * p["mstar"] * R_av[i] ** 3)))
                                  * (1.0 + mu / mu0) ** (-0.5)
                                  * (mu / mu0 + 2.0 * mu0 ** 2 * p["rexp"] * AU / R_av[i]) ** (-1.0)) / p["gas2dust"]
            mdustscale = False
        elif denstype in ("POW", "DOUBLEPOW", "SIMILARITY", "DOUBLEPOWSIM"):
            ra = R_av / AU
            g = p["gamma_exp"] if p["gamma_exp"] >= 0.0 else 2.0 - p["denspow"]   # Init.f:1568
            if denstype == "POW":
                d1 = (AU / R_av) ** (p["denspow"] + 1.0)
            elif denstype == "SIMILARITY":
                d1 = (AU / R_av) ** (p["denspow"] + 1.0) * np.exp(-(R_av / (AU * p["rexp"])) ** g)
            elif denstype == "DOUBLEPOW":
                inner = (ra < p["rpow2"]) & (ra > p["rpow3"])
                d1 = np.where(inner, (p["rpow2"] * AU / R_av) ** (p["denspow"] + 1.0),
                              (p["rpow2"] * AU / R_av) ** (p["denspow2"] + 1.0))
            else:
                d1 = np.where(ra < p["rpow2"], (p["rpow2"] * AU / R_av) ** (p["denspow"] + 1.0),
                              (p["rpow2"] * AU / R_av) ** (p["denspow2"] + 1.0) * np.exp(-(R_av / (AU * p["rexp"])) ** g))
            dens = np.broadcast_to(d1[:, None], (nR, nc)).copy()
        elif denstype == "WEDGE":
            dens = np.full((nR, nc), 1e-200)
            for jj in range(1, 11):
                theta = thet[:-1] + (thet[1:] - thet[:-1]) * jj / 11.0
                inside = (180.0 * (math.pi / 2.0 - theta) / math.pi) < p["wedgeopen"]
                dens = dens + np.where(inside[None, :], ((AU / R_av) ** (p["denspow"] + 1.0))[:, None], 0.0)
        else:
            raise ValueError("denstype %r is not a closed-form density" % denstype)
    dens = np.array(dens, float)
    dens[0] = 1e-60
    mass = float((dens[1:] * V[1:]).sum())
    if not mdustscale:
        mtot = mass
    dens[1:] = dens[1:] * (mtot / mass)
    return np.maximum(dens, 1e-60), V


def grain_rv(amin, amax, apow, ns):
    """rv = sqrt(<a^2>) of a bin's ns sizes in cm (ComputePart.f:950-976;
    number weights n(a) ~ a^(1 - apow) of ComputePart.f:276-292)"""
    if ns == 1:
        r = np.array([10 ** ((math.log10(amin) + math.log10(amax)) / 2)])
        nr = np.ones(1)
    else:
        r = 10 ** (math.log10(amin) + (math.log10(amax) - math.log10(amin)) * np.arange(ns) / (ns - 1))
        nr = r ** (1.0 - apow)
    return math.sqrt((nr * r * r).sum() / nr.sum()) * 1e-4


def fixed_mp_settling(R, Theta, ntheta, dens, V, w, rho_grain, rv, alpha, zone, gas2dust=100.0, gamma=2.0):
    """Vertical settling of every grain in a fixed-structure zone.

    FixedMPSettling (MPSettling.f:132-168): per ring i the gas surface
    density and, per grain ii, hH = (1/(1+gamma))^(1/4) sqrt(alpha Sigma /
    (sqrt(2 pi) rho_ii rv_ii)), scale factor hH / sqrt(1 + hH^2).  The
    grain's density in the ring then takes the zone profile with the scale
    height times that factor, renormalised to the grain's mass in the ring
    (DiskStructure.f:345-380, fix_struct zones).  dens (nR, nc), V (nR, nc),
    w (nR, nc, ngrains) are the unsettled dust density, cell volumes and
    grain mass fractions; returns the settled dens and w."""
    nR, nc = dens.shape
    ng = w.shape[2]
    R_av = AU * 10.0 ** ((np.log10(R[:-1]) + np.log10(R[1:])) / 2.0)
    th = theta_centres(ntheta)
    dens_new = dens.copy()
    w_new = w.copy()
    c1 = (1.0 / (1.0 + gamma)) ** 0.25
    for i in range(1, nR):
        rr = R_av[i] * np.sin(th) / AU
        zz = R_av[i] * np.cos(th) / AU
        sigma = (dens[i] * gas2dust * V[i]).sum() / (math.pi * (R[i + 1] ** 2 - R[i] ** 2) * AU ** 2)
        rho_g = np.zeros((nc, ng))
        for ii in range(ng):
            hH = c1 * math.sqrt(alpha * sigma / (math.sqrt(2.0 * math.pi) * rho_grain[ii] * rv[ii]))
            scale = hH / math.sqrt(1.0 + hH * hH)
            hr = scale * zone["sh"] * (rr / zone["rsh"]) ** zone["shpow"]
            prof = np.zeros(nc)
            ok = rr > 0.0  # the polar cell (theta_av = 0) gets the density floor
            f2 = -(zz[ok] / hr[ok]) ** 2
            if ok[nc - 1]:
                f2[-1] = 0.0
            prof[ok] = np.exp(np.log(rr[ok] ** (-zone["denspow"]) / hr[ok]) + f2)
            m0 = (dens[i] * V[i] * w[i, :, ii]).sum()
            m1 = (prof * V[i]).sum()
            rg = prof * (m0 / m1) if m1 > 0 else np.zeros(nc)
            rho_g[:, ii] = np.maximum(rg, 1e-50)
        d = rho_g.sum(1)
        dens_new[i] = d
        w_new[i] = rho_g / d[:, None]
    return dens_new, w_new


def mrn_abundances(rgrain, rmin, rmax, index):
    """Mass fraction of each size bin for n(a) ~ a^-index (MRN.f gsd_MRN)."""
    rg = np.asarray(rgrain, float)
    n = rg.size
    lr = np.zeros(n + 1)
    for i in range(1, n):
        lr[i] = (math.log(rg[i - 1]) + math.log(rg[i])) / 2.0
    lr[0] = 2 * math.log(rg[0]) - lr[1] if n > 1 else math.log(rmin)
    lr[n] = 2 * math.log(rg[n - 1]) - lr[n - 1] if n > 1 else math.log(rmax)
    rint = np.exp(lr)
    ri = 4.0 - index
    fac = 3.0 / ri

    def piece(a, b):
        if abs(index - 4.0) <= 1e-6:
            return math.log(b) - math.log(a)
        return fac * (b ** ri - a ** ri)

    ab = np.zeros(n)
    for i in range(n):
        a, b = rint[i], rint[i + 1]
        if a >= rmax or b <= rmin:
            continue
        ab[i] = piece(max(a, rmin), min(b, rmax))
    norm = piece(max(rint[0], rmin), min(rint[n], rmax))
    ab /= norm
    ab[ab <= 1e-100] = 0.0
    return ab


def grain_bins(amin, amax, ngrains):
    """computepartNN:ngrains=N -> N log-spaced [amin_i, amax_i] bins
    (Init.f:1388-1447)."""
    edges = [10 ** (math.log10(amin) + math.log10(amax / amin) * i / ngrains) for i in range(ngrains + 1)]
    return [(edges[i], edges[i + 1]) for i in range(ngrains)]


# ---------------------------------------------------------------- model
def luminosity(T, R):
    """Luminosity of a blackbody sphere, T [K], R [cm] (Subroutines.f:24-35,
    with its constants; pi there is a single-precision literal)"""
    k, c, h = 1.3807e-16, 2.9979e10, 6.6261e-27
    pi = float(np.float32(3.1415926536))
    p4, k4 = (pi * pi) * (pi * pi), (k * k) * (k * k)
    return (((((2.0 * p4) * k4) / ((15.0 * ((h * h) * h)) * (c * c))) * ((T * T) * (T * T))) * pi) * (R * R)


def _read_pairs(path):
    xs, ys = [], []
    with open(path) as f:
        for line in f:
            parts = line.replace("d", "e").replace("D", "E").split()
            if len(parts) < 2:
                continue
            try:
                x, y = float(parts[0]), float(parts[1])
            except ValueError:
                continue
            xs.append(x)
            ys.append(y)
    return np.array(xs), np.array(ys)


def read_star(path, grid):
    """A stellar spectrum file (wavelength [micron], flux; one pair per
    line) on the wavelength grid (readstar, Subroutines.f:130-216): the
    file's points inside a grid bin (edges at the geometric midpoints) are
    averaged with weights |d(1/lambda)|; bins without a point take the
    log-log interpolation of readstar_interpol (Subroutines.f:219-258), and
    points beyond the file fall off as lambda^-2 from its last point.

    The bin edges are the reference's: its last assignment puts the upper
    edge of bin n-1 at grid(n)^2 / edge(n-1) and leaves the upper edge of
    bin n unset, zero under its -finit-local-zero build, so bin n-1 reaches
    up to grid(n) times the half-step and bin n always interpolates."""
    grid = np.asarray(grid, float)
    n = grid.size
    if n < 3:
        raise ValueError("read_star: at least three wavelengths")
    xe = np.empty(n + 1)
    xe[1:n] = np.sqrt(grid[:-1] * grid[1:])
    xe[0] = grid[0] ** 2 / xe[1]
    xe[n - 1] = grid[n - 1] ** 2 / xe[n - 2]
    xe[n] = 0.0
    ls, Fs = _read_pairs(path)
    nls = ls.size
    if nls < 3:
        raise ValueError("%s: fewer than three points" % path)
    dls = np.empty(nls)
    dls[1:-1] = (1.0 / ls[:-2] - 1.0 / ls[2:]) / 2.0
    dls[0], dls[-1] = dls[1], dls[-2]
    y, tot = np.zeros(n), np.zeros(n)
    done = np.zeros(n, bool)
    j = 0
    for i in range(nls):
        while True:
            if ls[i] < xe[j]:
                break
            if ls[i] > xe[j + 1]:
                j += 1
                if j >= n:
                    break
                continue
            y[j] = y[j] + Fs[i] * dls[i]
            tot[j] = tot[j] + dls[i]
            done[j] = True
            break
        if j >= n:
            break
    y[done] = y[done] / tot[done]
    if not done.all():
        y[~done] = _star_interpol(ls, Fs, grid[~done])
    return y


def _star_interpol(ls, Fs, grid):
    """readstar_interpol (Subroutines.f:219-258) on the grid points given"""
    n = grid.size
    y = np.zeros(n)
    i = 0
    x0, y0 = ls[0], Fs[0]
    while i < n and x0 >= grid[i]:
        y[i] = y0
        i += 1
    x1, y1 = x0, y0
    for k in range(1, ls.size):
        x1, y1 = ls[k], Fs[k]
        while i < n and x0 < grid[i] <= x1:
            if y1 > 1e-60 and y0 > 1e-60:
                y[i] = 10.0 ** (math.log10(y1) + (math.log10(grid[i]) - math.log10(x1)) *
                                (math.log10(y0) - math.log10(y1)) / (math.log10(x0) - math.log10(x1)))
            else:
                y[i] = y1 + (grid[i] - x1) * (y0 - y1) / (x0 - x1)
            i += 1
        if i >= n:
            return y
        x0, y0 = x1, y1
    for j in range(i, n):
        y[j] = y1 * x1 ** 2 / grid[j] ** 2
    return y


def integrate(nu, spec):
    """Trapezoid over frequency in the reference's order (Radiation.f:1-18)."""
    L = 0.0
    for i in range(len(nu) - 1):
        L = L + (abs(nu[i] - nu[i + 1]) * 0.5) * (spec[i] + spec[i + 1])
    return L


class Model:
    """Everything mcg_set_model uploads (module globals of the reference)."""

    def __init__(self, **kw):
        self.__dict__.update(kw)

    @property
    def ncell(self):
        return self.nr * (self.nt - 1)


def synthetic_lnk(lam, kpref=0.03):
    """n(lam) = clip(1.7 + 0.1 log10 lam, 1.5, 3.5), k(lam) = clip(kpref lam^0.5,
    1e-3, 2) on the grid (the synthetic dust of the benchmark decks)."""
    lam = np.asarray(lam, float)
    n = np.clip(1.7 + 0.1 * np.log10(lam), 1.5, 3.5)
    k = np.clip(kpref * lam ** 0.5, 1e-3, 2.0)
    return n, k


def disk_model(ctx, *, tstar=10000.0, rstar=2.5, rin=0.5, rout=100.0, mdust=1e-5, sh=0.05 * math.sqrt(2.0),
               rsh=1.0, shpow=1.125, denspow=1.0, nrad=100, ntheta=60, lam1=0.1, lam2=3000.0, nlam=100,
               amin=0.1, amax=1.0, apow=3.5, ngrains=20, ns=5, nf=20, fmax=0.8, blend=True, porosity=0.25,
               rho=3.0, kpref=0.03, scat_how=2, compositions=None, opacities=None):
    """Build a passive-disk model: star, ZONES density, grain bins with DHS
    opacities from the library (ComputePart per bin), Planck table.
    `opacities` may pass precomputed (Kabs, Ksca, F) per bin."""
    rstar_cm = rstar * RSUN
    lam, nu = wavelength_grid(lam1, lam2, nlam)
    R, Theta, thet, SinTheta = spatial_grid(rstar_cm, rin, rout, nrad, ntheta)
    dens, V = zones_density(R, Theta, thet, [dict(rin=rin, rout=rout, mdust=mdust, denspow=denspow, sh=sh,
                                                  rsh=rsh, shpow=shpow)])
    BB = api.bb_table(lam)
    Fstar = math.pi * rstar_cm ** 2 * BB[:, 0].copy()
    for i in range(nlam):
        Fstar[i] = math.pi * rstar_cm ** 2 * api.planck(tstar, lam[i])
    Lstar = integrate(nu, Fstar)
    bins = grain_bins(amin, amax, ngrains)
    rg = [math.sqrt(a * b) * 1e-4 for a, b in bins]
    w = mrn_abundances(rg, amin * 1e-4, amax * 1e-4, apow)
    if opacities is None:
        comps = compositions or [synthetic_lnk(lam, kpref)]
        parts = []
        for a, b in bins:
            parts.append(dict(lam=lam, e1=np.array([c[0] for c in comps]), e2=np.array([c[1] for c in comps]),
                              frac=np.ones(len(comps)), rho=np.full(len(comps), rho), amin=a, amax=b, apow=apow,
                              fmax=fmax, porosity=porosity, blend=blend, ns=ns, nf=nf))
        res = ctx.compute_part_batch(parts)
        Kabs = np.array([r["kabs"] for r in res])
        Ksca = np.array([r["ksca"] for r in res])
        F = np.array([r["F"] for r in res])
    else:
        Kabs, Ksca, F = opacities
    if scat_how == 0:
        Kabs = Kabs.copy()
        Ksca = np.zeros_like(Ksca)
    if scat_how == 1:
        F = np.ones_like(F)
    nr = R.size - 1
    nt = Theta.size
    ncomp = len(bins)
    comp_w = np.tile(w, (nr * (nt - 1), 1))
    return Model(nr=nr, nt=nt, R=R, Theta=Theta, SinTheta=SinTheta, thet=thet, dens=dens.reshape(-1),
                 V=V.reshape(-1), ncomp=ncomp, comp_w=comp_w, nlam=nlam, lam=lam, nu=nu, Kabs=Kabs, Ksca=Ksca,
                 F=F, BB=BB, Fstar=Fstar, Lstar=Lstar, Tstar=tstar, Rstar_cm=rstar_cm, scat_how=scat_how,
                 bins=bins, w=w)


LEARNED_COMPOSITIONS = (
    # k prefactor of the synthetic .lnk, porosity, DHS fmax
    (0.003, 0.2, 0.8),
    (0.03, 0.4, 0.5),
    (0.3, 0.0, 0.8),
)


def learned_disk_parts(lam, ngrains=50, amin=0.01, amax=1000.0, apow=3.5, ns=5, nf=20, rho=3.0,
                       compositions=LEARNED_COMPOSITIONS):
    """ComputePart inputs of the learned-opacities deck: per composition
    ngrains log bins from amin to amax (one synthetic .lnk each)"""
    bins = grain_bins(amin, amax, ngrains)
    parts = []
    for kp, por, fmax in compositions:
        n, k = synthetic_lnk(lam, kp)
        for a, b in bins:
            parts.append(dict(lam=lam, e1=np.array([n]), e2=np.array([k]), frac=np.ones(1), rho=np.full(1, rho),
                              amin=a, amax=b, apow=apow, fmax=fmax, porosity=por, blend=True, ns=ns, nf=nf))
    return parts, bins


def learned_disk_model(ctx, *, opacity="dhs", params=None, tstar=10000.0, rstar=2.5, rin=0.5, rout=100.0,
                       mdust=1e-3, sh=0.05 * math.sqrt(2.0), rsh=1.0, shpow=1.125, denspow=1.0, nrad=200,
                       ntheta=120, lam1=0.1, lam2=3000.0, nlam=200, ngrains=50, amin=0.01, amax=1000.0, apow=3.5,
                       ns=5, nf=20, rho=3.0, alpha=1e-3, scat_how=2, compositions=LEARNED_COMPOSITIONS,
                       settle=True, correct_stride=10):
    """The learned-opacities deck: three compositions in ngrains log bins
    each, equal mass per composition and MRN within it, vertically settled
    with alpha (FixedMPSettling; settle=False leaves the zone's unsettled
    profile, for a structure loop that settles the grains itself),
    opacities from the DHS kernels (opacity='dhs'), from the surrogate
    network (opacity='surrogate'), or from the network corrected by the DHS
    kernels at every correct_stride-th wavelength (opacity='corrected',
    surrogate.compute_part_corrected).  The model carries each grain bin's
    density (rho_grain, g/cm^3) and size (rv, cm) for the settling.
    Returns (model, opacity-stage seconds, bins served by the network)."""
    import time
    rstar_cm = rstar * RSUN
    lam, nu = wavelength_grid(lam1, lam2, nlam)
    R, Theta, thet, SinTheta = spatial_grid(rstar_cm, rin, rout, nrad, ntheta)
    zone = dict(rin=rin, rout=rout, mdust=mdust, denspow=denspow, sh=sh, rsh=rsh, shpow=shpow)
    dens, V = zones_density(R, Theta, thet, [zone])
    BB = api.bb_table(lam)
    Fstar = np.array([math.pi * rstar_cm ** 2 * api.planck(tstar, x) for x in lam])
    Lstar = integrate(nu, Fstar)
    parts, bins = learned_disk_parts(lam, ngrains, amin, amax, apow, ns, nf, rho, compositions)
    t0 = time.perf_counter()
    if opacity == "dhs":
        res = ctx.compute_part_batch(parts)
        served = 0
    elif opacity == "surrogate":
        from . import surrogate as S
        res, used = S.compute_part_surrogate(ctx, parts, params)
        served = int(used.sum())
    elif opacity == "corrected":
        from . import surrogate as S
        res, used, _ = S.compute_part_corrected(ctx, parts, params, stride=correct_stride)
        served = int(used.sum())
    else:
        raise ValueError("opacity must be 'dhs', 'surrogate' or 'corrected'")
    t_opac = time.perf_counter() - t0
    Kabs = np.array([r["kabs"] for r in res])
    Ksca = np.array([r["ksca"] for r in res])
    F = np.array([r["F"] for r in res])
    if scat_how == 0:
        Ksca = np.zeros_like(Ksca)
    ncomp = len(parts)
    rg = [math.sqrt(a * b) * 1e-4 for a, b in bins]
    wmrn = mrn_abundances(rg, amin * 1e-4, amax * 1e-4, apow)
    w0 = np.concatenate([wmrn / len(compositions) for _ in compositions])
    nr = R.size - 1
    nc = Theta.size - 1
    w = np.tile(w0, (nr, nc, 1))
    rho_grain = np.array([r["rho_av"] for r in res])
    rv = np.array([grain_rv(p["amin"], p["amax"], apow, ns) for p in parts])
    if settle:
        dens2, w2 = fixed_mp_settling(R, Theta, ntheta, dens, V, w, rho_grain, rv, alpha, zone)
    else:
        dens2, w2 = dens, w
    m = Model(nr=nr, nt=Theta.size, R=R, Theta=Theta, SinTheta=SinTheta, thet=thet, dens=dens2.reshape(-1),
              V=V.reshape(-1), ncomp=ncomp, comp_w=w2.reshape(nr * nc, ncomp), nlam=nlam, lam=lam, nu=nu,
              Kabs=Kabs, Ksca=Ksca, F=F, BB=BB, Fstar=Fstar, Lstar=Lstar, Tstar=tstar, Rstar_cm=rstar_cm,
              scat_how=scat_how, bins=bins, w=w0, rho_grain=rho_grain, rv=rv)
    return m, t_opac, served


def deck_model(ctx, deck, overrides=(), compute_parts=None):
    """Model and run parameters from an MCMax input deck: the keywords the
    packet loop and ComputePart read (Init.f:462-1240), with the reference's
    defaults (Init.f:66-384).

    Keywords used: startype ('PLANCK', or 'FILE' with starfile and lstar
    [Lsun]), tstar, rstar [Rsun]; rin, rout, nrad,
    ntheta; denstype ('ZONES') with zoneN:rin, rout, mdust, denspow, sh,
    rsh, shpow; lam1, lam2, nlam; scattype (NONE, ISOTROPIC, FULL, and
    RAYLEIGH: the Henyey-Greenstein/Rayleigh matrices of asymNN, asymbNN,
    wasymbNN, pmaxNN for partNN and fitspartNN grains);
    computepartNN:file (particle file: ns, nf, then per material an .lnk
    path and 'frac rho'), amin, amax, apow, fmax, ngrains, blend,
    porosity, norm_abun, standard ('FILE'), with amin, amax, apow (micron)
    as the deck-wide defaults; fitspartNN (a particle FITS file), partNN (an
    ASCII particle file) and opacNN (an opacity table) as grains taken as
    given; abunNN (relative mass of
    grain entry NN); fixmpset, alphaturb (settling of a one-zone
    disk); denstype 'FILE' with densfile (a denstemp.dat: its dust density
    and the grid rebuilt from its cell centres; rin and rout still give the
    outer edges); the closed-form denstypes of analytic_density (PASCUCCI,
    MIN, PARAMETERIZED, PINTE, SHELL, WEDGE) with denspow, shpow, sh1au,
    rexp, tau550, wedgeopen and mdust [Msun]; randomwalk, factrw, maxinteract, nruns, idum; nphotdiffuse,
    dtdiffuse (the diffusion step after the run); zoneN:fix, mstar,
    maxiter, epsiter (structure iterations).  A value that
    selects physics outside the packet loop (another startype or denstype,
    tcontact false) raises ValueError.

    deck: a path or the deck text; overrides: 'key=value' strings applied
    after the file (the -s switches).  compute_parts(parts) returns the
    ComputePart results of a list of grain bins (default: the library's
    DHS kernels, ctx.compute_part_batch).  Returns (model, run) with run =
    dict(seed, randomwalk, factRW, maxinteract, nruns) for mcradiation plus
    nphotdiffuse, dtdiffuse (defaults 25 and 1, Init.f:140-141) and the
    structure-iteration inputs zones (rin, rout, sh, rsh, shpow, denspow,
    fix), Mstar [g], maxiter, epsiter (defaults 10 and 3, Init.f:113-114)."""
    base = "."
    if os.path.exists(str(deck)):
        base = os.path.dirname(os.path.abspath(deck))
        with open(deck) as f:
            text = f.read()
    else:
        text = deck
    d = parse_deck(text, overrides)

    def v(key, default, cast=float):
        return deck_value(d, key, default, cast)

    startype = v("startype", "PLANCK", str).upper()
    if startype not in ("PLANCK", "FILE"):
        raise ValueError("startype: 'PLANCK' or 'FILE' stars")
    denstype = v("denstype", "ZONES", str).upper()
    if denstype not in ("ZONES", "FILE", "SHELLFILE") + ANALYTIC_DENSITIES + THIN_START_DENSITIES:
        raise ValueError("denstype: 'ZONES', 'FILE' or one of %s"
                         % ", ".join(ANALYTIC_DENSITIES + THIN_START_DENSITIES))
    if denstype == "PARAMETERIZED" and ("scalesh" in d or "rimscale" in d):
        raise ValueError("PARAMETERIZED: scale-height factors (scalesh, rimscale) are not built")
    if not v("tcontact", True, bool):
        raise ValueError("tcontact: only thermal contact (Bjorkman-Wood with one temperature per cell)")
    scattype = v("scattype", "ISOTROPIC", str).upper()
    scat = {"NONE": 0, "ISOTROPIC": 1, "FULL": 2, "RAYLEIGH": 2}.get(scattype)
    if scat is None:
        raise ValueError("scattype: NONE, ISOTROPIC, FULL or RAYLEIGH")
    tstar, rstar = v("tstar", 10000.0), v("rstar", 2.1)
    rin, rout = v("rin", 0.5), v("rout", 1000.0)
    nrad, ntheta = v("nrad", 70, int), v("ntheta", 60, int)
    lam1, lam2, nlam = v("lam1", 0.1), v("lam2", 10000.0), v("nlam", 100, int)
    zones = []
    for iz in range(1, 11):
        kz = "zone%d:" % iz
        if not any(k.startswith(kz) for k in d):
            continue
        zones.append(dict(rin=v(kz + "rin", rin), rout=v(kz + "rout", rout), mdust=v(kz + "mdust", 1e-5),
                          denspow=v(kz + "denspow", 1.0), sh=v(kz + "sh", 0.01), rsh=v(kz + "rsh", 1.0),
                          shpow=v(kz + "shpow", 1.1), fix=v(kz + "fix", False, bool),
                          alphaturb=v(kz + "alphaturb", v("alphaturb", 1e-4))))
    if zones and denstype in ("SHELLFILE",) + ANALYTIC_DENSITIES + THIN_START_DENSITIES:
        raise ValueError("denstype %s takes no zoneN:* keywords" % denstype)
    if not zones and denstype == "ZONES":
        raise ValueError("no zoneN:* keywords")
    # grain bins of every computepart entry (Init.f:746-789, 1323-1420)
    # grains by index NN: computepartNN:* (computed, then split into size
    # bins), fitspartNN (a particle FITS file, ReadParticleFits), opacNN (an
    # opacity table, readopacity) and partNN (an ASCII particle file,
    # readparticle) (Init.f:697-740, 3333-3400)
    kinds = {}
    for k in d:
        if k.startswith("computepart") and ":" in k and k[11:k.index(":")].isdigit():
            kinds[int(k[11:k.index(":")])] = "computepart"
        elif k.startswith("fitspart") and k[8:].isdigit():
            kinds[int(k[8:])] = "fitspart"
        elif k.startswith("opac") and k[4:].isdigit():
            kinds[int(k[4:])] = "opac"
        elif k.startswith("part") and k[4:].isdigit():
            kinds[int(k[4:])] = "part"
    entries = sorted(kinds)
    if not entries:
        raise ValueError("no grains: computepartNN:*, fitspartNN or opacNN keywords")
    rstar_cm = rstar * RSUN
    lam, nu = wavelength_grid(lam1, lam2, nlam)
    parts, weights, slots = [], [], []
    abun = np.array([v("abun%02d" % e, v("abun%d" % e, 1.0)) for e in entries])
    abun = abun / abun.sum()

    def path_of(val):
        return val if os.path.isabs(val) else os.path.join(base, val)

    for e, ab in zip(entries, abun):
        if kinds[e] != "computepart":
            key = ("%s%02d" % (kinds[e], e)) if ("%s%02d" % (kinds[e], e)) in d else "%s%d" % (kinds[e], e)
            from . import particle_fits as PF
            mat = None
            if scattype == "RAYLEIGH" and kinds[e] != "opac":
                # Henyey-Greenstein / Rayleigh matrices (Init.f:3336-3348, 928-955)
                mat = PF.rayleigh_hg_matrix(v("asym%02d" % e, v("asym%d" % e, 2.0)),
                                            v("asymb%02d" % e, v("asymb%d" % e, 2.0)),
                                            v("wasymb%02d" % e, v("wasymb%d" % e, 0.0)),
                                            v("pmax%02d" % e, v("pmax%d" % e, 1.0)))
            extra = dict(nspike=v("nspike", 0, int) if scat == 2 else 0,
                         wasym2=v("wasymb%02d" % e, v("wasymb%d" % e, 0.0)),
                         asym2=v("asymb%02d" % e, v("asymb%d" % e, 2.0)))
            if kinds[e] == "fitspart":
                r = PF.read_particle_fits(path_of(v(key, "", str)), lam, matrix=mat, **extra)
            elif kinds[e] == "part":
                r = PF.read_particle_ascii(path_of(v(key, "", str)), lam, matrix=mat, **extra)
            else:
                r = PF.read_opacity_file(path_of(v(key, "", str)), lam)
            if kinds[e] != "fitspart":
                r.update(rho_av=float("nan"), rv=float("nan"), amin=float("nan"), amax=float("nan"))
            slots.append(("file", r))
            weights.append(ab)
            continue
        kp = "computepart%02d:" % e if any(k.startswith("computepart%02d:" % e) for k in d) else \
            "computepart%d:" % e
        if v(kp + "standard", "FILE", str).upper() != "FILE":
            raise ValueError(kp + "standard: only 'FILE' particle files")
        pfile = v(kp + "file", None, str)
        if not pfile:
            raise ValueError(kp + "file missing")
        ns, nf, mats = read_particle_file(path_of(pfile))
        e1, e2, frac, rho = [], [], [], []
        for lnk, fr, rh in mats:
            n_, k_ = readrefind(lnk, lam)
            e1.append(n_)
            e2.append(k_)
            frac.append(fr)
            rho.append(rh)
        # unset sizes fall back to the deck-wide size distribution
        # (Init.f:1155-1163, 1320-1322; defaults Init.f:174-176)
        amin, amax = v(kp + "amin", -1.0), v(kp + "amax", -1.0)
        apow, ngr = v(kp + "apow", 1e5), v(kp + "ngrains", 1, int)
        if amin <= 0:
            amin = v("amin", v("mrn_rmin", 0.01))
        if amax <= 0:
            amax = v("amax", v("mrn_rmax", 1000.0))
        if apow > 100:
            apow = v("apow", v("mrn_index", 3.5))
        bins = grain_bins(amin, amax, ngr) if ngr > 1 else [(amin, amax)]
        rg = [math.sqrt(a * b) * 1e-4 for a, b in bins]
        wmrn = mrn_abundances(rg, amin * 1e-4, amax * 1e-4, apow) if ngr > 1 else np.ones(1)
        for (a, b), wb in zip(bins, wmrn):
            slots.append(("part", len(parts)))
            parts.append(dict(lam=lam, e1=np.array(e1), e2=np.array(e2), frac=np.array(frac), rho=np.array(rho),
                              amin=a, amax=b, apow=apow, fmax=v(kp + "fmax", 0.0), porosity=v(kp + "porosity", 0.25),
                              blend=v(kp + "blend", True, bool), ns=ns, nf=nf,
                              normalize_abun=v(kp + "norm_abun", -1.0)))
            weights.append(ab * wb)
    computed = (compute_parts or ctx.compute_part_batch)(parts) if parts else []
    res, grain_info = [], []
    for kind, x in slots:
        if kind == "part":
            p = parts[x]
            res.append(computed[x])
            grain_info.append(((p["amin"], p["amax"]), grain_rv(p["amin"], p["amax"], p["apow"], p["ns"])))
        else:
            res.append(x)
            grain_info.append(((x["amin"], x["amax"]), x["rv"]))
    Kabs = np.array([r["kabs"] for r in res])
    Ksca = np.array([r["ksca"] for r in res])
    F = np.array([r["F"] for r in res])
    if scat == 0:
        Ksca = np.zeros_like(Ksca)
    if scat == 1:
        F = np.ones_like(F)
    gasdens = None
    if denstype == "FILE":
        # the dust density of a denstemp file and the grid rebuilt from its
        # cell centres (Init.f:2727-2752, readstruct InputOutput.f:579)
        from .outputs import read_denstemp, read_denstemp_fits
        dfile = v("densfile", "", str)
        if not os.path.isabs(dfile):
            dfile = os.path.join(base, dfile)
        dt = read_denstemp_fits(dfile) if ".fits" in os.path.basename(dfile) else read_denstemp(dfile)
        R, Theta, thet, SinTheta = grid_from_centres(rstar_cm, rin, rout, dt["r_av"], dt["theta_av"])
        V = cell_volumes(R, Theta)
        dens = np.full(V.shape, 1e-60)
        dens[1:] = dt["dens"]
    elif denstype == "SHELLFILE":
        # a radial density table taken as the cells' density, not scaled
        # to a dust mass (Init.f:3005-3023)
        R, Theta, thet, SinTheta = spatial_grid(rstar_cm, rin, rout, nrad, ntheta)
        V = cell_volumes(R, Theta)
        R_av = 10.0 ** ((np.log10(R[:-1]) + np.log10(R[1:])) / 2.0)
        dens = np.full(V.shape, 1e-60)
        dens[1:] = np.maximum(regridlog(path_of(v("densfile", "", str)), R_av[1:]), 1e-60)[:, None]
    elif denstype == "SURFFILE":
        R, Theta, thet, SinTheta = spatial_grid(rstar_cm, rin, rout, nrad, ntheta)
        gfile = v("gasdensfile", "", str)
        dens, V, gasdens = surface_density(
            R, Theta, path_of(v("densfile", "", str)), path_of(gfile) if gfile else None, v("gas2dust", 100.0),
            v("mdust", 1e-15) * MSUN if "mdust" in d else None)
    elif denstype in ANALYTIC_DENSITIES + THIN_START_DENSITIES:
        meixrin = v("meixrin", -1.0) if v("meixrin", -1.0) > 0.0 else rin
        meixd, meixe = v("meixd", 1.0), v("meixe", 3.0)
        if meixd <= 0.0:     # Init.f:1529-1530, in this order
            meixd = meixe
        if meixe <= 0.0:
            meixe = meixd
        timeshift = v("timeshift", 0.0)
        rin_g, rout_g = rin, rout
        if denstype == "MEIXNER" and timeshift != 0.0:
            # the shell has expanded for timeshift years at vexp1 km/s: the
            # grid's edges move out by timeshift vexp1 0.210944839 AU
            # (Init.f:1634-1636), while the shell's own inner radius stays
            # at the unshifted rin (MeixRin is set before, Init.f:1528)
            shift = timeshift * v("vexp1", v("vexp", 10.0)) * 0.210944839
            rin_g, rout_g = rin + shift, rout + shift
        R, Theta, thet, SinTheta = spatial_grid(rstar_cm, rin_g, rout_g, nrad, ntheta)
        kext = [r["kext"] if "kext" in r else np.asarray(r["kabs"]) + np.asarray(r["ksca"]) for r in res]
        dens, V = analytic_density(denstype, R, Theta, thet, dict(
            rin=rin, rout=rout, denspow=v("denspow", 1.0), shpow=v("shpow", 1.3), sh1au=v("sh1au", 0.03),
            rexp=v("rexp", 1e10), tau550=v("tau550", 100.0), wedgeopen=v("wedgeopen", 5.0),
            denspow2=v("denspow2", 1.0), rpow2=v("rpow2", 1e10), rpow3=v("rpow3", 0.0),
            gamma_exp=v("gamma_exp", -1.0),
            mdot=v("mdot", 1e-8) * MSUN / (365.25 * 24.0 * 60.0 * 60.0),
            minfall=(v("minfall", -1.0) if v("minfall", -1.0) >= 0.0 else v("mdot", 1e-8)) * MSUN / (365.25 * 24.0 * 60.0 * 60.0),
            vexp1=v("vexp1", v("vexp", 10.0)) * 100000.0,
            vexp2=(v("vexp2", -10.0) if v("vexp2", -10.0) > 0.0 else v("vexp1", v("vexp", 10.0))) * 100000.0,
            bexp=v("bexp", 0.5), gas2dust=v("gas2dust", 100.0), mstar=v("mstar", 2.5) * MSUN, rstar_cm=rstar_cm,
            meixa=v("meixa", 8.0), meixb=v("meixb", 2.0), meixc=v("meixc", 2.0), meixd=meixd,
            meixe=meixe, meixf=v("meixf", 1.0), meixrsw=v("meixrsw", 1800.0),
            meixrin=meixrin, timeshift=timeshift,
            mtot=v("mdust", 1e-15) * MSUN, mdustscale="mdust" in d), lam=lam, kext=kext)
    else:
        R, Theta, thet, SinTheta = spatial_grid(rstar_cm, rin, rout, nrad, ntheta)
        dens, V = zones_density(R, Theta, thet, zones)
    BB = api.bb_table(lam)
    if startype == "FILE":
        # the file's spectrum scaled to lstar solar luminosities (Init.f:504-509, 2677-2682)
        if "lstar" not in d:
            raise ValueError("startype 'FILE' needs lstar")
        sfile = v("starfile", "", str)
        if not os.path.isabs(sfile):
            sfile = os.path.join(base, sfile)
        Fstar = read_star(sfile, lam)
        Lstar = v("lstar", 1.0) * luminosity(5778.0, RSUN)
        Fstar = Lstar * Fstar / integrate(nu, Fstar)
    else:
        Fstar = np.array([math.pi * rstar_cm ** 2 * api.planck(tstar, x) for x in lam])
        Lstar = integrate(nu, Fstar)
    if v("av", 0.0) != 0.0 or v("adjustav", False, bool):
        # the interstellar extinction of the observed fluxes (Reddening.f,
        # Telescope.f:85-92, 233-234) is not built: refuse rather than write
        # unreddened fluxes
        raise ValueError("av / adjustav: interstellar reddening is not built")
    nr, nt = R.size - 1, Theta.size
    w0 = np.array(weights)
    w = np.tile(w0, (nr, nt - 1, 1))
    if v("fixmpset", False, bool):
        if len(zones) != 1:
            raise ValueError("fixmpset: settling of a one-zone disk")
        rv = np.array([g[1] for g in grain_info])
        rho_g = np.array([r["rho_av"] for r in res])
        if not (np.all(np.isfinite(rv)) and np.all(np.isfinite(rho_g))):
            raise ValueError("fixmpset: an opacNN grain has no size or density to settle")
        dens, w = fixed_mp_settling(R, Theta, ntheta, dens, V, w, rho_g, rv, v("alphaturb", 1e-4), zones[0])
    m = Model(nr=nr, nt=nt, R=R, Theta=Theta, SinTheta=SinTheta, thet=thet, dens=dens.reshape(-1), V=V.reshape(-1),
              ncomp=len(res), comp_w=w.reshape(nr * (nt - 1), len(res)), nlam=nlam, lam=lam, nu=nu, Kabs=Kabs,
              Ksca=Ksca, F=F, BB=BB, Fstar=Fstar, Lstar=Lstar, Tstar=tstar, Rstar_cm=rstar_cm, scat_how=scat,
              bins=[g[0] for g in grain_info], w=w0, distance=v("distance", 100.0),
              gasdens=None if gasdens is None else gasdens.reshape(-1))
    # the overflow roulette is on only when the deck sets maxinteract
    # (overflow = .false. by default, Init.f:139,144,637-639); maxruntime -1
    # is off (Init.f:355)
    run = dict(seed=abs(v("idum", -42, int)), randomwalk=v("randomwalk", False, bool), factRW=v("factrw", 10.0),
               maxinteract=v("maxinteract", 0, int), maxruntime=v("maxruntime", -1.0), nruns=v("nruns", 1, int),
               nphotdiffuse=v("nphotdiffuse", 25, int), dtdiffuse=v("dtdiffuse", 1.0),
               zones=[(z["rin"], z["rout"], z["sh"], z["rsh"], z["shpow"], z["denspow"], z["fix"]) for z in zones],
               Mstar=v("mstar", 2.5) * MSUN, maxiter=v("maxiter", 10, int), epsiter=v("epsiter", 3.0),
               incangle=v("incangle", 45.0), outputfits=v("outputfits", False, bool), posangle=v("posangle", 0.0),
               vis_norm_fov=v("vis_norm_fov", True, bool))
    # the structure loop runs for zones without a fixed structure or with
    # iter=.true. (Init.f:563,1519); it, the power-law densities and every
    # deck with zones start from the optically thin structure
    # (Init.f:3924-3960)
    mpset = v("mpset", False, bool)
    if mpset and v("fixmpset", False, bool):
        raise ValueError("mpset and fixmpset: one settling prescription at a time")
    run["iterate"] = any(not z["fix"] for z in zones) or v("iter", False, bool) or (mpset and bool(zones))
    run["settling"] = None
    run["fixed"] = None
    if v("fixmpset", False, bool):
        # FixedMPSettling again at the start of every structure pass
        # (DiskStructure.f:108), from the state the pass starts from
        run["fixed"] = dict(rho=rho_g, rv=rv, alpha=v("alphaturb", 1e-4), gas2dust=v("gas2dust", 100.0))
    if mpset:
        # MPSettling's inputs (Init.f:2906, 3070: the zones' alphaturb on their rings)
        R_av = AU * 10.0 ** ((np.log10(R[:-1]) + np.log10(R[1:])) / 2.0)
        alpha = np.full(nr, v("alphaturb", 1e-4))
        for z in zones:
            alpha[(R_av >= z["rin"] * AU) & (R_av <= z["rout"] * AU)] = z["alphaturb"]
        rv = np.array([g[1] for g in grain_info])
        rho_g = np.array([r["rho_av"] for r in res])
        if not (np.all(np.isfinite(rv)) and np.all(np.isfinite(rho_g))):
            raise ValueError("mpset: an opacNN grain has no size or density to settle")
        run["settling"] = dict(rho=rho_g, rv=rv, alpha=alpha,
                               rscale=np.array([r.get("rscale", 1.0) for r in res]), gas2dust=v("gas2dust", 100.0))
    # the reference runs the start whenever the deck has zones (nzones /= 0)
    # or settles with fixmpset (Init.f:3923-3927): its structure passes
    # rebuild a fixed zone's profile at the cell centres, with
    # FixedMPSettling's factors recomputed before each (run["fixed"])
    run["thin_start"] = (run["iterate"] or denstype in THIN_START_DENSITIES or mpset
                         or v("fixmpset", False, bool) or bool(zones))
    return m, run


CONFIGS = {
    # small thin disk: the case a CPU run finishes quickly
    "small_thin_disk": dict(mdust=1e-5, nrad=100, ntheta=60, nlam=100),
    # precision disk: optically thick midplane exercising the random walk
    "precision_disk": dict(mdust=1e-3, nrad=200, ntheta=120, nlam=200),
}
