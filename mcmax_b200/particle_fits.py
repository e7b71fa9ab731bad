"""The reference's particle cache: ComputePart results stored as
particleNNNN.fits(.gz), so that a run finds the opacities of a grain bin it
has computed before instead of computing them again, and so that MCMax
itself reads the files this library writes.

    particle_file_name(dir, ii, iopac, frac, abun_in_name)   ComputePart.f:161-187, 906-938
    read_opacity_file(path, lam), read_particle_ascii(...)   readopacity, readparticle (Init.f:4664-4990)
    dust_moments(amin, amax, apow, ns)                       ComputePart.f:276-292, 950-976
    write_particle_fits(path, lam, res, ...)                 ParticleFITS, ComputePart.f:884-1093
    check_particle_file(path, ...)                           checkparticlefile, ComputePart.f:559-688
    read_particle_fits(path, lam)                            ReadParticleFits, ReadParticleFits.f:1-312
    find_particle_file(dir, ii, ...)                         the cache lookup of ComputePart.f:160-205

The layout: a primary image of NAXIS1 = nlam, NAXIS2 = 4 (wavelength
[micron], Kext, Kabs, Ksca [cm^2/g]) and one IMAGE extension of NAXIS1 =
nlam, NAXIS2 = 6, NAXIS3 = 180 (F11, F12, F22, F33, F34, F44 per
scattering-angle bin), both 64-bit IEEE big-endian, with the grain keywords
(R_MIN, R_MAX, R_POW, F_MAX, A1-A3, DENSITY, POROSITY, FILEnn, FRACnn,
RHOnn, N_RADII, N_MAT) in the primary header.  The FITS container itself
(2880-byte blocks of 80-character cards, strings longer than a card on
CONTINUE cards) is written and read here from the FITS standard; no FITS
library is needed.
"""
import gzip
import math
import os

import numpy as np

BLOCK = 2880
CARD = 80
NANG = 180


# ---------------------------------------------------------------- names
def particle_file_name(particledir, ii, iopac=1, frac=None, abun_in_name=0, gz=True):
    """particleNNNN[_fX.X...][_NN].fits[.gz]: the volume fractions in the
    name when abun_in_name > 0 (1-4 digits after the point, 5 above)"""
    name = "particle%04d" % ii
    if abun_in_name > 0:
        nd = abun_in_name if abun_in_name <= 4 else 5
        for fr in frac:
            name += "_f" + ("%*.*f" % (nd + 2, nd, float(np.float32(fr))))
    if iopac != 1:
        name += "_%02d" % iopac
    name += ".fits" + (".gz" if gz else "")
    return os.path.join(particledir, name)


def dust_moments(amin, amax, apow, ns):
    """(a1, a2, a3) = <a>, <a^2>, <a^3> in micron powers over the ns sizes
    of a bin with number weights a^(1 - apow); sizes and weights in single
    precision as the reference holds them"""
    if ns == 1:
        r = np.array([10.0 ** ((math.log10(amin) + math.log10(amax)) / 2.0)], np.float32)
        nr = np.ones(1, np.float32)
    else:
        k = np.arange(ns)
        r = (10.0 ** (math.log10(amin) + (math.log10(amax) - math.log10(amin)) * k / (ns - 1))).astype(np.float32)
        nr = (r.astype(np.float64) ** (1.0 - apow)).astype(np.float32)
        nr = (nr / (nr.astype(np.float64) * r.astype(np.float64) ** 3).sum()).astype(np.float32)
    r64, n64 = r.astype(np.float64), nr.astype(np.float64)
    a0 = n64.sum()
    return tuple(float(np.float32((n64 * r64 ** p).sum() / a0)) for p in (1, 2, 3))


# ---------------------------------------------------------------- FITS cards
def _string_cards(key, value, comment=""):
    """a string keyword; values longer than one card continue on CONTINUE
    cards, each part but the last ending in '&' (the FITS long-string
    convention)"""
    parts, cur = [], ""
    for ch in str(value):
        esc = "''" if ch == "'" else ch
        if len(cur) + len(esc) > 66:
            parts.append(cur + "&")
            cur = ""
        cur += esc
    parts.append(cur)
    cards = []
    for k, part in enumerate(parts):
        head = key.upper().ljust(8)[:8] + "= " if k == 0 else "CONTINUE  "
        c = head + ("'" + part.ljust(8) + "'").ljust(20)
        if comment and k == len(parts) - 1 and len(c) + 3 + len(comment) <= CARD:
            c += " / " + comment
        cards.append(c.ljust(CARD))
    return "".join(cards)


def _card(key, value=None, comment="", decimals=8):
    if isinstance(value, str):
        return _string_cards(key, value, comment)
    if value is None:
        c = key.ljust(8)
    else:
        if isinstance(value, bool):
            v = ("T" if value else "F").rjust(20)
        elif isinstance(value, (int, np.integer)):
            v = str(int(value)).rjust(20)
        else:
            v = ("%.*E" % (decimals, float(value))).rjust(20)
        c = key.upper().ljust(8)[:8] + "= " + v
        if comment:
            c += " / " + comment
    if len(c) > CARD:
        raise ValueError("FITS card longer than 80 characters: %r" % c)
    return c.ljust(CARD)


def _header(cards):
    h = "".join(cards) + "END".ljust(CARD)
    h += " " * ((-len(h)) % BLOCK)
    return h.encode("ascii")


def _data(a):
    b = np.ascontiguousarray(a, dtype=">f8").tobytes()
    return b + b"\0" * ((-len(b)) % BLOCK)


def _parse_value(s):
    s = s.strip()
    if s.startswith("'"):
        out, i = "", 1
        while i < len(s):
            if s[i] == "'":
                if i + 1 < len(s) and s[i + 1] == "'":
                    out += "'"
                    i += 2
                    continue
                break
            out += s[i]
            i += 1
        return out.rstrip()
    v = s.split("/")[0].strip()
    if v in ("T", "F"):
        return v == "T"
    try:
        return int(v)
    except ValueError:
        return float(v.replace("D", "E").replace("d", "e"))


def _read_hdus(raw):
    """[(header dict, data array in C order)] of every HDU"""
    hdus, pos = [], 0
    while pos + BLOCK <= len(raw):
        hdr, done, last = {}, False, None
        while not done:
            blk = raw[pos:pos + BLOCK].decode("ascii")
            pos += BLOCK
            for k in range(0, BLOCK, CARD):
                c = blk[k:k + CARD]
                key = c[:8].strip()
                if key == "END":
                    done = True
                    break
                if key == "CONTINUE" and isinstance(hdr.get(last), str) and hdr[last].endswith("&"):
                    hdr[last] = hdr[last][:-1] + _parse_value(c[10:])
                elif c[8:10] == "= ":
                    hdr[key] = _parse_value(c[10:])
                    last = key
        bitpix = hdr["BITPIX"]
        shape = [hdr["NAXIS%d" % i] for i in range(hdr["NAXIS"], 0, -1)]
        dt = {-64: ">f8", -32: ">f4", 8: "u1", 16: ">i2", 32: ">i4", 64: ">i8"}[bitpix]
        n = int(np.prod(shape)) if shape else 0
        nb = n * abs(bitpix) // 8
        data = np.frombuffer(raw[pos:pos + nb], dtype=dt).astype(np.float64).reshape(shape) if n else None
        pos += nb + ((-nb) % BLOCK)
        hdus.append((hdr, data))
    return hdus


def _open(path):
    with open(path, "rb") as f:
        raw = f.read()
    return gzip.decompress(raw) if raw[:2] == b"\x1f\x8b" else raw


# ---------------------------------------------------------------- write / check / read
def write_particle_fits(path, lam, res, amin, amax, apow, fmax, blend, porosity, frac, rho, lnkfiles, ns):
    """ParticleFITS: the ComputePart result `res` (kext, kabs, ksca, F
    (nlam, 6, 180), rho_av) of one grain bin on wavelengths lam.  frac is
    normalised to a sum of 1 as the reference does before writing.
    Returns the file's dust moments (a1, a2, a3)."""
    lam = np.asarray(lam, float)
    nlam = lam.size
    frac = np.asarray(frac, float)
    frac = frac / frac.sum()
    a1, a2, a3 = dust_moments(amin, amax, apow, ns)
    r32 = lambda x: float(np.float32(x))
    cards = [_card("SIMPLE", True, "file does conform to FITS standard"),
             _card("BITPIX", -64, "number of bits per data pixel"),
             _card("NAXIS", 2, "number of data axes"),
             _card("NAXIS1", nlam, "length of data axis 1"),
             _card("NAXIS2", 4, "length of data axis 2"),
             _card("EXTEND", True, "FITS dataset may contain extensions"),
             _card("r_min", r32(amin), "[micron]"), _card("r_max", r32(amax), "[micron]"),
             _card("r_pow", r32(apow)), _card("f_max", r32(fmax)),
             _card("a1", a1, "[micron]"), _card("a2", a2, "[micron^2]"), _card("a3", a3, "[micron^3]"),
             _card("density", r32(res["rho_av"]), "[g/cm^3]")]
    if blend:
        cards.append(_card("porosity", r32(porosity), "[g/cm^3]"))
    for i, fn in enumerate(lnkfiles):
        cards.append(_card("file%02d" % (i + 1), str(fn)))
    for i, fr in enumerate(frac):
        cards.append(_card("frac%02d" % (i + 1), r32(fr), "[volume fraction]"))
    for i, rh in enumerate(rho):
        cards.append(_card("rho%02d" % (i + 1), r32(rh), "[g/cm^3]"))
    cards += [_card("n_radii", int(ns)), _card("n_mat", len(frac))]
    hdu0 = np.stack([lam, np.asarray(res["kext"], float), np.asarray(res["kabs"], float),
                     np.asarray(res["ksca"], float)])
    F = np.asarray(res["F"], float).reshape(nlam, 6, NANG)
    ext = [_card("XTENSION", "IMAGE", "IMAGE extension"), _card("BITPIX", -64, "number of bits per data pixel"),
           _card("NAXIS", 3, "number of data axes"), _card("NAXIS1", nlam, "length of data axis 1"),
           _card("NAXIS2", 6, "length of data axis 2"), _card("NAXIS3", NANG, "length of data axis 3"),
           _card("PCOUNT", 0, "required keyword; must = 0"), _card("GCOUNT", 1, "required keyword; must = 1")]
    raw = _header(cards) + _data(hdu0) + _header(ext) + _data(F.transpose(2, 1, 0))
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(path, "wb") as f:
        f.write(gzip.compress(raw) if path.endswith(".gz") else raw)
    return a1, a2, a3


def _e8(x):
    return "%.7E" % float(np.float32(x))


def check_particle_file(path, amin, amax, apow, ns, fmax, blend, porosity, frac, rho, lnkfiles, checkfrac=True):
    """checkparticlefile: True when the cached file was made for the same
    grain: at least ns sizes, the same size range and power (the power
    only for ns > 1), fmax, porosity (blended grains), volume fractions
    (checkfrac), material densities and .lnk files, single-precision
    values compared to 8 significant digits"""
    try:
        hdr = _read_hdus(_open(path))[0][0]
    except (OSError, ValueError, KeyError, UnicodeDecodeError):
        return False
    try:
        if hdr["N_RADII"] < ns:
            return False
        if _e8(hdr["R_MIN"]) != _e8(amin) or _e8(hdr["R_MAX"]) != _e8(amax):
            return False
        if ns > 1 and _e8(hdr["R_POW"]) != _e8(apow):
            return False
        if _e8(hdr["F_MAX"]) != _e8(fmax):
            return False
        if blend and _e8(hdr["POROSITY"]) != _e8(porosity):
            return False
        fr = np.asarray(frac, float)
        fr = fr / fr.sum()
        for i in range(len(fr)):
            if checkfrac and _e8(hdr["FRAC%02d" % (i + 1)]) != _e8(fr[i]):
                return False
            if _e8(hdr["RHO%02d" % (i + 1)]) != _e8(rho[i]):
                return False
            if str(hdr["FILE%02d" % (i + 1)]).strip() != str(lnkfiles[i]).strip():
                return False
    except KeyError:
        return False
    return True


def _regrid(L, Kx, Ka, Ks, M, lam, nspike=0, spike="min", wasym2=0.0, asym2=2.0):
    """opacities and matrices of a tabulated grain on the wavelength grid
    lam, as ReadParticleFits (ReadParticleFits.f:112-222) and readopacity
    (Init.f:4929-4972) regrid them: below the table's first wavelength the
    first entry; inside, linear in wavelength between the bracketing entries
    (Kext too); beyond the last, Ksca ~ lam^-4, Kabs ~ lam^-2, Kext = Kabs +
    Ksca and F held; then every matrix renormalised so that sum F11
    sin(theta) = sum sin(theta) over the 180 bins.  M: (nl, 6, 180).

    nspike > 0 (with full scattering) makes the first nspike degrees flat:
    F11 there takes the smallest F11 of bins 1..nspike+1 (spike "min",
    ReadParticleFits.f:224-270) or F11 of bin nspike+1 (spike "next",
    readparticle, Init.f:4816-4845), the other elements scaled alike; Ksca
    drops by the removed part and the matrix is renormalised.  wasym2 != 0
    mixes a Henyey-Greenstein F11 of asymmetry asym2 in with that weight
    (ReadParticleFits.f:272-285)."""
    lam = np.asarray(lam, float)
    nlam = lam.size
    kext, kabs, ksca = np.zeros(nlam), np.zeros(nlam), np.zeros(nlam)
    F = np.zeros((nlam, 6, NANG))
    nl = L.size
    i = 0
    while i < nlam and L[0] >= lam[i]:
        kext[i], kabs[i], ksca[i], F[i] = Kx[0], Ka[0], Ks[0], M[0]
        i += 1
    for r in range(1, nl):
        l0, l1 = L[r - 1], L[r]
        while i < nlam and l0 <= lam[i] <= l1:
            t = (lam[i] - l1) / (l0 - l1)
            kext[i] = Kx[r] + t * (Kx[r - 1] - Kx[r])
            ksca[i] = Ks[r] + t * (Ks[r - 1] - Ks[r])
            kabs[i] = Ka[r] + t * (Ka[r - 1] - Ka[r])
            F[i] = M[r] + t * (M[r - 1] - M[r])
            i += 1
    if 0 < i < nlam:
        j = np.arange(i, nlam)
        ksca[j] = ksca[i - 1] * (lam[i - 1] / lam[j]) ** 4
        kabs[j] = kabs[i - 1] * (lam[i - 1] / lam[j]) ** 2
        kext[j] = kabs[j] + ksca[j]
        F[j] = F[i - 1]
    elif i == 0:
        raise ValueError("the wavelength grid starts above the table's range")
    s = np.sin(math.pi * (np.arange(1, NANG + 1) - 0.5) / 180.0)
    tot = (F[:, 0, :] * s).sum(1)
    F *= (s.sum() / tot)[:, None, None]
    if 0 < nspike < NANG:
        for j in range(nlam):
            lvl = F[j, 0, :nspike + 1].min() if spike == "min" else F[j, 0, nspike]
            f = lvl / F[j, 0, :nspike]
            F[j, 1:, :nspike] *= f[None, :]
            F[j, 0, :nspike] = lvl
            t = (F[j, 0] * s).sum()
            ksca[j] = ksca[j] * t / s.sum()
            kext[j] = kabs[j] + ksca[j]
            F[j] *= s.sum() / t
    if wasym2 != 0.0:
        th = (np.arange(1, NANG + 1) - 0.5) * math.pi / 180.0
        hg = np.array([hg_binned(asym2, x) for x in th])
        F[:, 0, :] = F[:, 0, :] * (1.0 - wasym2) + wasym2 * hg[None, :]
    return kext, kabs, ksca, F


def read_particle_fits(path, lam, matrix=None, nspike=0, wasym2=0.0, asym2=2.0):
    """ReadParticleFits: the file's opacities and matrices on the wavelength
    grid lam (see _regrid); matrix (6, 180), when given, replaces the file's
    at every wavelength (the Rayleigh / Henyey-Greenstein option, see
    rayleigh_hg_matrix); nspike, wasym2, asym2 as _regrid.  Returns dict(kabs, ksca, kext, F (nlam, 6, 180),
    rho_av, a1, a2, a3, rv [cm], amin, amax)."""
    (hdr, a), (_, m) = _read_hdus(_open(path))[:2]
    L, Kx, Ka, Ks = a
    M = m.transpose(2, 1, 0) if matrix is None else np.broadcast_to(matrix, (L.size, 6, NANG))
    kext, kabs, ksca, F = _regrid(L, Kx, Ka, Ks, M, lam, nspike, "min", 0.0 if matrix is not None else wasym2, asym2)
    a2 = float(hdr["A2"])
    return dict(kabs=kabs, ksca=ksca, kext=kext, F=F, rho_av=float(hdr["DENSITY"]), a1=float(hdr["A1"]), a2=a2,
                a3=float(hdr["A3"]), rv=math.sqrt(a2) * 1e-4, amin=float(hdr.get("R_MIN", float("nan"))),
                amax=float(hdr.get("R_MAX", float("nan"))))


def hg_binned(g, theta):
    """HG (Init.f:5594-5612): the Henyey-Greenstein phase function averaged
    with sin(t) weights over 1000 angles across the one-degree bin at theta,
    the offsets formed in single precision as there"""
    n = 1000
    i = np.arange(1, n + 1, dtype=np.float32)
    off = ((i - np.float32(1)) / np.float32(n - 1) - np.float32(0.5)) * np.float32(3.1415926536)
    t = theta + off.astype(np.float64) / 180.0
    f = (1.0 - g * g) / (1.0 - 2.0 * g * np.cos(t) + g * g) ** 1.5 / 2.0
    return float(np.sum(f * np.sin(t)) / np.sum(np.sin(t)))


def rayleigh_hg_matrix(asym=2.0, asym2=2.0, wasym2=0.0, pmax=1.0):
    """the matrix readparticle and ReadParticleFits put in place of a file's
    under scattype 'RAYLEIGH' (Init.f:4689-4707, ReadParticleFits.f:
    125-143): Henyey-Greenstein F11 (plus wasym2 of a second one) with a
    Rayleigh-shaped polarisation Pmax when |asym| < 1, else Rayleigh.
    Returns (6, 180)."""
    th = (np.arange(1, NANG + 1) - 0.5) * math.pi / 180.0
    c = np.cos(th)
    if -1.0 < asym < 1.0:
        F11 = np.array([hg_binned(asym, x) for x in th])
        if wasym2 != 0.0:
            F11 = F11 + wasym2 * np.array([hg_binned(asym2, x) for x in th])
        F12 = -pmax * F11 * (1.0 - c * c) / (1.0 + c * c)
    else:
        F11 = (1.0 + c * c) / 2.0
        F12 = -(1.0 - c * c) / 2.0
    return np.stack([F11, F12, F11, c * F11 / (1.0 + c * c), np.zeros(NANG), c * F11 / (1.0 + c * c)])


def rayleigh_matrix():
    """the scattering matrix readopacity gives a tabulated grain
    (Init.f:4920-4927): Rayleigh-like, (6, 180)"""
    th = (np.arange(1, NANG + 1) - 0.5) * math.pi / 180.0
    c = np.cos(th)
    return np.stack([(1 + c * c) / 2, -(1 - c * c) / 2, (1 + c * c) / 2, c, np.zeros(NANG), c])


def read_opacity_file(path, lam):
    """readopacity (Init.f:4886-4990): an ASCII table of wavelength
    [micron], Kext, Kabs, Ksca [cm^2/g] per line, with the Rayleigh-like
    matrix, on the wavelength grid lam.  Returns dict(kabs, ksca, kext, F)."""
    rows = []
    with open(path) as f:
        for line in f:
            parts = line.replace("d", "e").replace("D", "E").split()
            if len(parts) < 4:
                continue
            try:
                rows.append([float(x) for x in parts[:4]])
            except ValueError:
                continue
    if len(rows) < 2:
        raise ValueError("%s: fewer than two wavelengths" % path)
    t = np.array(rows)
    M = np.broadcast_to(rayleigh_matrix(), (t.shape[0], 6, NANG))
    kext, kabs, ksca, F = _regrid(t[:, 0], t[:, 1], t[:, 2], t[:, 3], M, lam)
    return dict(kabs=kabs, ksca=ksca, kext=kext, F=F)


def read_particle_ascii(path, lam, matrix=None, nspike=0, wasym2=0.0, asym2=2.0):
    """readparticle (Init.f:4664-4780): an ASCII particle file of records
    'wavelength Kext Kabs Ksca' followed by F11, F12, F22, F33, F34, F44 of
    180 values each.  As the reference's list-directed reads, every read
    starts on a new line and takes as many lines as its values need, the
    rest of its last line unread.  Regridded as _regrid; matrix as in
    read_particle_fits.  Returns dict(kabs, ksca, kext, F)."""
    with open(path) as f:
        lines = [ln.replace("d", "e").replace("D", "E").split() for ln in f]
    lines = [ln for ln in lines if ln]
    k = 0
    L, Kx, Ka, Ks, Ms = [], [], [], [], []
    while k < len(lines):
        head = lines[k]
        k += 1
        if len(head) < 4:
            break
        M6 = []
        for _ in range(6):
            vals = []
            while len(vals) < NANG and k < len(lines):
                vals += lines[k]
                k += 1
            if len(vals) < NANG:
                break
            M6.append([float(x) for x in vals[:NANG]])
        if len(M6) < 6:
            break
        L.append(float(head[0]))
        Kx.append(float(head[1]))
        Ka.append(float(head[2]))
        Ks.append(float(head[3]))
        Ms.append(M6)
    if len(L) < 1:
        raise ValueError("%s: no complete wavelength record" % path)
    Ms = np.array(Ms) if matrix is None else np.broadcast_to(matrix, (len(L), 6, NANG))
    kext, kabs, ksca, F = _regrid(np.array(L), np.array(Kx), np.array(Ka), np.array(Ks), Ms, lam, nspike, "next",
                                  0.0 if matrix is not None else wasym2, asym2)
    return dict(kabs=kabs, ksca=ksca, kext=kext, F=F)


def find_particle_file(particledir, ii, amin, amax, apow, ns, fmax, blend, porosity, frac, rho, lnkfiles, iopac=1,
                       abun_in_name=0):
    """The cache lookup: the first of particle0001 ... particleNNNN (ii),
    as .fits and then .fits.gz, whose keywords match; None if none does"""
    fr = np.asarray(frac, float)
    fr = fr / fr.sum()
    for k in range(1, ii + 1):
        for gz in (False, True):
            p = particle_file_name(particledir, k, iopac, fr, abun_in_name, gz)
            if os.path.exists(p) and check_particle_file(p, amin, amax, apow, ns, fmax, blend, porosity, fr, rho,
                                                         lnkfiles, checkfrac=abun_in_name <= 0):
                return p
    return None
