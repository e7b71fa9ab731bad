"""ctypes bindings of the CPU oracle (oracle/liboracle_mcmax.so).  Test
infrastructure only."""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "liboracle_mcmax.so")
TMAX = 10000
TT = TMAX + 1
AU = float(np.float32(1.49598e13))   # Modules.f:8, a single-precision literal
dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int32)
u8p = C.POINTER(C.c_uint8)


def P(a):
    if a is None:
        return None
    if a.dtype == np.float64:
        return a.ctypes.data_as(dp)
    if a.dtype == np.int32:
        return a.ctypes.data_as(ip)
    if a.dtype == np.uint8:
        return a.ctypes.data_as(u8p)
    raise TypeError(a.dtype)


class OrcModel(C.Structure):
    _fields_ = [("nr", C.c_int), ("nt", C.c_int), ("R", dp), ("Theta", dp), ("SinTheta", dp),
                ("dens", dp), ("V", dp), ("thick", u8p), ("nlam", C.c_int), ("lam", dp), ("nu", dp),
                ("KabsTot", dp), ("KscaTot", dp), ("KpCell", dp), ("kp_uniform", C.c_int), ("BB", dp), ("Fstar", dp),
                ("Lstar", C.c_double), ("ncomp", C.c_int), ("comp_w", dp), ("Ksca_comp", dp),
                ("F_comp", dp), ("IF_comp", dp), ("sinthet", dp), ("cos2phi", dp), ("sin2phi", dp),
                ("KDext", dp), ("KDabs", dp), ("g_comp", dp), ("rw_y", dp), ("rw_phi", dp)]


class OrcRun(C.Structure):
    _fields_ = [("nphot", C.c_int64), ("seed", C.c_uint64), ("scat_how", C.c_int), ("randomwalk", C.c_int),
                ("factRW", C.c_double), ("maxinteract", C.c_int64), ("rng", C.c_int), ("idum", C.c_int32)]


class OrcResult(C.Structure):
    _fields_ = [("EJv", dp), ("EJv2", dp), ("Eabs", dp), ("T", dp), ("Ni", ip), ("spec", dp),
                ("scatspec", dp), ("ispec", ip), ("counters", C.c_int64 * 16), ("tautot", C.c_double),
                ("Nabs", ip)]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_LIB):
            build()
        _lib = C.CDLL(ORACLE_LIB)
        _lib.orc_planck.restype = C.c_double
        _lib.orc_planck.argtypes = [C.c_double, C.c_double]
        _lib.orc_determine_t.restype = C.c_double
        _lib.orc_increase_t.restype = C.c_double
        _lib.orc_integrate.restype = C.c_double
        _lib.orc_ran1.restype = C.c_double
        for name in ("orc_determine_t", "orc_increase_t"):
            getattr(_lib, name).argtypes = [dp, C.c_double, C.c_double]
    return _lib


def dmilay(rcore, rshell, wvno, m_re, m_im, core_re=1.0, core_im=0.0, mu=None):
    L = load()
    if mu is None:
        mu = np.cos((np.arange(1, 91) - 0.5) / 90 * np.pi / 2)
    mu = np.ascontiguousarray(mu, float)
    n = mu.size
    m1, m2, s21, d21 = (np.zeros(2 * n) for _ in range(4))
    q = [C.c_double() for _ in range(4)]
    e = L.orc_dmilay(C.c_double(rcore), C.c_double(rshell), C.c_double(wvno), C.c_double(m_re),
                     C.c_double(m_im), C.c_double(core_re), C.c_double(core_im), P(mu), n,
                     *[C.byref(x) for x in q], P(m1), P(m2), P(s21), P(d21))
    return e, [x.value for x in q], (m1, m2, s21, d21)


def mie(rad, lam, e1, e2):
    L = load()
    f = [np.zeros(180) for _ in range(4)]
    cs, ce = C.c_double(), C.c_double()
    e = L.orc_meerhoff_mie(C.c_double(rad), C.c_double(lam), C.c_double(e1), C.c_double(e2), C.byref(cs),
                           C.byref(ce), *[P(x) for x in f], 180)
    return e, cs.value, ce.value, f


def blender(e1, e2, abun):
    L = load()
    a, b = C.c_double(), C.c_double()
    e1 = np.ascontiguousarray(e1, float)
    e2 = np.ascontiguousarray(e2, float)
    abun = np.ascontiguousarray(abun, float)
    L.orc_blender(P(e1), P(e2), P(abun), e1.size, C.byref(a), C.byref(b))
    return a.value, b.value


def compute_part(lam, e1, e2, frac, rho, amin, amax, apow, fmax, blend, porosity, ns, nf, normalize_abun=-1.0):
    L = load()
    lam = np.ascontiguousarray(lam, float)
    e1 = np.ascontiguousarray(np.atleast_2d(e1), float)
    e2 = np.ascontiguousarray(np.atleast_2d(e2), float)
    frac = np.ascontiguousarray(np.atleast_1d(frac), float)
    rho = np.ascontiguousarray(np.atleast_1d(rho), float)
    nlam = lam.size
    kabs, ksca, kext = np.zeros(nlam), np.zeros(nlam), np.zeros(nlam)
    F = np.zeros((nlam, 6, 180))
    rav, ms, rs = C.c_double(), C.c_double(), C.c_double()
    cnt = (C.c_int64 * 3)()
    st = L.orc_compute_part(nlam, P(lam), e1.shape[0], P(e1), P(e2), P(frac), P(rho), C.c_double(amin),
                            C.c_double(amax), C.c_double(apow), C.c_double(fmax), int(blend),
                            C.c_double(porosity), int(ns), int(nf), C.c_double(normalize_abun), P(kabs),
                            P(ksca), P(kext), P(F), C.byref(rav), C.byref(ms), C.byref(rs), cnt)
    assert st == 0
    return dict(kabs=kabs, ksca=ksca, kext=kext, F=F, rho_av=rav.value, mscale=ms.value, rscale=rs.value,
                n_dhs=cnt[0], n_mie=cnt[1], n_dhs_fail=cnt[2])


def bb_table(lam):
    L = load()
    lam = np.ascontiguousarray(lam, float)
    BB = np.zeros((lam.size, TT))
    L.orc_bb_table(lam.size, P(lam), P(BB))
    return BB


def transport_tables(model, randomwalk=False, factRW=10.0, lazy_kd=False):
    """Every table the oracle transport reads, built by the oracle's own
    table builders (Init.f / MCRadiation.f / Dtable.f restatements)."""
    L = load()
    m = model
    nlam, ncomp = m.nlam, m.ncomp
    ncell = m.ncell
    nu = np.ascontiguousarray(m.nu, float)
    BB = np.ascontiguousarray(m.BB, float)
    Kabs = np.ascontiguousarray(m.Kabs, float)
    Ksca = np.ascontiguousarray(m.Ksca, float)
    comp_w = np.ascontiguousarray(m.comp_w, float)
    Kp = np.zeros((ncomp, TT))
    L.orc_kp_table(nlam, P(nu), P(BB), ncomp, P(Kabs), P(Kp))
    KabsTot = np.zeros((ncell, nlam))
    KscaTot = np.zeros((ncell, nlam))
    uniform = bool(np.all(comp_w == comp_w[0]))
    KpCell = np.zeros((ncell, TT))
    if uniform:
        # one Planck-mean row serves every cell (identical mixtures)
        KpCell = np.zeros((1, TT))
        kt_a, kt_s = np.zeros((1, nlam)), np.zeros((1, nlam))
        L.orc_cell_tables(1, ncomp, nlam, P(comp_w), P(Kabs), P(Ksca), P(Kp), P(kt_a), P(kt_s), P(KpCell))
        KabsTot = np.ascontiguousarray(np.broadcast_to(kt_a, (ncell, nlam)))
        KscaTot = np.ascontiguousarray(np.broadcast_to(kt_s, (ncell, nlam)))
    else:
        L.orc_cell_tables(ncell, ncomp, nlam, P(comp_w), P(Kabs), P(Ksca), P(Kp), P(KabsTot), P(KscaTot), P(KpCell))
    sinthet = np.array([np.nan] * 180)
    cos2phi = np.zeros(361)
    sin2phi = np.zeros(361)
    L.orc_const_tables(P(sinthet), P(cos2phi), P(sin2phi))
    F = np.ascontiguousarray(m.F, float)
    IF = np.zeros((ncomp, nlam, 2))
    L.orc_if_table(ncomp * nlam, P(F), P(sinthet), P(IF))
    g = np.zeros((ncomp, nlam))
    L.orc_g_table(ncomp * nlam, P(F), P(g))
    rw_y, rw_phi = np.zeros(1000), np.zeros(1000)
    L.orc_rw_table(P(rw_y), P(rw_phi))
    out = dict(kp_uniform=int(uniform), Kp=Kp, KabsTot=KabsTot, KscaTot=KscaTot, KpCell=KpCell, sinthet=sinthet, cos2phi=cos2phi,
               sin2phi=sin2phi, IF=IF, g=g, rw_y=rw_y, rw_phi=rw_phi, thick=None, KDext=None, KDabs=None)
    if randomwalk and lazy_kd:
        # thick flags only; DiffCoeffCell is evaluated lazily inside the run
        thick = np.zeros(ncell, np.uint8)
        keep = [np.ascontiguousarray(a, float) for a in (m.R, m.Theta, m.SinTheta, m.dens, m.V, m.lam, m.BB, m.Fstar,
                                                         Ksca, m.F)]
        om = OrcModel(m.nr, m.nt, P(keep[0]), P(keep[1]), P(keep[2]), P(keep[3]), P(keep[4]), None, nlam,
                      P(keep[5]), P(nu), P(KabsTot), P(KscaTot), P(KpCell), int(uniform), P(keep[6]), P(keep[7]), float(m.Lstar),
                      ncomp, P(comp_w), P(keep[8]), P(keep[9]), P(IF), P(sinthet), P(cos2phi), P(sin2phi), None, None,
                      P(g), P(rw_y), P(rw_phi))
        L.orc_init_random_walk(C.byref(om), int(m.scat_how), C.c_double(factRW), P(thick))
        out.update(thick=thick)
    elif randomwalk:
        scattering = int(m.scat_how != 0 and np.any(KscaTot != 0))
        KDext = np.zeros((ncell, TT))
        KDabs = np.zeros((ncell, TT))
        thick = np.zeros(ncell, np.uint8)
        gcell = np.zeros(nlam)
        nc = m.nt - 1
        dens = np.asarray(m.dens, float)
        for c in range(ncell):
            i = c // nc
            L.orc_cell_g(ncomp, nlam, P(comp_w[c]), P(g), P(Ksca), P(KscaTot[c]), P(gcell))
            L.orc_diffcoeff_cell(nlam, P(nu), P(BB), P(KabsTot[c]), P(KscaTot[c]), P(gcell), scattering,
                                 P(KDext[c]), P(KDabs[c]))
            if i >= 1:
                for iT in (100, 600, 1100, 1600):
                    lr = 1.0 / ((AU * KDext[c, iT]) * dens[c])
                    if (m.R[i + 1] - m.R[i]) > factRW * lr:
                        thick[c] = 1
        out.update(KDext=KDext, KDabs=KDabs, thick=thick)
    return out


def mcradiation(model, nphot, seed=1, randomwalk=False, factRW=10.0, maxinteract=0, rng=0, idum=-42, tables=None):
    L = load()
    m = model
    t = tables or transport_tables(model, randomwalk, factRW)
    keep = {}

    def A(name, a, dt=np.float64):
        keep[name] = np.ascontiguousarray(a, dt)
        return P(keep[name])

    om = OrcModel(m.nr, m.nt, A("R", m.R), A("Theta", m.Theta), A("SinTheta", m.SinTheta), A("dens", m.dens),
                  A("V", m.V), A("thick", t["thick"], np.uint8) if t["thick"] is not None else None, m.nlam,
                  A("lam", m.lam), A("nu", m.nu), A("KabsTot", t["KabsTot"]), A("KscaTot", t["KscaTot"]),
                  A("KpCell", t["KpCell"]), int(t["kp_uniform"]), A("BB", m.BB), A("Fstar", m.Fstar), float(m.Lstar), m.ncomp,
                  A("comp_w", m.comp_w), A("Ksca", m.Ksca), A("F", m.F), A("IF", t["IF"]),
                  A("sinthet", t["sinthet"]), A("cos2phi", t["cos2phi"]), A("sin2phi", t["sin2phi"]),
                  A("KDext", t["KDext"]) if t["KDext"] is not None else None,
                  A("KDabs", t["KDabs"]) if t["KDabs"] is not None else None, A("g", t["g"]), A("rw_y", t["rw_y"]),
                  A("rw_phi", t["rw_phi"]))
    run = OrcRun(int(nphot), int(seed), int(m.scat_how), int(bool(randomwalk)), float(factRW), int(maxinteract),
                 int(rng), int(idum))
    nc = m.ncell
    ns = m.nlam * 31
    out = dict(EJv=np.zeros(nc), EJv2=np.zeros(nc), Eabs=np.zeros(nc), T=np.zeros(nc), Ni=np.zeros(nc, np.int32),
               spec=np.zeros(ns), scatspec=np.zeros(ns), ispec=np.zeros(ns, np.int32), Nabs=np.zeros(nc, np.int32))
    res = OrcResult(*[P(out[k]) for k in ("EJv", "EJv2", "Eabs", "T", "Ni", "spec", "scatspec", "ispec")])
    res.Nabs = P(out["Nabs"])
    st = L.orc_mcradiation(C.byref(om), C.byref(run), C.byref(res))
    out["status"] = st
    out["counters"] = np.array(res.counters[:], np.int64)
    out["tautot"] = res.tautot
    for k in ("spec", "scatspec", "ispec"):
        out[k] = out[k].reshape(m.nlam, 31)
    return out


def diffuse(model, tables, Ni, dT, T, nphotmin=25, dtmax=1.0):
    """orc_diffuse on (Ni, dT, T); tables from transport_tables(model,
    randomwalk=True) (KDext, thick).  Returns (T, EJv, thick, stats)."""
    L = load()
    m = model
    T = np.array(T, float)
    EJv = np.full(m.ncell, np.nan)
    thick = np.array(tables["thick"], np.uint8)
    stats = np.zeros(4, np.int32)
    Ni = np.ascontiguousarray(Ni, np.int32)
    dT = np.ascontiguousarray(dT, float)
    keep = [np.ascontiguousarray(a, float) for a in (m.R, m.Theta, m.dens, m.comp_w)]
    L.orc_diffuse(m.nr, m.nt, P(keep[0]), P(keep[1]), P(keep[2]), m.ncomp, P(keep[3]), P(tables["KDext"]),
                  P(tables["KpCell"]), int(tables["kp_uniform"]), P(thick), int(nphotmin), C.c_double(dtmax),
                  P(Ni), P(dT), P(T), P(EJv), P(stats))
    return T, EJv, thick, stats


def disk_structure(st, Temp, dens, dens0, gasdens, w, w0):
    """orc_disk_structure; arguments as hostcheck_ffi.disk_structure"""
    import hostcheck_ffi as H
    return H._structure_call(load().orc_disk_structure, st, Temp, dens, dens0, gasdens, w, w0)


class OrcScatOpts(C.Structure):
    _fields_ = [("nphot", C.c_int64), ("nstar", C.c_int64), ("seed", C.c_uint64), ("nexits", C.c_int)]


def _trace_model(m, T, dens, scatter):
    """the orc_model of the ray tracer (with the Mueller tables when a
    scattered-light field is asked for) and the arrays it points into"""
    dens = np.maximum(np.asarray(m.dens, float), 1e-50) if dens is None else np.asarray(dens, float)
    keep = [np.ascontiguousarray(a, float) for a in (m.R, m.Theta, m.SinTheta, dens, m.V, m.lam, m.nu, m.BB, m.Fstar,
                                                     m.comp_w, m.Kabs, m.Ksca, T)]
    if scatter:
        t = transport_tables(m)
        more = [np.ascontiguousarray(a, float) for a in (m.F, t["IF"], t["sinthet"], t["cos2phi"], t["sin2phi"])]
        keep += more
        om = OrcModel(m.nr, m.nt, P(keep[0]), P(keep[1]), P(keep[2]), P(keep[3]), P(keep[4]), None, m.nlam,
                      P(keep[5]), P(keep[6]), None, None, None, 0, P(keep[7]), P(keep[8]), float(m.Lstar), m.ncomp,
                      P(keep[9]), P(keep[11]), P(more[0]), P(more[1]), P(more[2]), P(more[3]), P(more[4]), None, None,
                      None, None, None)
        so = OrcScatOpts(int(scatter.get("nphot", 0)), int(scatter.get("nphot_star", 0)),
                         int(scatter.get("seed", 1)) & (2 ** 64 - 1), int(scatter.get("nexits", 5)))
    else:
        om = OrcModel(m.nr, m.nt, P(keep[0]), P(keep[1]), P(keep[2]), P(keep[3]), P(keep[4]), None, m.nlam,
                      P(keep[5]), P(keep[6]), None, None, None, 0, P(keep[7]), P(keep[8]), float(m.Lstar), m.ncomp,
                      P(keep[9]), None, None, None, None, None, None, None, None, None, None, None)
        so = None
    return om, so, keep


def trace_spectrum(model, T, lam_obs, angle, nphi=45, nj0=2, Rfix=(), lam_path=0.55, tracestar=1, dimstar=1.0,
                   dens=None, scatter=None):
    """orc_trace_spectrum (orc_trace_spectrum_scat with a scattered-light
    field: scatter = dict(nphot, nphot_star, seed, nexits)); returns (flux,
    image radii count, bad rays)"""
    L = load()
    m = model
    om, so, keep = _trace_model(m, T, dens, scatter)
    lam_obs = np.ascontiguousarray(lam_obs, float)
    Rfix = np.ascontiguousarray(Rfix, float)
    flux = np.zeros(lam_obs.size)
    info = np.zeros(2, np.int32)
    args = [C.byref(om), P(keep[10]), P(keep[11]), P(keep[12]), int(m.scat_how), C.c_double(angle),
            int(nphi), int(nj0), int(Rfix.size), P(Rfix) if Rfix.size else None, C.c_double(lam_path),
            int(tracestar), C.c_double(dimstar), int(lam_obs.size), P(lam_obs), P(flux), P(info)]
    if so is None:
        L.orc_trace_spectrum(*args)
    else:
        L.orc_trace_spectrum_scat(*args, C.byref(so))
    return flux, int(info[0]), int(info[1])


def trace_image(model, T, lam0, angle, npix, nint, Rmax, pa=0.0, seed=42, linear=0, nphi=45, nj0=2, Rfix=(),
                tracestar=1, dimstar=1.0, dens=None, scatter=None):
    """orc_trace_image (orc_trace_image_scat with a scattered-light field);
    returns (image (npix, npix), flux, image radii, bad rays)"""
    L = load()
    m = model
    om, so, keep = _trace_model(m, T, dens, scatter)
    Rfix = np.ascontiguousarray(Rfix, float)
    flux = np.zeros(1)
    im = np.zeros(npix * npix)
    info = np.zeros(2, np.int32)
    args = [C.byref(om), P(keep[10]), P(keep[11]), P(keep[12]), int(m.scat_how), C.c_double(angle),
            int(nphi), int(nj0), int(Rfix.size), P(Rfix) if Rfix.size else None, int(tracestar),
            C.c_double(dimstar), C.c_double(lam0), int(npix), int(nint), C.c_double(Rmax), C.c_double(pa),
            C.c_uint64(seed), int(linear), P(flux), P(im), P(info)]
    if so is None:
        L.orc_trace_image(*args)
    else:
        L.orc_trace_image_scat(*args, C.byref(so))
    return im.reshape(npix, npix), float(flux[0]), int(info[0]), int(info[1])


def scatter_field(model, T, lam0, angle, nphot=1000, nphot_star=1000, seed=1, nexits=5, tables=None):
    """orc_scatter_field: the ray tracer's scattered-light field at lam0
    [micron] for inclination angle [rad]; returns (field (nr, nsub, 2, 91),
    info [nsub, geometry failures, interaction-cap kills, no start])"""
    L = load()
    m = model
    t = tables or transport_tables(model)
    keep = {}

    def A(name, a, dt=np.float64):
        keep[name] = np.ascontiguousarray(a, dt)
        return P(keep[name])

    om = OrcModel(m.nr, m.nt, A("R", m.R), A("Theta", m.Theta), A("SinTheta", m.SinTheta),
                  A("dens", np.maximum(np.asarray(m.dens, float), 1e-50)), A("V", m.V), None, m.nlam,
                  A("lam", m.lam), A("nu", m.nu), A("KabsTot", t["KabsTot"]), A("KscaTot", t["KscaTot"]),
                  A("KpCell", t["KpCell"]), int(t["kp_uniform"]), A("BB", m.BB), A("Fstar", m.Fstar), float(m.Lstar),
                  m.ncomp, A("comp_w", m.comp_w), A("Ksca", m.Ksca), A("F", m.F), A("IF", t["IF"]),
                  A("sinthet", t["sinthet"]), A("cos2phi", t["cos2phi"]), A("sin2phi", t["sin2phi"]), None, None,
                  A("g", t["g"]), A("rw_y", t["rw_y"]), A("rw_phi", t["rw_phi"]))
    nc = m.nt - 1
    th = np.arccos(np.asarray(m.Theta, float))
    th[0], th[-1] = 0.0, np.pi / 2
    if int(m.scat_how) == 2:
        nrg = [max(1, int((th[j] - th[j - 1]) * 270.0 / np.pi)) for j in range(1, nc + 1)]
    else:
        nrg = [1] * nc
    nsub = int(sum(nrg))
    SF = np.zeros(m.nr * nsub * 2 * 91)
    info = np.zeros(4, np.int64)
    st = L.orc_scatter_field(C.byref(om), A("Kabs_c", m.Kabs), A("Ksca_c", m.Ksca), A("T", T), int(m.scat_how),
                             C.c_double(angle), C.c_double(lam0), C.c_int64(int(nphot)), C.c_int64(int(nphot_star)),
                             C.c_uint64(int(seed) & (2 ** 64 - 1)), int(nexits), P(SF),
                             info.ctypes.data_as(C.POINTER(C.c_int64)))
    assert st == 0 and int(info[0]) == nsub
    return SF.reshape(m.nr, nsub, 2, 91), info
