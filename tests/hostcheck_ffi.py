"""ctypes bindings of tests/native/libhostcheck.so: the device cores built
for the host (test infrastructure only)."""
import ctypes as C
import os
import subprocess

import numpy as np

from oracle_ffi import P, dp

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "native", "hostcheck.cpp")
LIB = os.path.join(HERE, "native", "libhostcheck.so")
DEPS = [SRC] + [os.path.join(HERE, "..", "mcmax_b200", "csrc", f) for f in
                ("dhs_core.cuh", "transport_core.cuh", "transport_fast.cuh", "diffuse_core.cuh", "dstruct_core.cuh",
                 "rt_core.cuh", "surrogate_phase.h", "detmath.h", "cplx.h", "philox.h")]


class HcModel(C.Structure):
    _fields_ = [("nr", C.c_int), ("nt", C.c_int), ("nlam", C.c_int), ("ncomp", C.c_int), ("scat_how", C.c_int),
                ("uniform_mix", C.c_int), ("rw", C.c_int), ("factRW", C.c_double), ("Lstar", C.c_double),
                ("nphot", C.c_int64), ("maxinteract", C.c_int64), ("seed", C.c_uint64)] + \
               [(n, dp) for n in ("R", "Theta", "SinTheta", "dens", "V", "nu", "BB", "Fstar", "KabsTot", "KscaTot",
                                  "KpCell", "comp_w", "Ksca_c", "F_c", "IF_c", "sinthet", "cos2phi", "sin2phi",
                                  "KDext", "KDabs", "rw_y", "rw_phi")] + [("thick", C.POINTER(C.c_uint8))]


_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(d) for d in DEPS):
            subprocess.run(["g++", "-O2", "-fPIC", "-shared", "-std=c++17", "-ffp-contract=off", "-fno-fast-math",
                            "-o", LIB, SRC], check=True)
        _lib = C.CDLL(LIB)
    return _lib


def dhs_sample(rcore, rshell, wvno, mre, mim, mu):
    L = load()
    F = np.zeros(720)
    ce, cs = C.c_double(), C.c_double()
    mu = np.ascontiguousarray(mu, float)
    e = L.hc_dhs_sample(C.c_double(rcore), C.c_double(rshell), C.c_double(wvno), C.c_double(mre), C.c_double(mim),
                        P(mu), P(F), C.byref(ce), C.byref(cs))
    return e, ce.value, cs.value, F.reshape(4, 180)


def mie_sample(rad, lam, e1, e2):
    L = load()
    F = np.zeros(720)
    cs, ce = C.c_double(), C.c_double()
    e = L.hc_mie_sample(C.c_double(rad), C.c_double(lam), C.c_double(e1), C.c_double(e2), P(F), C.byref(cs),
                        C.byref(ce))
    return e, cs.value, ce.value, F.reshape(4, 180)


def mcradiation(model, tables, nphot, seed=1, randomwalk=False, factRW=10.0, maxinteract=0, fast=None, first=0,
                count=None, inflight=1):
    """Serial host replay of the device packet loop.  fast=None: the
    reference-order kernel; fast='fp64' / 'mixed': the GPU-ordered kernel
    (uniform mixtures), packets [first, first+count); with inflight > 1 that
    many packets advance one event at a time in turn (a GPU launch's
    concurrency)."""
    L = load()
    m, t = model, tables
    keep = {}

    def A(name, a, dt=np.float64):
        if a is None:
            return None
        keep[name] = np.ascontiguousarray(a, dt)
        return P(keep[name])

    uniform = int(all(np.array_equal(m.comp_w[0], m.comp_w[c]) for c in range(m.ncell)))
    h = HcModel(m.nr, m.nt, m.nlam, m.ncomp, int(m.scat_how), uniform, int(bool(randomwalk)), float(factRW),
                float(m.Lstar), int(nphot), int(maxinteract), int(seed),
                A("R", m.R), A("Theta", m.Theta), A("SinTheta", m.SinTheta), A("dens", m.dens), A("V", m.V),
                A("nu", m.nu), A("BB", m.BB), A("Fstar", m.Fstar), A("KabsTot", t["KabsTot"]),
                A("KscaTot", t["KscaTot"]), A("KpCell", t["KpCell"]), A("comp_w", m.comp_w), A("Ksca", m.Ksca),
                A("F", m.F), A("IF", t["IF"]), A("sinthet", t["sinthet"]), A("cos2phi", t["cos2phi"]),
                A("sin2phi", t["sin2phi"]), A("KDext", t["KDext"]), A("KDabs", t["KDabs"]), A("rw_y", t["rw_y"]),
                A("rw_phi", t["rw_phi"]), A("thick", t["thick"], np.uint8))
    nc = m.ncell
    ns = m.nlam * 31
    out = dict(EJv=np.zeros(nc), EJv2=np.zeros(nc), Eabs=np.zeros(nc), T=np.zeros(nc), Ni=np.zeros(nc, np.int32),
               spec=np.zeros(ns), scatspec=np.zeros(ns), ispec=np.zeros(ns, np.int32), Nabs=np.zeros(nc, np.int32))
    cnt = (C.c_ulonglong * 16)()
    tau = C.c_double(0.0)
    if fast is not None and inflight > 1:
        L.hc_fast_interleaved(C.byref(h), int(fast == "mixed"),
                              *[P(out[k]) for k in ("EJv", "EJv2", "Eabs", "T", "Ni", "spec")], cnt, C.byref(tau),
                              int(inflight), P(out["Nabs"]))
    elif fast is None:
        L.hc_mcradiation(C.byref(h), *[P(out[k]) for k in ("EJv", "EJv2", "Eabs", "T", "Ni", "spec", "scatspec",
                                                           "ispec")], cnt, C.byref(tau))
    else:
        L.hc_fast(C.byref(h), int(fast == "mixed"), *[P(out[k]) for k in ("EJv", "EJv2", "Eabs", "T", "Ni", "spec")],
                  cnt, C.byref(tau), C.c_int64(first), C.c_int64(nphot if count is None else count))
    out["counters"] = np.array(cnt[:], np.int64)
    out["tautot"] = tau.value
    for k in ("spec", "scatspec", "ispec"):
        out[k] = out[k].reshape(m.nlam, 31)
    return out


class HcDiffuseTables(C.Structure):
    _fields_ = [("nlam", C.c_int), ("ncomp", C.c_int), ("scattering", C.c_int), ("uniform_mix", C.c_int)] + \
               [(n, dp) for n in ("comp_w", "g_c", "Ksca_c", "KabsTot", "KscaTot", "nu", "BB", "KpCell")]


def diffuse(model, tables, Ni, dT, T, nphotmin=25, dtmax=1.0, factRW=10.0):
    """the host logic of mcg_diffuse with serial loops in place of its
    kernels; returns (T, EJv, stats [selected, unknowns, solved, failed
    passes, box rows, half-bandwidth])"""
    L = load()
    m = model
    arrs = [np.ascontiguousarray(a, float) for a in (m.comp_w, tables["g"], m.Ksca, tables["KabsTot"],
                                                     tables["KscaTot"], m.nu, m.BB, tables["KpCell"])]
    scattering = int(m.scat_how != 0 and np.any(np.asarray(tables["KscaTot"]) != 0))
    t = HcDiffuseTables(m.nlam, m.ncomp, scattering, int(tables["kp_uniform"]), *[P(a) for a in arrs])
    T = np.array(T, float)
    EJv = np.full(m.ncell, np.nan)
    stats = np.zeros(6, np.int32)
    geo = [np.ascontiguousarray(a, float) for a in (m.R, m.Theta, m.dens)]
    L.hc_diffuse(m.nr, m.nt, P(geo[0]), P(geo[1]), P(geo[2]), C.byref(t), int(nphotmin), C.c_double(dtmax),
                 C.c_double(factRW), P(np.ascontiguousarray(Ni, np.int32)), P(np.ascontiguousarray(dT, float)), P(T),
                 P(EJv), P(stats))
    return T, EJv, stats


def band_solve(nb, w, coef, rhs):
    L = load()
    x = np.zeros(nb)
    code = L.hc_band_solve(int(nb), int(w), P(np.ascontiguousarray(coef, float)), P(np.ascontiguousarray(rhs, float)),
                           P(x))
    return code, x


def _structure_call(fn, st, Temp, dens, dens0, gasdens, w, w0):
    """st: dict(nr, nt, ng, R, Theta, V, Mstar, zones [(rin, rout, sh, rsh,
    shpow, denspow, fix)], shscale, grain_scale, shtype (ng codes)).
    Returns the updated (dens, dens0, gasdens, w, w0)."""
    out = [np.array(a, dtype=np.float64) for a in (dens, dens0, gasdens, w, w0)]
    zones = np.ascontiguousarray(np.array(st.get("zones", []), dtype=np.float64).reshape(-1))
    arrs = [np.ascontiguousarray(st[k], float) for k in ("R", "Theta", "V")]
    sh = None if st.get("shscale") is None else np.ascontiguousarray(st["shscale"], float)
    gs = None if st.get("grain_scale") is None else np.ascontiguousarray(st["grain_scale"], float)
    sht = None if st.get("shtype") is None else np.ascontiguousarray(st["shtype"], np.int32)
    rc = fn(int(st["nr"]), int(st["nt"]), int(st["ng"]), P(arrs[0]), P(arrs[1]), P(arrs[2]), C.c_double(st["Mstar"]),
            len(st.get("zones", [])), P(zones) if zones.size else None, P(sh), P(gs), P(sht),
            P(np.ascontiguousarray(Temp, float)), *[P(a) for a in out])
    assert rc == 0
    return tuple(out)


def disk_structure(st, Temp, dens, dens0, gasdens, w, w0):
    return _structure_call(load().hc_disk_structure, st, Temp, dens, dens0, gasdens, w, w0)


def trace_spectrum(model, T, lam_obs, angle, nphi=45, nj0=2, Rfix=(), lam_path=0.55, tracestar=1, dimstar=1.0,
                   dens=None, cap=20000):
    """the host logic of mcg_trace_spectrum with its kernels as loops;
    returns (flux, R_image, image (nr, nphi) of the last wavelength, bad rays)"""
    L = load()
    m = model
    dens = np.maximum(np.asarray(m.dens, float), 1e-50) if dens is None else np.asarray(dens, float)
    arrs = [np.ascontiguousarray(a, float) for a in (m.R, m.Theta, dens, m.comp_w, m.Kabs, m.Ksca, m.BB, m.lam,
                                                     m.Fstar, T)]
    lam_obs = np.ascontiguousarray(lam_obs, float)
    Rfix = np.ascontiguousarray(Rfix, float)
    flux = np.zeros(lam_obs.size)
    info = np.zeros(2, np.int32)
    Rimg = np.zeros(cap)
    image = np.zeros(cap * nphi)
    rc = L.hc_trace_spectrum(m.nr, m.nt, P(arrs[0]), P(arrs[1]), P(arrs[2]), int(m.scat_how), m.ncomp, m.nlam,
                             P(arrs[3]), P(arrs[4]), P(arrs[5]), P(arrs[6]), P(arrs[7]), P(arrs[8]), P(arrs[9]),
                             C.c_double(angle), int(nphi), int(nj0), int(Rfix.size), P(Rfix) if Rfix.size else None,
                             C.c_double(lam_path), int(tracestar), C.c_double(dimstar), int(lam_obs.size), P(lam_obs),
                             P(flux), P(info), P(Rimg), int(cap), P(image))
    assert rc == 0
    nr = int(info[0])
    return flux, Rimg[:nr], image[:nr * nphi].reshape(nr, nphi), int(info[1])


def trace_image(model, T, lam0, angle, npix, nint, Rmax, pa=0.0, seed=42, linear=0, nphi=45, nj0=2, Rfix=(),
                tracestar=1, dimstar=1.0, dens=None):
    """the host logic of mcg_trace_image with its kernels as one loop over
    the points; returns (image (npix, npix), flux, image radii, bad rays)"""
    L = load()
    m = model
    dens = np.maximum(np.asarray(m.dens, float), 1e-50) if dens is None else np.asarray(dens, float)
    arrs = [np.ascontiguousarray(a, float) for a in (m.R, m.Theta, dens, m.comp_w, m.Kabs, m.Ksca, m.BB, m.lam,
                                                     m.Fstar, T)]
    Rfix = np.ascontiguousarray(Rfix, float)
    flux = np.zeros(1)
    im = np.zeros(npix * npix)
    info = np.zeros(2, np.int32)
    rc = L.hc_trace_image(m.nr, m.nt, P(arrs[0]), P(arrs[1]), P(arrs[2]), int(m.scat_how), m.ncomp, m.nlam,
                          P(arrs[3]), P(arrs[4]), P(arrs[5]), P(arrs[6]), P(arrs[7]), P(arrs[8]), P(arrs[9]),
                          C.c_double(angle), int(nphi), int(nj0), int(Rfix.size), P(Rfix) if Rfix.size else None,
                          int(tracestar), C.c_double(dimstar), C.c_double(lam0), int(npix), int(nint),
                          C.c_double(Rmax), C.c_double(pa), C.c_ulonglong(seed), int(linear), P(flux), P(im), P(info))
    assert rc == 0
    return im.reshape(npix, npix), float(flux[0]), int(info[0]), int(info[1])


def surr_phase(chi, beta, gam, delta, deltam=1):
    """surrogate_phase.h: the Mueller matrix (6, 180) from Legendre moments"""
    L = load()
    a = [np.ascontiguousarray(x, float) for x in (chi, beta, gam, delta)]
    F = np.zeros(6 * 180)
    L.hc_surr_phase(P(a[0]), P(a[1]), P(a[2]), P(a[3]), int(deltam), P(F))
    return F.reshape(6, 180)
