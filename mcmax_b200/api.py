"""Python host mirror of the two MCMax entry points the library replaces.

    ComputePart(p, ii, input, amin, amax, apow, fmax, blend, porosity,
                inp_abun, iopac, normalize_abun, standard, nsubgrains)
        ComputePart.f:1 -- fills p.Kabs/Ksca/Kext[iopac], p.F[iopac],
        p.rho[iopac], p.mscale/rscale[iopac] from a particle file.

    MCRadiation(model, NphotTot, niter, dofastvisc)
        MCRadiation.f:6 -- runs the photon-packet loop on the model's grid and
        opacities and stores EJv/EJv2/Eabs/Ni/T and the MC spectra in the
        model; returns NphotTot (in/out in the reference).

Both go through libmcmax_gpu.so (include/mcmax_gpu.h); errors raise McgError
with the library's message, the counterpart of the reference's `stop`.
"""
import ctypes as C
import math
import os

import numpy as np

from . import _ffi
from ._ffi import TT, NANG


class McgError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (_ffi.STATUS_NAMES.get(status, status), msg))
        self.status = status


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Context:
    """One library context on one CUDA device."""

    def __init__(self, device=0):
        self.lib = _ffi.load()
        h = C.c_void_p()
        st = self.lib.mcg_create(C.byref(h), int(device))
        if st != 0:
            raise McgError(st, "mcg_create(device=%d) failed" % device)
        self.h = h
        self._keep = []

    def close(self):
        if getattr(self, "h", None):
            self.lib.mcg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != 0:
            raise McgError(st, self.lib.mcg_last_error(self.h).decode())

    # ------------------------------------------------------------ opacities
    def compute_part_batch(self, parts):
        """parts: list of dicts with lam, e1, e2 (nm x nlam), frac, rho, amin,
        amax, apow, fmax, porosity, blend, ns, nf, normalize_abun.  Returns a
        list of dicts with kabs, ksca, kext, F (nlam,6,180), rho_av, mscale,
        rscale and the evaluation counters."""
        n = len(parts)
        ins = (_ffi.PartIn * n)()
        outs = (_ffi.PartOut * n)()
        keep, res = [], []
        for k, p in enumerate(parts):
            lam = _f64(p["lam"])
            e1 = _f64(np.atleast_2d(p["e1"]))
            e2 = _f64(np.atleast_2d(p["e2"]))
            frac = _f64(np.atleast_1d(p["frac"]))
            rho = _f64(np.atleast_1d(p["rho"]))
            nlam = lam.size
            o = dict(kabs=np.zeros(nlam), ksca=np.zeros(nlam), kext=np.zeros(nlam),
                     F=np.zeros((nlam, 6, NANG)))
            keep += [lam, e1, e2, frac, rho]
            ins[k] = _ffi.PartIn(nlam, _ffi.ptr(lam), e1.shape[0], _ffi.ptr(e1), _ffi.ptr(e2),
                                 _ffi.ptr(frac), _ffi.ptr(rho), float(p["amin"]), float(p["amax"]),
                                 float(p["apow"]), float(p["fmax"]), float(p.get("porosity", 0.0)),
                                 float(p.get("normalize_abun", -1.0)), int(bool(p.get("blend", False))),
                                 int(p["ns"]), int(p["nf"]))
            outs[k].kabs = _ffi.ptr(o["kabs"])
            outs[k].ksca = _ffi.ptr(o["ksca"])
            outs[k].kext = _ffi.ptr(o["kext"])
            outs[k].F = _ffi.ptr(o["F"])
            res.append(o)
        self._check(self.lib.mcg_compute_part_batch(self.h, n, ins, outs))
        for k, o in enumerate(res):
            o.update(rho_av=outs[k].rho_av, mscale=outs[k].mscale, rscale=outs[k].rscale,
                     n_dhs=outs[k].n_dhs, n_mie=outs[k].n_mie, n_dhs_fail=outs[k].n_dhs_fail)
        return res

    # ------------------------------------------------------------ transport
    def set_model(self, model):
        """Upload a model (see mcmax_b200.model.Model) and build the device
        tables."""
        m = model
        arrs = dict(R=_f64(m.R), Theta=_f64(m.Theta), SinTheta=_f64(m.SinTheta), dens=_f64(m.dens),
                    V=_f64(m.V), comp_w=_f64(m.comp_w), lam=_f64(m.lam), nu=_f64(m.nu),
                    Kabs=_f64(m.Kabs), Ksca=_f64(m.Ksca), F=_f64(m.F) if m.F is not None else None,
                    BB=_f64(m.BB), Fstar=_f64(m.Fstar))
        self._model_arrays = arrs
        g = _ffi.Grid(m.nr, m.nt, _ffi.ptr(arrs["R"]), _ffi.ptr(arrs["Theta"]), _ffi.ptr(arrs["SinTheta"]),
                      _ffi.ptr(arrs["dens"]), _ffi.ptr(arrs["V"]), m.ncomp, _ffi.ptr(arrs["comp_w"]))
        o = _ffi.Opacity(m.nlam, _ffi.ptr(arrs["lam"]), _ffi.ptr(arrs["nu"]), m.ncomp, _ffi.ptr(arrs["Kabs"]),
                         _ffi.ptr(arrs["Ksca"]), _ffi.ptr(arrs["F"]), _ffi.ptr(arrs["BB"]),
                         _ffi.ptr(arrs["Fstar"]), float(m.Lstar), float(m.Tstar), float(m.Rstar_cm),
                         int(m.scat_how))
        self._check(self.lib.mcg_set_model(self.h, C.byref(g), C.byref(o)))
        self.model = m

    def mcradiation(self, nphot, seed=1, randomwalk=False, factRW=10.0, maxinteract=0, nruns=1,
                    precision="exact", threads=0, block=0, fetch=True, maxruntime=-1.0, t4_single=False):
        """Run the packet loop; returns (nphot_out, result dict).  nphot_out
        is smaller than nphot when maxruntime (seconds, > 0) cut the run.
        t4_single: the temperature interpolations in the reference's single
        precision (mcg_run.t4_single)."""
        m = self.model
        prec = {"fp64": _ffi.PREC_FP64, "mixed": _ffi.PREC_MIXED, "exact": _ffi.PREC_EXACT}[precision]
        run = _ffi.Run(int(seed), int(bool(randomwalk)), float(factRW), int(maxinteract), int(nruns), prec,
                       int(threads), int(block), float(maxruntime), int(bool(t4_single)))
        out = {}
        res = _ffi.Result()
        if fetch:
            nc = m.ncell
            ns = m.nlam * (_ffi.NANGLE_SED + 1)
            out = dict(EJv=np.zeros(nc), EJv2=np.zeros(nc), Eabs=np.zeros(nc), T=np.zeros(nc),
                       Ni=np.zeros(nc, np.int32), spec=np.zeros(ns), scatspec=np.zeros(ns),
                       ispec=np.zeros(ns, np.int32), Nabs=np.zeros(nc, np.int32))
            for k, v in out.items():
                setattr(res, k, _ffi.ptr(v))
        n = C.c_int64(int(nphot))
        self._check(self.lib.mcg_mcradiation(self.h, C.byref(run), C.byref(n), C.byref(res)))
        out["counters"] = np.array(res.counters[:], dtype=np.int64)
        out["tautot"] = res.tautot
        out["device_ms"] = res.device_ms
        out["progress_ms"] = list(res.progress_ms)
        if fetch:
            for k in ("spec", "scatspec", "ispec"):
                out[k] = out[k].reshape(m.nlam, _ffi.NANGLE_SED + 1)
        return n.value, out

    def _grid_opacity(self, m):
        arrs = dict(R=_f64(m.R), Theta=_f64(m.Theta), SinTheta=_f64(m.SinTheta), dens=_f64(m.dens),
                    V=_f64(m.V), comp_w=_f64(m.comp_w), lam=_f64(m.lam), nu=_f64(m.nu),
                    Kabs=_f64(m.Kabs), Ksca=_f64(m.Ksca), F=_f64(m.F) if m.F is not None else None,
                    BB=_f64(m.BB), Fstar=_f64(m.Fstar))
        g = _ffi.Grid(m.nr, m.nt, _ffi.ptr(arrs["R"]), _ffi.ptr(arrs["Theta"]), _ffi.ptr(arrs["SinTheta"]),
                      _ffi.ptr(arrs["dens"]), _ffi.ptr(arrs["V"]), m.ncomp, _ffi.ptr(arrs["comp_w"]))
        o = _ffi.Opacity(m.nlam, _ffi.ptr(arrs["lam"]), _ffi.ptr(arrs["nu"]), m.ncomp, _ffi.ptr(arrs["Kabs"]),
                         _ffi.ptr(arrs["Ksca"]), _ffi.ptr(arrs["F"]), _ffi.ptr(arrs["BB"]),
                         _ffi.ptr(arrs["Fstar"]), float(m.Lstar), float(m.Tstar), float(m.Rstar_cm),
                         int(m.scat_how))
        return arrs, g, o

    def add_model(self, model):
        """Keep a model on the device for batched runs; returns its id."""
        arrs, g, o = self._grid_opacity(model)
        mid = C.c_int(-1)
        self._check(self.lib.mcg_add_model(self.h, C.byref(g), C.byref(o), C.byref(mid)))
        if not hasattr(self, "kept"):
            self.kept = {}
        self.kept[mid.value] = model
        return mid.value

    def mcradiation_batch(self, ids, nphot, seeds, precision="mixed", randomwalk=False, factRW=10.0,
                          maxinteract=0, threads=0, block=0, blocks_per_sm=0, chunk=0, autotune=False,
                          use_graph=False, fetch=True):
        """One launch over kept models ids[k] with nphot[k] packets and seed
        seeds[k]; returns (nphot_out, results, launch info)."""
        n = len(ids)
        prec = {"fp64": _ffi.PREC_FP64, "mixed": _ffi.PREC_MIXED}[precision]
        runs = (_ffi.Run * n)()
        for k in range(n):
            runs[k] = _ffi.Run(int(seeds[k]), int(bool(randomwalk)), float(factRW), int(maxinteract), 1, prec,
                               int(threads), 0)
        cids = (C.c_int * n)(*[int(i) for i in ids])
        cn = (C.c_int64 * n)(*[int(x) for x in nphot])
        res = (_ffi.Result * n)()
        outs = []
        kept = getattr(self, "kept", {})
        for k in range(n):
            m = kept.get(ids[k])
            out = {}
            if fetch and m is not None:
                nc = m.ncell
                ns = m.nlam * (_ffi.NANGLE_SED + 1)
                out = dict(EJv=np.zeros(nc), EJv2=np.zeros(nc), Eabs=np.zeros(nc), T=np.zeros(nc),
                           Ni=np.zeros(nc, np.int32), spec=np.zeros(ns), scatspec=np.zeros(ns),
                           ispec=np.zeros(ns, np.int32))
                for key, v in out.items():
                    setattr(res[k], key, _ffi.ptr(v))
            outs.append(out)
        opts = _ffi.BatchOpts(int(block), int(blocks_per_sm), int(chunk), int(bool(autotune)), int(bool(use_graph)),
                              0.0)
        self._check(self.lib.mcg_mcradiation_batch(self.h, n, cids, runs, cn, res, C.byref(opts)))
        for k in range(n):
            outs[k]["counters"] = np.array(res[k].counters[:], dtype=np.int64)
            outs[k]["tautot"] = res[k].tautot
            if fetch:
                m = kept[ids[k]]
                for key in ("spec", "scatspec", "ispec"):
                    outs[k][key] = outs[k][key].reshape(m.nlam, _ffi.NANGLE_SED + 1)
        info = dict(block=opts.block, blocks_per_sm=opts.blocks_per_sm, chunk=opts.chunk, device_ms=opts.device_ms)
        return list(cn), outs, info

    def finalize_t(self):
        nc = self.model.ncell
        T, dT, dE = np.zeros(nc), np.zeros(nc), np.zeros(nc)
        self._check(self.lib.mcg_finalize_t(self.h, _ffi.ptr(T), _ffi.ptr(dT), _ffi.ptr(dE)))
        return T, dT, dE

    @staticmethod
    def _trace_opts(angle, nphi, nr, Rfix, lam_path, tracestar, dimstar, scatter):
        sc = dict(nphot=0, nphot_star=0, seed=1, nexits=5)
        sc.update(scatter or {})
        return _ffi.TraceOpts(float(angle), int(nphi), int(nr), int(Rfix.size), _ffi.ptr(Rfix) if Rfix.size else None,
                              float(lam_path), int(bool(tracestar)), float(dimstar), int(sc["nphot"]),
                              int(sc["nphot_star"]), int(sc["seed"]) & (2 ** 64 - 1), int(sc["nexits"]))

    def trace_spectrum(self, T, lam_obs, angle, nphi=45, nr=2, Rfix=(), lam_path=0.55, tracestar=True,
                       dimstar=1.0, scatter=None):
        """mcg_trace_spectrum on the current model: the ray-traced flux at
        inclination `angle` [rad] for each wavelength of lam_obs, from the
        cell temperatures T.  scatter: the scattered-light field's
        settings, dict(nphot, nphot_star, seed, nexits) (an observation's
        defaults are 1000, 1000, -, 5; None or both counts 0: no scattered
        light).  Returns (flux, info) with flux in the reference's units
        (x 1e23 / distance^2 for Jy) and info = (image radii, rays ended by
        a geometry failure)."""
        T = _f64(T).reshape(-1)
        lam_obs = _f64(np.atleast_1d(lam_obs))
        Rfix = _f64(np.atleast_1d(np.asarray(Rfix, float)))
        o = self._trace_opts(angle, nphi, nr, Rfix, lam_path, tracestar, dimstar, scatter)
        flux = np.zeros(lam_obs.size)
        info = np.zeros(2, np.int32)
        self._check(self.lib.mcg_trace_spectrum(self.h, C.byref(o), _ffi.ptr(T), lam_obs.size, _ffi.ptr(lam_obs),
                                                _ffi.ptr(flux), _ffi.ptr(info)))
        return flux, (int(info[0]), int(info[1]))

    def scatter_field(self, T, lam0, angle, nphot=1000, nphot_star=1000, seed=1, nexits=5):
        """mcg_scatter_field: one scattered-light field of the current model
        at wavelength lam0 [micron] for inclination `angle` [rad].  Returns
        (field (nr, nsub, 2, 91), info dict) or (None, info) when the model
        gets no field (no scattering)."""
        T = _f64(T).reshape(-1)
        o = self._trace_opts(angle, 45, 2, np.zeros(0), 0.55, True, 1.0,
                             dict(nphot=nphot, nphot_star=nphot_star, seed=seed, nexits=nexits))
        info = np.zeros(6, np.int64)
        ip = info.ctypes.data_as(C.POINTER(C.c_int64))
        self._check(self.lib.mcg_scatter_field(self.h, C.byref(o), _ffi.ptr(T), float(lam0), None, 0, ip))
        keys = ("nsub", "length", "geometry_failures", "interaction_cap", "no_start", "mode")
        if int(info[5]) == 0:
            return None, dict(zip(keys, (int(x) for x in info)))
        field = np.zeros(int(info[1]))
        self._check(self.lib.mcg_scatter_field(self.h, C.byref(o), _ffi.ptr(T), float(lam0), _ffi.ptr(field),
                                               field.size, ip))
        out = dict(zip(keys, (int(x) for x in info)))
        return field.reshape(self.model.nr, out["nsub"], 2, 91), out

    def trace_image(self, T, lam0, angle, npixel=500, nint=1000, Rmax=None, pa=0.0, nphi=45, nr=2, Rfix=(),
                    tracestar=True, dimstar=1.0, seed=42, linear=None, lam_path=None, scatter=None):
        """mcg_trace_image on the current model: the rectangular image at
        wavelength lam0 [micron] and inclination `angle` [rad] (MakeImage).
        Rmax: half the field of view [AU], by default the grid's outer radius
        (the reference's default fov is twice that); pa: position angle
        [deg]; linear: interpolate the ray intensities linearly (default:
        as the reference does for the model's scattering, linear for the
        full Mueller matrix, log-linear otherwise).  Returns dict(image
        (npixel, npixel) indexed [ix-1, iy-1] in the reference's units per
        pixel (x 1e23 zscale / distance^2 for Jy), flux at lam0, R (image
        radii, AU), rphi (nr, nphi) ray intensities, info).  lam_path: the
        wavelength of the tau = 0.1 radius that places the image rays (an
        IMAGE observation traces at lam0, the default; an IFU at 0.55)."""
        m = self.model
        T = _f64(T).reshape(-1)
        Rfix = _f64(np.atleast_1d(np.asarray(Rfix, float)))
        if Rmax is None:
            Rmax = float(np.asarray(m.R)[-1])
        if linear is None:
            linear = int(m.scat_how) == 2
        nRfix = int(Rfix.size)
        cap = nr * (m.nr - 1) if nr > 0 else (m.nr - 2) // (-nr) + 1
        cap += (m.nt - 1) * 2 * (nRfix + 2) + 1 + 30 + (180 * (nRfix + 1) if int(m.scat_how) == 2 else 0)
        Rimg = np.zeros(cap)
        rphi = np.zeros(cap * int(nphi))
        lam_path = float(lam0) if lam_path is None else float(lam_path)
        o = self._trace_opts(angle, nphi, nr, Rfix, lam_path, tracestar, dimstar, scatter)
        io = _ffi.ImageOpts(int(npixel), int(nint), float(Rmax), float(pa), int(seed) & (2 ** 64 - 1),
                            int(bool(linear)), int(cap), _ffi.ptr(Rimg), _ffi.ptr(rphi))
        flux = np.zeros(1)
        im = np.zeros(int(npixel) * int(npixel))
        info = np.zeros(2, np.int32)
        self._check(self.lib.mcg_trace_image(self.h, C.byref(o), _ffi.ptr(T), float(lam0), C.byref(io),
                                             _ffi.ptr(flux), _ffi.ptr(im), _ffi.ptr(info)))
        n = int(info[0])
        return dict(image=im.reshape(int(npixel), int(npixel)), flux=float(flux[0]), R=Rimg[:n].copy(),
                    rphi=rphi[:n * int(nphi)].reshape(n, int(nphi)).copy(), info=(n, int(info[1])))

    def disk_structure(self, R, Theta, V, Mstar, zones, Temp, dens, dens0, gasdens, w, w0, shscale=None,
                       grain_scale=None, shtype=None):
        """mcg_disk_structure: zones is a list of (rin, rout, sh, rsh, shpow,
        denspow, fix_struct); cell arrays in the library's cell order, w and
        w0 (ncell, ngrains).  shtype: per grain a scale-height type, by name
        ('DISK', 'ZODI', 'HALO', 'LOBE', 'JET', 'SHELL', 'CYLI', 'CAVITY',
        'WEDGE'; any other name keeps the grain's densities, as the
        reference does for an unknown type) or MCG_SH_* code; None: all
        'DISK'.  Returns the new (dens, dens0, gasdens, w, w0)."""
        R, Theta, V, Temp = _f64(R), _f64(Theta), _f64(V), _f64(Temp)
        nr, nt = R.size - 1, Theta.size
        ncell = nr * (nt - 1)
        out = [np.array(a, dtype=np.float64) for a in (dens, dens0, gasdens, w, w0)]
        ng = out[3].size // ncell
        if any(a.size != ncell for a in out[:3]) or out[3].size != ncell * ng or out[4].size != ncell * ng or \
                V.size != ncell or Temp.size != ncell:
            raise McgError(_ffi.MCG_ERR_ARG, "disk_structure: cell arrays need %d cells" % ncell)
        zs = (_ffi.Zone * max(len(zones), 1))()
        for k, z in enumerate(zones):
            zs[k] = _ffi.Zone(*[float(x) for x in z[:6]], int(bool(z[6])))
        keep = [None if a is None else _f64(a) for a in (shscale, grain_scale)]
        sht = None if shtype is None else shtype_codes(shtype, ng)
        st = _ffi.Structure(nr, nt, ng, _ffi.ptr(R), _ffi.ptr(Theta), _ffi.ptr(V), float(Mstar), len(zones), zs,
                            _ffi.ptr(keep[0]), _ffi.ptr(keep[1]), _ffi.ptr(sht))
        self._check(self.lib.mcg_disk_structure(self.h, C.byref(st), _ffi.ptr(Temp), *[_ffi.ptr(a) for a in out]))
        out[3] = out[3].reshape(ncell, ng)
        out[4] = out[4].reshape(ncell, ng)
        return tuple(out)

    def diffuse(self, Ni, dT, T, nphotmin=25, dtmax=1.0, factRW=10.0):
        """mcg_diffuse on the current model: returns (T, EJv, counts) with
        EJv NaN where no diffusion temperature was given and counts =
        (selected, unknowns, solved in the last pass, failed passes)."""
        nc = self.model.ncell
        Ni = np.ascontiguousarray(Ni, dtype=np.int32).reshape(-1)
        dT = _f64(dT).reshape(-1)
        T = np.array(T, dtype=np.float64).reshape(-1)
        if Ni.size != nc or dT.size != nc or T.size != nc:
            raise McgError(_ffi.MCG_ERR_ARG, "diffuse: Ni, dT and T need one value per cell (%d)" % nc)
        EJv = np.full(nc, np.nan)
        counts = np.zeros(4, np.int32)
        self._check(self.lib.mcg_diffuse(self.h, int(nphotmin), float(dtmax), float(factRW), _ffi.ptr(Ni),
                                         _ffi.ptr(dT), _ffi.ptr(T), _ffi.ptr(EJv), _ffi.ptr(counts)))
        return T, EJv, tuple(int(x) for x in counts)


def shtype_codes(shtype, ngrains):
    """int32 MCG_SH_* codes of a per-grain list of scale-height types (names
    as the keyword shtypeN takes them, or codes); a name the reference does
    not know keeps the grain's densities (MCG_SH_KEEP)"""
    if len(shtype) != ngrains:
        raise McgError(_ffi.MCG_ERR_ARG, "shtype needs %d entries" % ngrains)
    out = np.zeros(ngrains, np.int32)
    for k, v in enumerate(shtype):
        if isinstance(v, str):
            name = v.strip().upper()
            out[k] = _ffi.SHTYPES.index(name) if name in _ffi.SHTYPES else _ffi.SHTYPES.index("KEEP")
        else:
            out[k] = int(v)
    return out


def bb_table(lam):
    """Planck table BB[l, iT] (Init.f:2616-2622) built by the library."""
    lib = _ffi.load()
    lam = _f64(lam)
    BB = np.zeros((lam.size, TT))
    st = lib.mcg_bb_table(lam.size, _ffi.ptr(lam), _ffi.ptr(BB))
    if st != 0:
        raise McgError(st, "mcg_bb_table: invalid wavelengths")
    return BB


def planck(T, lam):
    return _ffi.load().mcg_planck(float(T), float(lam))


# ---------------------------------------------------------------- mirrors

class Particle:
    """The fields of `type(Particle)` (Modules.f:59-83) that ComputePart
    writes, one entry per opacity set iopac."""

    def __init__(self, nlam, nopac=1):
        self.nopac = nopac
        self.Kabs = np.zeros((nopac, nlam))
        self.Ksca = np.zeros((nopac, nlam))
        self.Kext = np.zeros((nopac, nlam))
        self.F = np.zeros((nopac, nlam, 6, NANG))
        self.rho = np.zeros(nopac)
        self.mscale = np.ones(nopac)
        self.rscale = np.ones(nopac)
        self.rv = np.zeros(nopac)
        self.counters = [None] * nopac


def ComputePart(ctx, p, ii, input, amin, amax, apow, fmax, blend, porosity, inp_abun, iopac,
                normalize_abun, standard, nsubgrains, lam, particledir=None, abun_in_name=0):
    """ComputePart.f:1 for standard='FILE': `input` is a particle file (ns,
    nf, then per material an .lnk path and 'frac rho').  iopac is 1-based as
    in the reference.  `lam` is the wavelength grid (module global there).

    particledir (the reference's `dirparticle`, a module global there):
    when given, a cached particleNNNN.fits(.gz) made for the same grain
    (ComputePart.f:160-205) is read instead of computing, and a computed
    bin is written as particle<ii>.fits.gz (ComputePart.f:529)."""
    from .model import read_particle_file, readrefind
    from . import particle_fits as PF
    if standard != "FILE":
        raise McgError(_ffi.MCG_ERR_ARG, "standard=%r: only 'FILE' particle files are supported" % standard)
    ns, nf, mats = read_particle_file(input)
    e1, e2, frac, rho = [], [], [], []
    for k, (lnk, fr, rh) in enumerate(mats):
        if inp_abun is not None and k < len(inp_abun) and inp_abun[k] >= 0.0:
            fr = inp_abun[k]
        n_, k_ = readrefind(lnk, lam)
        e1.append(n_)
        e2.append(k_)
        frac.append(fr)
        rho.append(rh)
    io = iopac - 1
    lnkfiles = [m[0] for m in mats]
    if particledir is not None:
        hit = PF.find_particle_file(particledir, ii, amin, amax, apow, ns, fmax, blend, porosity, frac, rho,
                                    lnkfiles, iopac, abun_in_name)
        if hit is not None:
            res = PF.read_particle_fits(hit, lam)
            p.Kabs[io], p.Ksca[io], p.Kext[io], p.F[io] = res["kabs"], res["ksca"], res["kext"], res["F"]
            p.rho[io] = res["rho_av"]
            p.rv[io] = res["rv"]
            p.counters[io] = None
            return p
    res = ctx.compute_part_batch([dict(lam=lam, e1=np.array(e1), e2=np.array(e2), frac=frac, rho=rho,
                                       amin=amin, amax=amax, apow=apow, fmax=fmax, porosity=porosity,
                                       blend=blend, ns=ns, nf=nf, normalize_abun=normalize_abun)])[0]
    p.Kabs[io] = res["kabs"]
    p.Ksca[io] = res["ksca"]
    p.Kext[io] = res["kext"]
    p.F[io] = res["F"]
    p.rho[io] = res["rho_av"]
    p.mscale[io] = res["mscale"]
    p.rscale[io] = res["rscale"]
    p.counters[io] = (res["n_dhs"], res["n_mie"], res["n_dhs_fail"])
    p.rv[io] = math.sqrt(PF.dust_moments(amin, amax, apow, ns)[1]) * 1e-4
    if particledir is not None:
        fr = np.asarray(frac, float) / np.sum(frac)
        PF.write_particle_fits(PF.particle_file_name(particledir, ii, iopac, fr, abun_in_name), lam, res, amin, amax,
                               apow, fmax, blend, porosity, frac, rho, lnkfiles, ns)
    return p


def MCRadiation(ctx, model, NphotTot, niter=1, dofastvisc=False, **run):
    """MCRadiation.f:6: the packet loop on `model` (uploaded on first use).
    Results are stored on the model (EJv, EJv2, Eabs, Ni, T, spec, ...).
    Viscous heating is not part of the built path (dofastvisc is accepted
    for signature parity and ignored)."""
    if getattr(ctx, "model", None) is not model:
        ctx.set_model(model)
    n, out = ctx.mcradiation(NphotTot, **run)
    for k, v in out.items():
        setattr(model, k, v)
    return n


def Diffuse(ctx, model, NPhotMin=25, dTMax=1.0, factRW=10.0):
    """Diffusion.f:9 after MCRadiation on `model`: the post-MC temperatures
    (Main.f:498-549), then the diffusion step for the thick cells that too
    few packets reached (defaults NphotDiffuse = 25, dTDiffuse = 1,
    Init.f:140-141).  Stores T, dT and the diffused cells' EJv on the model;
    returns (selected, unknowns, solved, failed passes)."""
    if getattr(ctx, "model", None) is not model:
        raise McgError(_ffi.MCG_ERR_STATE, "Diffuse: run MCRadiation on this model first")
    T, dT, _ = ctx.finalize_t()
    T, EJv, counts = ctx.diffuse(model.Ni, dT, T, NPhotMin, dTMax, factRW)
    model.T, model.dT, model.EJvDiffuse = T, dT, EJv
    return counts


# ---------------------------------------------------------------- surrogate network
def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _mlp_methods():
    """Context methods of the opacity-surrogate network (include/mcmax_gpu.h,
    mcg_mlp_*)."""

    def mlp_set_params(self, params):
        p = _f32(params)
        self._check(self.lib.mcg_mlp_set_params(self.h, _ffi.ptr(p), p.size))

    def mlp_get_params(self):
        p = np.zeros(_ffi.MLP_NPARAMS, np.float32)
        self._check(self.lib.mcg_mlp_get_params(self.h, _ffi.ptr(p), p.size))
        return p

    def mlp_forward(self, x):
        x = _f32(x).reshape(-1, _ffi.MLP_NIN)
        y = np.zeros((x.shape[0], _ffi.MLP_NOUT), np.float32)
        self._check(self.lib.mcg_mlp_forward(self.h, x.shape[0], _ffi.ptr(x), _ffi.ptr(y)))
        return y

    def mlp_gradient(self, x, t, w):
        x = _f32(x).reshape(-1, _ffi.MLP_NIN)
        t = _f32(t).reshape(-1, _ffi.MLP_NOUT)
        w = _f32(w)
        g = np.zeros(_ffi.MLP_NPARAMS, np.float32)
        loss = C.c_double(0.0)
        self._check(self.lib.mcg_mlp_gradient(self.h, x.shape[0], _ffi.ptr(x), _ffi.ptr(t), _ffi.ptr(w),
                                              _ffi.ptr(g), C.byref(loss)))
        return g, loss.value

    def mlp_train(self, x, t, w, epochs=10, batch=16384, lr=2e-3, lr_min=2e-5, seed=1):
        x = _f32(x).reshape(-1, _ffi.MLP_NIN)
        t = _f32(t).reshape(-1, _ffi.MLP_NOUT)
        w = _f32(w)
        o = _ffi.MlpTrainOpts(int(epochs), int(batch), float(lr), float(lr_min), int(seed))
        r = _ffi.MlpTrainReport()
        self._check(self.lib.mcg_mlp_train(self.h, x.shape[0], _ffi.ptr(x), _ffi.ptr(t), _ffi.ptr(w), C.byref(o),
                                           C.byref(r)))
        ne = min(int(epochs), _ffi.MLP_MAX_EPOCH_LOG)
        return dict(final_loss=r.final_loss, steps=r.steps, device_ms=r.device_ms,
                    epoch_loss=list(r.epoch_loss[:ne]))

    def mlp_gemm_check(self, a_bits, b_bits):
        a = np.ascontiguousarray(a_bits, dtype=np.uint16)
        b = np.ascontiguousarray(b_bits, dtype=np.uint16)
        n = b.shape[0]
        d = np.zeros((128, n), np.float32)
        self._check(self.lib.mcg_mlp_gemm_check(self.h, n, _ffi.ptr(a), _ffi.ptr(b), _ffi.ptr(d)))
        return d

    return dict(mlp_set_params=mlp_set_params, mlp_get_params=mlp_get_params, mlp_forward=mlp_forward,
                mlp_gradient=mlp_gradient, mlp_train=mlp_train, mlp_gemm_check=mlp_gemm_check)


for _k, _v in _mlp_methods().items():
    setattr(Context, _k, _v)
