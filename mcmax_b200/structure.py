"""Structure iterations: the main loop of Main.f:202-792 for a disk whose
vertical structure follows hydrostatic equilibrium (struct_iter, set for
every zone without a fixed structure, Init.f:1519).

Each pass runs the packet loop, the post-Monte-Carlo temperatures and the
diffusion step, then averages the temperatures over the passes
(TempAverage, DiskStructure.f:25-75), rebuilds the densities
(mcg_disk_structure) and compares the temperatures with the previous
pass's (compareCells, DiskStructure.f:551-584).  When two passes in a row
agree to epsiter, or after maxiter passes, one last packet run is made on
the final structure (Main.f:778-790).

    temp_average(Temp, T, fw)                 TempAverage
    compare_cells(T1, dT1, T2, dT2, nr, nt)   compareCells (errT)
    initial_state(model)                      dens0 = dens, w0 = w, gasdens = dens (Init.f:3904)
    planck_means(model)                       Kp(iT) and Kpabsstar of every grain (Init.f:3785-3798)
    thin_temperature(model)                   OpticallyThin's temperatures (Radiation.f:1253-1370)
    mp_settling(...)                          MPSettling's per-grain scale factors (MPSettling.f:8-121)
    fixed_settling(...)                       FixedMPSettling's factors (MPSettling.f:132-168)
    thin_start(ctx, model, zones, Mstar)      the structure the first pass starts from (Init.f:3924-3960)
    iterate(ctx, model, zones, Mstar, nphot)  the loop
"""
import math

import numpy as np

TMAX = 10000


def temp_average(Temp, T, fw):
    """TempAverage: the structure's temperature, a running average of the
    passes' cell temperatures (T below 2.7 K taken as 2.7 K).  The first
    call (Temp None) copies T."""
    T = np.asarray(T, float)
    if Temp is None:
        return T.copy()
    return (1.0 - fw) * np.asarray(Temp, float) + fw * np.maximum(T, 2.7)


def compare_cells(T1, dT1, T2, dT2, nr, nt):
    """errT of compareCells over cells i = 1..nR-1 with both errors above
    1e-200: the mean of (T1 - T2)^2 / (dT1^2 + dT2^2), divided by the cell
    count less one (that count formed in single precision, as the
    reference's real(...) does)"""
    nc = nt - 1
    s = slice(nc, nr * nc)
    T1, dT1, T2, dT2 = (np.asarray(a, float)[s] for a in (T1, dT1, T2, dT2))
    ok = (dT1 > 1e-200) & (dT2 > 1e-200)
    err = float(np.sum((T1[ok] - T2[ok]) ** 2 / (dT1[ok] ** 2 + dT2[ok] ** 2)))
    n = float(np.float32(nr - 1) * np.float32(nt - 1)) - 1.0
    return err / n


def initial_state(model):
    """cell arrays of the structure step at the start: the unsettled
    condensable density and abundances equal the dust's, and the gas
    density (in dust-density units) equals the dust density, unless the
    model carries its own (a gas surface-density file, Init.f:3904)"""
    dens = np.asarray(model.dens, float).copy()
    w = np.asarray(model.comp_w, float).reshape(model.ncell, -1).copy()
    gas = getattr(model, "gasdens", None)
    gas = dens.copy() if gas is None else np.asarray(gas, float).copy()
    return dict(dens=dens, dens0=dens.copy(), gasdens=gas, w=w, w0=w.copy())


def planck_means(model):
    """Per grain (component) the Planck-mean table Kp[k, iT] =
    integrate(BB(:, iT) Kabs) on the 1 K grid and Kpabsstar[k] =
    integrate(Fstar Kabs) / Lstar (Init.f:3785-3798), each trapezoid summed
    in the reference's order (Radiation.f:1-18)."""
    nu = np.asarray(model.nu, float)
    BB = np.asarray(model.BB, float).reshape(model.nlam, TMAX + 1)
    Kabs = np.asarray(model.Kabs, float).reshape(model.ncomp, model.nlam)
    Fstar = np.asarray(model.Fstar, float)
    Kp = np.zeros((model.ncomp, TMAX + 1))
    ks = np.zeros(model.ncomp)
    for i in range(model.nlam - 1):
        c = abs(nu[i] - nu[i + 1]) * 0.5
        Kp = Kp + c * (BB[i][None, :] * Kabs[:, i][:, None] + BB[i + 1][None, :] * Kabs[:, i + 1][:, None])
        ks = ks + c * (Fstar[i] * Kabs[:, i] + Fstar[i + 1] * Kabs[:, i + 1])
    return Kp, ks / model.Lstar


def _cell_energy(Kp, w, iT):
    """computeE_QHP (Radiation.f:924-936): sum over the grains of Kp(iT) w,
    in grain order, for each cell's own iT"""
    E = np.zeros(w.shape[0])
    for k in range(w.shape[1]):
        E = E + Kp[k, iT] * w[:, k]
    return E


def thin_temperature(model, Kp=None, kpabsstar=None):
    """The optically thin temperatures OpticallyThin(.false.) gives at the
    start (Radiation.f:1253-1370, thermal contact, no viscous heating): each
    cell absorbs the dilute stellar field, E = W Lstar / (pi Rstar^2)
    sum_ii Kpabsstar w / sum_ii w with W = (1 - sqrt(1 - (Rstar/r)^2)) / 2
    at the cell's inner radius (the grid's inner edge for the star cell),
    and T solves sum_ii Kp(T) w = E as computeT_QHP does (Radiation.f:848-
    921): the bracketing 1 K steps around E, T^4 interpolated between them
    (in FP64), 1 K below the table and TMAX - 1 above it, 3 K for NaN.  The
    back-warming factors of the reference's three inner passes do not enter
    when OpticallyThin is called with BW false, so one pass is the same.
    Returns T per cell (the library's cell order)."""
    from .model import AU
    if Kp is None or kpabsstar is None:
        Kp, kpabsstar = planck_means(model)
    nr, nc = model.nr, model.nt - 1
    w = np.asarray(model.comp_w, float).reshape(model.ncell, model.ncomp)
    R = np.asarray(model.R, float)
    r = np.repeat(np.where(np.arange(nr) == 0, R[1], R[:nr]) * AU, nc)
    W = 0.5 * (1.0 - np.sqrt(1.0 - (model.Rstar_cm / r) ** 2))
    E = np.zeros(model.ncell)
    for k in range(model.ncomp):
        E = E + kpabsstar[k] * w[:, k]
    E = W * E * model.Lstar / (math.pi * model.Rstar_cm ** 2) / w.sum(1)
    Emin, Emax = _cell_energy(Kp, w, np.ones(model.ncell, int)), _cell_energy(Kp, w, np.full(model.ncell, TMAX, int))
    lo = np.ones(model.ncell, int)
    hi = np.full(model.ncell, TMAX, int)
    while np.any(hi - lo > 1):
        mid = (lo + hi) // 2
        Em = _cell_energy(Kp, w, mid)
        up = Em <= E
        lo = np.where(up & (hi - lo > 1), mid, lo)
        hi = np.where(~up & (hi - lo > 1), mid, hi)
    E0, E1 = _cell_energy(Kp, w, lo), _cell_energy(Kp, w, hi)
    t4 = lambda i: (i.astype(float) ** 2) ** 2
    with np.errstate(invalid="ignore", divide="ignore"):
        T = np.sqrt(np.sqrt(t4(lo) + ((t4(hi) - t4(lo)) * (E - E0)) / (E1 - E0)))
    T = np.where(E1 == E0, lo.astype(float), T)
    T = np.where(E > Emax, float(TMAX - 1), T)
    T = np.where(E < Emin, 1.0, T)
    return np.where(np.isnan(E), 3.0, T)


def mp_settling(model, state, T, Mstar, rho, rv, alpha, rscale=None, gas2dust=100.0):
    """Dust scale-height factors of MPSettling (MPSettling.f:8-121, after
    Dubrulle et al. 1995), recomputed before every structure pass: per grain
    ii and ring i, the stopping time of the midplane cell, tau_f =
    <rho_ii rv_ii rscale> / (c_s rho_gas) (the grain's density-weighted
    mean over the ring's cells, rho_gas from the midplane gas density, or
    the dust's times gas2dust when that is below 1e-5 of the dust's), with
    c_s = sqrt(k T / (2.3 amu)) at the midplane temperature, Omega =
    sqrt(G Mstar / R^3), h = (1/3)^(1/4) sqrt(alpha / (Omega tau_f)) and
    the factor h / sqrt(1 + h^2).  The reference's constants are kept: G =
    6.672e-8, mu = 2.3 as a single-precision literal.  rho, rv [cm],
    rscale: per grain; alpha: per ring (the zone's alphaturb).  Returns the
    grain_scale array (ngrains, nr) of mcg_disk_structure (ring 0 unused,
    1)."""
    from .model import AU
    nr, nc = model.nr, model.nt - 1
    ng = model.ncomp
    dens = np.asarray(state["dens"], float).reshape(nr, nc)
    gas = np.asarray(state["gasdens"], float).reshape(nr, nc)
    w = np.asarray(state["w"], float).reshape(nr, nc, ng)
    T = np.asarray(T, float).reshape(nr, nc)
    rscale = np.ones(ng) if rscale is None else np.asarray(rscale, float)
    R = np.asarray(model.R, float)
    R_av = AU * 10.0 ** ((np.log10(R[:-1]) + np.log10(R[1:])) / 2.0)
    GG, amu, kb, mu, gamma = 6.672e-8, 1.66053886e-24, 1.3806503e-16, float(np.float32(2.3)), 2.0
    omega_r = math.sqrt(GG * Mstar)
    cs_T = math.sqrt(kb / (mu * amu))
    prefac = (1.0 / (1.0 + gamma)) ** 0.25
    scale = np.ones((ng, nr))
    for ii in range(ng):
        for i in range(1, nr):
            t, tot = 0.0, 0.0
            for j in range(nc):
                t = t + dens[i, j] * w[i, j, ii] * rho[ii] * rv[ii] * rscale[ii]
                tot = tot + dens[i, j] * w[i, j, ii]
            t = t / tot if tot > 1e-100 else rho[ii] * rv[ii]
            rho_g = gas[i, nc - 1] * gas2dust
            if rho_g < dens[i, nc - 1] / 1e5:
                rho_g = dens[i, nc - 1] * gas2dust
            cs = cs_T * math.sqrt(T[i, nc - 1])
            omegatau = (omega_r / R_av[i] ** 1.5) * (t / (cs * rho_g))
            h = prefac * math.sqrt(alpha[i] / omegatau)
            scale[ii, i] = h * (1.0 + h ** 2) ** (-0.5)
    return scale


def fixed_settling(model, state, rho, rv, alpha, rscale=None, gas2dust=100.0):
    """Dust scale-height factors of FixedMPSettling (MPSettling.f:132-168),
    which DiskStructure recomputes at the start of every structure pass
    (DiskStructure.f:108): per ring i the gas surface density Sigma =
    sum_j gasdens gas2dust V / (pi (R(i+1)^2 - R(i)^2) AU^2), per grain the
    density-weighted mean of rho rv rscale over the ring's cells (rho rv
    when the grain is absent), hH = (1/3)^(1/4) sqrt(alpha Sigma /
    (sqrt(2 pi) <rho rv rscale>)) and the factor hH / sqrt(1 + hH^2).
    alpha: a number or one value per ring (the midplane cell's alphaturb);
    the sums over theta are numpy's.  Returns grain_scale (ngrains, nr) of
    mcg_disk_structure (ring 0 unused, 1)."""
    from .model import AU
    nr, nc = model.nr, model.nt - 1
    ng = model.ncomp
    dens = np.asarray(state["dens"], float).reshape(nr, nc)
    gas = np.asarray(state["gasdens"], float).reshape(nr, nc)
    w = np.asarray(state["w"], float).reshape(nr, nc, ng)
    V = np.asarray(model.V, float).reshape(nr, nc)
    R = np.asarray(model.R, float)
    rho = np.asarray(rho, float)
    rv = np.asarray(rv, float)
    rscale = np.ones(ng) if rscale is None else np.asarray(rscale, float)
    alpha = np.broadcast_to(np.asarray(alpha, float), (nr,))
    c1 = (1.0 / (1.0 + 2.0)) ** 0.25
    scale = np.ones((ng, nr))
    for i in range(1, nr):
        sigma = (gas[i] * gas2dust * V[i]).sum() / (math.pi * (R[i + 1] ** 2 - R[i] ** 2) * AU ** 2)
        dw = dens[i][:, None] * w[i]                                  # (nc, ng)
        tot = dw.sum(0)
        t = (dw * (rho * rv * rscale)[None, :]).sum(0)
        t = np.where(tot > 1e-100, t / np.where(tot > 1e-100, tot, 1.0), rho * rv)
        hH = c1 * np.sqrt(alpha[i] * sigma / (math.sqrt(2.0 * math.pi) * t))
        scale[:, i] = hH / np.sqrt(1.0 + hH ** 2)
    return scale


def _grain_scale(model, state, T, Mstar, grain_scale, settling, fixed):
    if fixed:
        return fixed_settling(model, state, **fixed)
    if settling:
        return mp_settling(model, state, T, Mstar, **settling)
    return grain_scale


def thin_start(ctx, model, zones, Mstar, shscale=None, grain_scale=None, settling=None, fixed=None, shtype=None):
    """The vertical structure the first Monte Carlo pass starts from
    (Init.f:3924-3960): dens0 = gasdens = dens, the optically thin
    temperatures (BackWarming(1) changes nothing before the first pass:
    no cell has absorbed packets yet), their average (the first
    TempAverage copies them) and three DiskStructure passes on them.
    settling: the keyword arguments of mp_settling (rho, rv, alpha,
    rscale, gas2dust) when the grains settle (mpset); their factors are
    then recomputed before every pass, at the thin temperatures.  fixed:
    the keyword arguments of fixed_settling (fixmpset), recomputed before
    every pass the same way.  shtype: per grain its scale-height type
    (Context.disk_structure).
    Regridding in theta and dead zones are not built.  Updates the model's
    dens and comp_w; returns dict(state, Temp)."""
    state = initial_state(model)
    Tthin = thin_temperature(model)
    Temp = temp_average(None, Tthin, 1.0)
    for _ in range(3):
        grain_scale = _grain_scale(model, state, Tthin, Mstar, grain_scale, settling, fixed)
        out = ctx.disk_structure(model.R, model.Theta, model.V, Mstar, zones, Temp, state["dens"], state["dens0"],
                                 state["gasdens"], state["w"], state["w0"], shscale, grain_scale, shtype)
        state = dict(zip(("dens", "dens0", "gasdens", "w", "w0"), out))
    model.dens = state["dens"]
    model.comp_w = state["w"].reshape(model.ncell, -1)
    return dict(state=state, Temp=Temp)


def iterate(ctx, model, zones, Mstar, nphot, run=None, maxiter=10, epsiter=3.0, f_weight=0.5, niter0=1000,
            nphotdiffuse=25, dtdiffuse=1.0, shscale=None, grain_scale=None, precision="mixed", log=None,
            thin=False, settling=None, fixed=None, shtype=None, on_pass=None):
    """Run the structure iterations on `model` (one opacity set per grain:
    comp_w holds the grains' abundances).  zones: (rin, rout, sh, rsh,
    shpow, denspow, fix_struct) per zone; Mstar in g; run: the keyword
    arguments of Context.mcradiation.  thin: start from the optically thin
    structure (thin_start), as the reference does before its first pass;
    otherwise from the model's densities.  settling: mp_settling's keyword
    arguments when the grains settle (mpset): the factors are recomputed
    from the current state and temperatures before every structure pass;
    fixed: fixed_settling's arguments (fixmpset), recomputed the same way.
    shtype: per grain its scale-height type.  on_pass(n, result, T): called
    after every packet run (n the run's packet count).  Each packet run
    takes its own Philox key, run['seed'] plus the number of runs before
    it, where the reference's one random stream runs on.
    The model's dens and comp_w are updated in place.  Returns dict(T, dT,
    Temp, state, history, nphot, result) with one history entry (niter,
    errT, packets) per structure pass and the last packet run's count and
    result."""
    run = dict(run or {})
    if thin:
        state = thin_start(ctx, model, zones, Mstar, shscale, grain_scale, settling, fixed, shtype)["state"]
    else:
        state = initial_state(model)
    Temp = None
    niter = 0
    finaliter = lastiter = False
    Tprev = dTprev = np.zeros(model.ncell)
    history = []
    while True:
        model.dens = state["dens"]
        model.comp_w = state["w"].reshape(model.ncell, -1)
        ctx.set_model(model)
        runk = dict(run)
        if "seed" in runk:
            runk["seed"] = int(runk["seed"]) + len(history)
        n, res = ctx.mcradiation(int(nphot), precision=precision, **runk)
        T, dT, _ = ctx.finalize_t()
        if nphotdiffuse > 0 or dtdiffuse < 1.0:
            T, _, _ = ctx.diffuse(res["Ni"], dT, T, nphotdiffuse, dtdiffuse, run.get("factRW", 10.0))
        if on_pass:
            on_pass(n, res, T)
        if lastiter or maxiter <= 0:
            break
        niter += 1
        if niter > niter0:
            fw = 1.0 / (niter - niter0)
        elif niter > 1:
            fw = f_weight
        else:
            fw = 1.0
        Temp = temp_average(Temp, T, fw)
        grain_scale = _grain_scale(model, state, T, Mstar, grain_scale, settling, fixed)
        out = ctx.disk_structure(model.R, model.Theta, model.V, Mstar, zones, Temp, state["dens"], state["dens0"],
                                 state["gasdens"], state["w"], state["w0"], shscale, grain_scale, shtype)
        state = dict(zip(("dens", "dens0", "gasdens", "w", "w0"), out))
        errT = compare_cells(Tprev, dTprev, T, dT, model.nr, model.nt)
        history.append(dict(niter=niter, errT=errT, packets=n))
        if log:
            log("structure pass %d: errT %.3g sigma" % (niter, errT))
        Tprev, dTprev = T, dT
        if (errT < epsiter and finaliter) or niter > maxiter:
            lastiter = True
            continue
        finaliter = errT < epsiter
    model.dens = state["dens"]
    model.comp_w = state["w"].reshape(model.ncell, -1)
    return dict(T=T, dT=dT, Temp=Temp, state=state, history=history, nphot=n, result=res)

