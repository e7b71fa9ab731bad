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
    iterate(ctx, model, zones, Mstar, nphot)  the loop
"""
import numpy as np


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
    density (in dust-density units) equals the dust density (Init.f:3904)"""
    dens = np.asarray(model.dens, float).copy()
    w = np.asarray(model.comp_w, float).reshape(model.ncell, -1).copy()
    return dict(dens=dens, dens0=dens.copy(), gasdens=dens.copy(), w=w, w0=w.copy())


def iterate(ctx, model, zones, Mstar, nphot, run=None, maxiter=10, epsiter=3.0, f_weight=0.5, niter0=1000,
            nphotdiffuse=25, dtdiffuse=1.0, shscale=None, grain_scale=None, precision="mixed", log=None):
    """Run the structure iterations on `model` (one opacity set per grain:
    comp_w holds the grains' abundances).  zones: (rin, rout, sh, rsh,
    shpow, denspow, fix_struct) per zone; Mstar in g; run: the keyword
    arguments of Context.mcradiation.  The model's dens and comp_w are
    updated in place.  Returns dict(T, dT, Temp, state, history, nphot,
    result) with one history entry (niter, errT, packets) per structure
    pass and the last packet run's count and result."""
    run = dict(run or {})
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
        n, res = ctx.mcradiation(int(nphot), precision=precision, **run)
        T, dT, _ = ctx.finalize_t()
        if nphotdiffuse > 0 or dtdiffuse < 1.0:
            T, _, _ = ctx.diffuse(res["Ni"], dT, T, nphotdiffuse, dtdiffuse, run.get("factRW", 10.0))
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
        out = ctx.disk_structure(model.R, model.Theta, model.V, Mstar, zones, Temp, state["dens"], state["dens0"],
                                 state["gasdens"], state["w"], state["w0"], shscale, grain_scale)
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

