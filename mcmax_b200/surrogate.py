"""Opacity surrogate: a 6 -> 4x256 -> 64 network standing in for the
coated-sphere (DHS) sums of ComputePart (ComputePart.f:318-447) inside its
training box, with the DHS kernels as the fallback outside it.  No
counterpart in the reference.

    samples = sobol_samples(n, seed)              # (a, lambda, n, k, porosity, fmax)
    T = targets(ctx, samples)                     # ComputePart on the GPU, one size each
    params, info = train(ctx, samples, T)         # tcgen05 forward/backward + Adam
    save(path, params, info); load(path)
    compute_part_surrogate(ctx, parts, params)    # drop-in for Context.compute_part_batch

The network inputs and outputs are documented in include/mcmax_gpu.h
(mcg_surrogate_targets, mcg_compute_part_surrogate)."""
import ctypes as C
import time

import numpy as np

from . import _ffi

NIN, NOUT, H = 6, 64, 256
NMOM = 12
# training box: log10 a [micron], log10 lambda [micron], n, log10 k, porosity, fmax
BOX_LO = np.array([-2.0, -1.0, 1.5, -3.5, 0.0, 0.0])
BOX_HI = np.array([3.0, np.log10(3000.0), 3.5, np.log10(2.0), 0.6, 0.8])
RHO_TRAIN = 3.0
NF_TRAIN = 20
# loss weight per output: the two opacities, the F11 moments, the F12
# moments, the F33 and F34 moments (polarisation only)
OUT_WEIGHT = np.zeros(NOUT, np.float32)
OUT_WEIGHT[0:2] = 16.0
OUT_WEIGHT[2:14] = 1.0
OUT_WEIGHT[14:27] = 0.5
OUT_WEIGHT[27:53] = 0.25


def sobol_samples(n, seed=0):
    """n points of a scrambled Sobol sequence over the training box, as
    physical samples (a [micron], lambda [micron], n, k, porosity, fmax)."""
    from scipy.stats import qmc
    u = qmc.Sobol(d=NIN, scramble=True, seed=seed).random(n)
    v = BOX_LO + u * (BOX_HI - BOX_LO)
    s = np.empty_like(v)
    s[:, 0] = 10.0 ** v[:, 0]
    s[:, 1] = 10.0 ** v[:, 1]
    s[:, 2] = v[:, 2]
    s[:, 3] = 10.0 ** v[:, 3]
    s[:, 4] = v[:, 4]
    s[:, 5] = v[:, 5]
    return s


def normalize(samples):
    """network inputs in [-1, 1] of physical samples"""
    s = np.asarray(samples, float)
    v = np.stack([np.log10(s[:, 0]), np.log10(s[:, 1]), s[:, 2], np.log10(s[:, 3]), s[:, 4], s[:, 5]], axis=1)
    return (2.0 * (v - BOX_LO) / (BOX_HI - BOX_LO) - 1.0).astype(np.float32)


def targets(ctx, samples, rho=RHO_TRAIN, nf=NF_TRAIN):
    """ComputePart targets of single-size samples, computed on the GPU."""
    s = np.ascontiguousarray(samples, dtype=np.float64)
    out = np.zeros((s.shape[0], NOUT), np.float32)
    ctx._check(ctx.lib.mcg_surrogate_targets(ctx.h, s.shape[0], _ffi.ptr(s), float(rho), int(nf), _ffi.ptr(out)))
    return out


def init_params(seed=0):
    """He-style initialisation of the flat parameter vector"""
    rng = np.random.default_rng(seed)
    W0 = rng.normal(0, 1.0 / np.sqrt(NIN), (H, NIN))
    W = rng.normal(0, 1.0 / np.sqrt(H), (3, H, H))
    W4 = rng.normal(0, 0.5 / np.sqrt(H), (NOUT, H))
    return np.concatenate([W0.ravel(), np.zeros(H), W.ravel(), np.zeros(3 * H), W4.ravel(),
                           np.zeros(NOUT)]).astype(np.float32)


def fold_output_scaling(params, mean, std):
    """network trained on (t - mean) / std -> network that outputs t"""
    p = np.array(params, np.float32)
    o4 = H * NIN + H + 3 * H * H + 3 * H
    W4 = p[o4:o4 + NOUT * H].reshape(NOUT, H)
    b4 = p[o4 + NOUT * H:]
    W4 *= std[:, None]
    b4[:] = b4 * std + mean
    return p


def train(ctx, samples, T, epochs=300, batch=8192, lr=2e-3, lr_min=2e-5, seed=1, weights=None):
    """Train on (samples, targets); returns (params, info).  Targets are
    standardised per output for training and the scaling is folded into
    the output layer, so the returned network outputs physical targets."""
    X = normalize(samples)
    T = np.asarray(T, np.float32)
    mean = T.mean(0)
    std = T.std(0)
    std[std < 1e-6] = 1.0
    # powers of two: folding them into the output layer commutes with the
    # BF16 rounding of its weights, so the folded network computes exactly
    # what was trained
    std = (2.0 ** np.round(np.log2(std))).astype(np.float32)
    Ts = ((T - mean) / std).astype(np.float32)
    ctx.mlp_set_params(init_params(seed))
    t0 = time.perf_counter()
    w = OUT_WEIGHT if weights is None else np.asarray(weights, np.float32)
    rep = ctx.mlp_train(X, Ts, w, epochs=epochs, batch=batch, lr=lr, lr_min=lr_min, seed=seed)
    wall = time.perf_counter() - t0
    p = fold_output_scaling(ctx.mlp_get_params(), mean, std)
    ctx.mlp_set_params(p)
    info = dict(epochs=epochs, batch=batch, lr=lr, lr_min=lr_min, seed=seed, n=int(X.shape[0]),
                final_loss=rep["final_loss"], device_ms=rep["device_ms"], wall_s=wall,
                epoch_loss=np.array(rep["epoch_loss"]), rho=RHO_TRAIN, nf=NF_TRAIN)
    return p, info


def save(path, params, info):
    np.savez_compressed(path, params=np.asarray(params, np.float32), box_lo=BOX_LO, box_hi=BOX_HI,
                        **{k: np.asarray(v) for k, v in info.items()})


def load(path):
    z = np.load(path)
    info = {k: z[k] for k in z.files if k not in ("params",)}
    return z["params"].astype(np.float32), info


def compute_part_surrogate(ctx, parts, params=None, rho_train=RHO_TRAIN, nf_train=NF_TRAIN):
    """Context.compute_part_batch with the network serving every bin that
    qualifies (mcg_compute_part_surrogate); returns (results, used)."""
    if params is not None:
        ctx.mlp_set_params(params)
    from .api import _f64
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
        o = dict(kabs=np.zeros(nlam), ksca=np.zeros(nlam), kext=np.zeros(nlam), F=np.zeros((nlam, 6, 180)))
        keep += [lam, e1, e2, frac, rho]
        ins[k] = _ffi.PartIn(nlam, _ffi.ptr(lam), e1.shape[0], _ffi.ptr(e1), _ffi.ptr(e2), _ffi.ptr(frac),
                             _ffi.ptr(rho), float(p["amin"]), float(p["amax"]), float(p["apow"]), float(p["fmax"]),
                             float(p.get("porosity", 0.0)), float(p.get("normalize_abun", -1.0)),
                             int(bool(p.get("blend", False))), int(p["ns"]), int(p["nf"]))
        for key in ("kabs", "ksca", "kext", "F"):
            setattr(outs[k], key, _ffi.ptr(o[key]))
        res.append(o)
    used = np.zeros(n, np.int32)
    ctx._check(ctx.lib.mcg_compute_part_surrogate(ctx.h, n, ins, outs, float(rho_train), int(nf_train),
                                                  _ffi.ptr(used)))
    for k, o in enumerate(res):
        o.update(rho_av=outs[k].rho_av, mscale=outs[k].mscale, rscale=outs[k].rscale, n_dhs=outs[k].n_dhs,
                 n_mie=outs[k].n_mie, n_dhs_fail=outs[k].n_dhs_fail)
    return res, used


def correction_wavelengths(nlam, stride):
    """indices of the wavelengths ComputePart evaluates for the correction:
    every stride-th and the last"""
    return np.unique(np.r_[np.arange(0, nlam, max(1, int(stride))), nlam - 1])


def correct_with_exact(res, used, parts, exact, idx):
    """Scale the network's kappa_abs and kappa_sca of every bin it served by
    the ratio ComputePart / network at the wavelengths idx, the log10 ratio
    interpolated linearly in log10 lambda between them (constant beyond the
    ends); kappa_ext becomes their sum.  `exact` holds ComputePart's results
    at parts' wavelengths idx, one per served bin in order.  The Mueller
    matrix stays the network's.  A key whose values are not all positive
    keeps the network's values."""
    served = [k for k in range(len(parts)) if used[k]]
    if len(exact) != len(served):
        raise ValueError("one exact result per bin served by the network")
    for k, e in zip(served, exact):
        o = res[k]
        ll = np.log10(np.asarray(parts[k]["lam"], np.float64))
        for key in ("kabs", "ksca"):
            net = np.asarray(o[key], np.float64)
            ex = np.asarray(e[key], np.float64)
            if np.all(net[idx] > 0) and np.all(ex > 0):
                o[key] = net * 10.0 ** np.interp(ll, ll[idx], np.log10(ex) - np.log10(net[idx]))
        o["kext"] = np.asarray(o["kabs"]) + np.asarray(o["ksca"])
    return res


def compute_part_corrected(ctx, parts, params=None, stride=10, rho_train=RHO_TRAIN, nf_train=NF_TRAIN):
    """compute_part_surrogate, then ComputePart itself (the DHS kernels) at
    every stride-th wavelength of the bins the network served, which
    corrects the network's kappa_abs and kappa_sca (correct_with_exact).
    Every bin's wavelengths are evaluated independently by ComputePart, so
    the subset gives the same values as the full grid there.  Returns
    (results, used, wavelengths evaluated per served bin)."""
    res, used = compute_part_surrogate(ctx, parts, params, rho_train, nf_train)
    served = [k for k in range(len(parts)) if used[k]]
    if not served:
        return res, used, 0
    idx = correction_wavelengths(np.asarray(parts[served[0]]["lam"]).size, stride)
    sub = []
    for k in served:
        p = parts[k]
        if np.asarray(p["lam"]).size != np.asarray(parts[served[0]]["lam"]).size:
            raise ValueError("the bins served by the network must share one wavelength count")
        q = dict(p)
        q["lam"] = np.asarray(p["lam"], np.float64)[idx]
        q["e1"] = np.atleast_2d(p["e1"])[:, idx]
        q["e2"] = np.atleast_2d(p["e2"])[:, idx]
        sub.append(q)
    exact = ctx.compute_part_batch(sub)
    return correct_with_exact(res, used, parts, exact, idx), used, int(idx.size)
