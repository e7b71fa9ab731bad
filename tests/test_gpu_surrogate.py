"""The opacity surrogate: its training targets are ComputePart's own
numbers, and the trained network serves config-style grain bins faster than
the DHS kernels at a bounded opacity error, falling back to DHS outside its
training box."""
import time

import numpy as np
import pytest

from mcmax_b200 import model as M
from mcmax_b200 import surrogate as S

pytestmark = pytest.mark.gpu


def _moments(F, nmom=S.NMOM):
    th = np.pi * (np.arange(180) + 0.5) / 180
    mu, w = np.cos(th), np.sin(th)
    P = [np.ones(180), mu]
    for l in range(1, nmom):
        P.append(((2 * l + 1) * mu * P[l] - l * P[l - 1]) / (l + 1))
    f11, f12, f33, f34 = F[0] * w, F[1] * w, F[3] * w, F[4] * w
    s0 = f11.sum()
    return (np.array([(f11 * P[l]).sum() / s0 for l in range(1, nmom + 1)]),
            np.array([(f12 * P[l]).sum() / s0 for l in range(0, nmom + 1)]),
            np.array([(f33 * P[l]).sum() / s0 for l in range(0, nmom + 1)]),
            np.array([(f34 * P[l]).sum() / s0 for l in range(0, nmom + 1)]))


def test_targets_are_compute_part_of_one_size(ctx):
    samples = np.array([[0.3, 0.55, 1.7, 0.02, 0.25, 0.8], [2.0, 10.0, 2.4, 0.3, 0.0, 0.5],
                        [0.05, 3.0, 1.6, 0.003, 0.5, 0.0], [40.0, 100.0, 3.0, 1.2, 0.3, 0.7]])
    T = S.targets(ctx, samples)
    for s, t in zip(samples, T):
        a, lam, n, k, por, fmax = s
        r = ctx.compute_part_batch([dict(lam=[lam, 1.01 * lam], e1=[[n, n]], e2=[[k, k]], frac=[1.0], rho=[3.0],
                                         amin=a, amax=a, apow=3.5, fmax=fmax, porosity=por, blend=True, ns=1,
                                         nf=20)])[0]
        assert abs(t[0] - np.log10(r["kabs"][0])) < 1e-5
        assert abs(t[1] - np.log10(r["ksca"][0])) < 1e-5
        chi, beta, gamma, delta = _moments(r["F"][0])
        assert np.allclose(t[2:14], chi, atol=2e-6)
        assert np.allclose(t[14:27], beta, atol=2e-6)
        assert np.allclose(t[27:40], gamma, atol=2e-6)
        assert np.allclose(t[40:53], delta, atol=2e-6)
        assert np.all(t[53:] == 0)


def _config_bins(nlam=60):
    """grain bins in the style of the learned-opacities deck: three
    compositions (k prefactors 0.003 / 0.03 / 0.3), sizes 0.01-1000 micron"""
    lam, _ = M.wavelength_grid(0.1, 3000.0, nlam)
    bins = M.grain_bins(0.01, 1000.0, 10)
    parts = []
    for kp, por, fmax in ((0.003, 0.2, 0.8), (0.03, 0.4, 0.5), (0.3, 0.0, 0.8)):
        n, k = M.synthetic_lnk(lam, kp)
        for a, b in bins[::3]:
            parts.append(dict(lam=lam, e1=[n], e2=[k], frac=[1.0], rho=[3.0], amin=a, amax=b, apow=3.5, fmax=fmax,
                              porosity=por, blend=True, ns=4, nf=20))
    return parts


def test_surrogate_trains_and_serves_bins(ctx):
    samples = S.sobol_samples(1 << 16, seed=3)
    T = S.targets(ctx, samples)
    params, info = S.train(ctx, samples, T, epochs=40, batch=2048, lr=2e-3, lr_min=2e-5, seed=2)
    # held-out single-size error in log10 kappa (a small training run: the
    # full 2e6-sample network is measured by the bench)
    test = S.sobol_samples(4096, seed=99)
    Tt = S.targets(ctx, test)
    Y = ctx.mlp_forward(S.normalize(test))
    err_abs = np.abs(Y[:, 0] - Tt[:, 0])
    err_sca = np.abs(Y[:, 1] - Tt[:, 1])
    assert np.median(err_abs) < 0.1 and np.median(err_sca) < 0.1, (np.median(err_abs), np.median(err_sca),
                                                                  info["epoch_loss"])
    # grain bins: network vs the DHS kernels
    parts = _config_bins()
    t0 = time.perf_counter()
    ref = ctx.compute_part_batch(parts)
    t_dhs = time.perf_counter() - t0
    t0 = time.perf_counter()
    got, used = S.compute_part_surrogate(ctx, parts)
    t_net = time.perf_counter() - t0
    assert used.all()
    lk = np.concatenate([np.log10(g["kabs"] / r["kabs"]) for g, r in zip(got, ref)])
    ls = np.concatenate([np.log10(g["ksca"] / r["ksca"]) for g, r in zip(got, ref)])
    assert np.median(np.abs(lk)) < 0.1 and np.median(np.abs(ls)) < 0.1, (np.median(np.abs(lk)),
                                                                         np.median(np.abs(ls)))
    # the gain: the network replaces the coated-sphere sums
    assert t_net < 0.5 * t_dhs, (t_net, t_dhs)
    for g in got:
        F = g["F"]
        assert np.all(F[:, 0] >= 0) and np.all(np.abs(F[:, 1]) <= F[:, 0] + 1e-12)
        # spheres: F22 = F11, F44 = F33 and F12^2 + F33^2 + F34^2 <= F11^2
        assert np.array_equal(F[:, 2], F[:, 0]) and np.array_equal(F[:, 5], F[:, 3])
        assert np.all(F[:, 1] ** 2 + F[:, 3] ** 2 + F[:, 4] ** 2 <= F[:, 0] ** 2 * (1 + 1e-9) + 1e-300)
    # the polarisation elements follow the DHS kernels': F34 is not zero
    f34 = np.concatenate([g["F"][:, 4].ravel() for g in got])
    assert np.abs(f34).max() > 0


def test_surrogate_falls_back_outside_the_box(ctx):
    ctx.mlp_set_params(S.init_params(0))
    lam, _ = M.wavelength_grid(0.1, 3000.0, 12)
    n, k = M.synthetic_lnk(lam, 0.03)
    inside = dict(lam=lam, e1=[n], e2=[k], frac=[1.0], rho=[3.0], amin=0.1, amax=1.0, apow=3.5, fmax=0.8,
                  porosity=0.25, blend=True, ns=2, nf=20)
    outside = dict(inside, porosity=0.7)           # porosity beyond the box
    two_mat = dict(inside, e1=[n, n], e2=[k, k], frac=[0.5, 0.5], rho=[3.0, 2.0])
    res, used = S.compute_part_surrogate(ctx, [inside, outside, two_mat])
    assert list(used) == [1, 0, 0]
    ref = ctx.compute_part_batch([outside, two_mat])
    for g, r in zip(res[1:], ref):
        for key in ("kabs", "ksca", "F"):
            assert np.array_equal(g[key], r[key])
