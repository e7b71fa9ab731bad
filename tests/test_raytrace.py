"""The ray-traced spectrum (TracePath + TraceFlux without a scattering
field) on CPU: the host logic of mcg_trace_spectrum with its kernels as
loops (tests/native/hostcheck.cpp) against the oracle, which stores every
ray's path first and integrates it per wavelength as the reference does
(oracle/oracle_mc.c), bit for bit; and against closed forms: the stellar
flux seen face-on through an empty disk, the optically thin sum of the
cells' emission."""
import math

import numpy as np
import pytest

import hostcheck_ffi as H
import models
import oracle_ffi as O


def _temps(m):
    nc = m.nt - 1
    R_av = np.sqrt(m.R[:-1] * m.R[1:])
    return np.maximum((400.0 * R_av[:, None] ** -0.5 * np.ones(nc)[None, :]).ravel(), 3.0)


LAM = np.geomspace(0.2, 2000.0, 7)


@pytest.mark.parametrize("deg,nj0,Rfix", [(0.0, 2, ()), (45.0, 2, (3.0, 20.0)), (80.0, -2, ()), (30.0, 3, (7.5,))])
def test_replay_matches_oracle(deg, nj0, Rfix):
    m = models.small_disk(nrad=20, ntheta=12, nlam=30, mdust=1e-5)
    T = _temps(m)
    fo, nro, bo = O.trace_spectrum(m, T, LAM, math.radians(deg), nphi=30, nj0=nj0, Rfix=Rfix)
    fh, Rimg, img, bh = H.trace_spectrum(m, T, LAM, math.radians(deg), nphi=30, nj0=nj0, Rfix=Rfix)
    assert bo == bh == 0
    assert nro == Rimg.size
    assert np.array_equal(fo, fh)
    assert np.all(np.diff(Rimg) > 0)
    assert np.all(np.isfinite(fh)) and np.all(fh > 0)


def test_star_through_an_empty_disk():
    m = models.small_disk(nrad=20, ntheta=12, nlam=30, mdust=1e-14)
    f, Rimg, img, bad = H.trace_spectrum(m, _temps(m), [0.3, 0.5], 0.0)
    fstar = np.interp([0.3, 0.5], m.lam, m.Fstar)
    # 30 rays over the stellar disk, trapezoid in radius: a few 1e-3
    assert np.allclose(f / fstar, 1.0, rtol=5e-3), f / fstar


def test_optically_thin_emission_sum():
    """f - star = sum over cells of B(T) Kabs rho V when every ray is thin"""
    m = models.small_disk(nrad=20, ntheta=12, nlam=30, mdust=1e-9)
    T = _temps(m)
    lam_obs = np.array([100.0, 1000.0])
    dens = np.maximum(m.dens, 1e-50)
    nc = m.nt - 1
    thin = []
    for l0 in lam_obs:
        l1 = np.searchsorted(m.lam, l0) - 1
        w2 = (l0 - m.lam[l1]) / (m.lam[l1 + 1] - m.lam[l1])
        iT = np.floor(T).astype(int)
        B = lambda l: (1 - (T - iT)) * m.BB[l, iT] + (T - iT) * m.BB[l, iT + 1]
        src = (1 - w2) * B(l1) * (m.comp_w @ m.Kabs[:, l1]) + w2 * B(l1 + 1) * (m.comp_w @ m.Kabs[:, l1 + 1])
        thin.append(np.sum((src * dens * m.V)[nc:]))
    fstar = np.interp(lam_obs, m.lam, m.Fstar)
    for deg in (0.0, 60.0):
        f, _, _, _ = H.trace_spectrum(m, T, lam_obs, math.radians(deg), nphi=60, nj0=4)
        assert np.allclose((f - fstar) / np.array(thin), 1.0, rtol=0.04), (deg, (f - fstar) / np.array(thin))


def test_edge_on_disk_hides_the_star():
    m = models.small_disk(nrad=20, ntheta=12, nlam=30, mdust=1e-5)
    T = _temps(m)
    f0, _, _, _ = H.trace_spectrum(m, T, [0.3], 0.0)
    f80, _, _, _ = H.trace_spectrum(m, T, [0.3], math.radians(80.0))
    assert f80[0] < 1e-6 * f0[0]


def test_wavelengths_outside_the_grid_give_zero():
    m = models.small_disk(nrad=20, ntheta=12, nlam=30, mdust=1e-5)
    f, _, _, _ = H.trace_spectrum(m, _temps(m), [0.01, 1e5, 1.0], 0.3)
    assert f[0] == 0.0 and f[1] == 0.0 and f[2] > 0.0


@pytest.mark.parametrize("deg,pa,linear,nj0", [(45.0, 20.0, 0, 2), (80.0, 0.0, 1, 2), (10.0, -35.0, 0, -2)])
def test_image_replay_matches_oracle(deg, pa, linear, nj0):
    """MakeImage: the host logic of mcg_trace_image (per-point function of
    the sample kernel, points summed in order) against the oracle's own
    loop, bit for bit"""
    m = models.small_disk(nrad=20, ntheta=12, nlam=30, mdust=1e-5)
    T = _temps(m)
    Rmax = 0.7 * float(m.R[-1])
    io, fo, no, bo = O.trace_image(m, T, 10.0, math.radians(deg), 48, 20, Rmax, pa=pa, seed=5, linear=linear,
                                   nphi=30, nj0=nj0)
    ih, fh, nh, bh = H.trace_image(m, T, 10.0, math.radians(deg), 48, 20, Rmax, pa=pa, seed=5, linear=linear,
                                   nphi=30, nj0=nj0)
    assert (no, bo) == (nh, bh) and bo == 0
    assert fo == fh and np.array_equal(io, ih)
    assert np.all(np.isfinite(ih)) and np.all(ih >= 0) and (ih > 0).sum() > 100


@pytest.mark.parametrize("linear,tol", [(1, 0.01), (0, 0.03)])
def test_image_total_is_the_flux(linear, tol):
    """a field of view around the whole grid collects every point: the
    pixel sum is the Monte Carlo estimate of the flux the trapezoid gives
    (the log-linear interpolation lies a little below the linear one)"""
    m = models.small_disk(nrad=20, ntheta=12, nlam=30, mdust=1e-5)
    T = _temps(m)
    im, f, n, _ = H.trace_image(m, T, 10.0, math.radians(45.0), 64, 40, 1.01 * float(m.R[-1]), seed=1,
                                linear=linear, nphi=30)
    assert abs(im.sum() / f - 1.0) < tol, im.sum() / f


def test_image_is_mirror_symmetric():
    """every point also lands at -phi: with no position angle the image is
    symmetric under y -> -y up to points on a pixel edge"""
    m = models.small_disk(nrad=20, ntheta=12, nlam=30, mdust=1e-5)
    im, f, _, _ = H.trace_image(m, _temps(m), 10.0, math.radians(60.0), 40, 30, float(m.R[-1]), seed=2, nphi=30)
    assert abs(im.sum() - im[:, ::-1].sum()) <= 1e-12 * im.sum()
    same = np.isclose(im, im[:, ::-1], rtol=1e-12, atol=0)
    assert same.mean() > 0.98, same.mean()


def test_image_rotates_with_the_position_angle():
    """pa = 90 degrees turns the image by a quarter: a point at (x, y)
    moves to (y, -x), so b[i, j] = a[n-1-j, i] in 0-based pixels"""
    m = models.small_disk(nrad=20, ntheta=12, nlam=30, mdust=1e-5)
    T = _temps(m)
    R = float(m.R[-1])
    a, _, _, _ = H.trace_image(m, T, 10.0, math.radians(60.0), 40, 30, R, pa=0.0, seed=2, nphi=30)
    b, _, _, _ = H.trace_image(m, T, 10.0, math.radians(60.0), 40, 30, R, pa=90.0, seed=2, nphi=30)
    assert abs(b.sum() / a.sum() - 1.0) < 1e-12
    assert np.isclose(b, a[::-1].T, rtol=1e-9, atol=0).mean() > 0.97
