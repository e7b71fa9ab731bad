"""mcg_trace_spectrum and mcg_trace_image on the GPU against the host replay
of the same host logic and per-ray arithmetic and against the oracle's own
restatement of TraceMono/MakeImage, bit for bit (the unit is built with
--fmad=false, the replay and the oracle with -ffp-contract=off, and the ray
set-up and attenuation use detmath.h)."""
import math

import numpy as np
import pytest

import hostcheck_ffi as H
import models
import oracle_ffi as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("deg", [0.0, 45.0, 80.0])
def test_trace_spectrum_matches_replay(ctx, deg):
    m = models.small_disk(nrad=20, ntheta=12, nlam=30, mdust=1e-5)
    nc = m.nt - 1
    R_av = np.sqrt(m.R[:-1] * m.R[1:])
    T = np.maximum((400.0 * R_av[:, None] ** -0.5 * np.ones(nc)[None, :]).ravel(), 3.0)
    lam = np.geomspace(0.2, 2000.0, 7)
    ctx.set_model(m)
    fg, info = ctx.trace_spectrum(T, lam, math.radians(deg), nphi=30, nr=2)
    fh, Rimg, _, bad = H.trace_spectrum(m, T, lam, math.radians(deg), nphi=30, nj0=2)
    assert info == (Rimg.size, bad) and bad == 0
    assert np.array_equal(fg, fh)
    fo, nro, bo = O.trace_spectrum(m, T, lam, math.radians(deg), nphi=30, nj0=2)
    assert (nro, bo) == info
    assert np.array_equal(fg, fo)


@pytest.mark.parametrize("deg,pa,linear", [(45.0, 20.0, 0), (80.0, 0.0, 1)])
def test_trace_image_matches_replay(ctx, deg, pa, linear):
    """the sample kernel, the stable sort and the per-pixel sums give the
    sequential loop's image bit for bit"""
    m = models.small_disk(nrad=20, ntheta=12, nlam=30, mdust=1e-5)
    nc = m.nt - 1
    R_av = np.sqrt(m.R[:-1] * m.R[1:])
    T = np.maximum((400.0 * R_av[:, None] ** -0.5 * np.ones(nc)[None, :]).ravel(), 3.0)
    ctx.set_model(m)
    Rmax = 0.6 * float(m.R[-1])
    g = ctx.trace_image(T, 10.0, math.radians(deg), npixel=64, nint=50, Rmax=Rmax, pa=pa, nphi=30, nr=2, seed=9,
                        linear=bool(linear))
    ih, fh, nh, bh = H.trace_image(m, T, 10.0, math.radians(deg), 64, 50, Rmax, pa=pa, seed=9, linear=linear,
                                   nphi=30, nj0=2)
    assert g["info"] == (nh, bh) and bh == 0
    assert g["flux"] == fh
    assert np.array_equal(g["image"], ih)
    io, fo, no, bo = O.trace_image(m, T, 10.0, math.radians(deg), 64, 50, Rmax, pa=pa, seed=9, linear=linear,
                                   nphi=30, nj0=2)
    assert g["info"] == (no, bo) and g["flux"] == fo
    assert np.array_equal(np.ravel(g["image"]), np.ravel(io))
    _, Rimg, rphi, _ = H.trace_spectrum(m, T, [10.0], math.radians(deg), nphi=30, nj0=2, lam_path=10.0)
    assert np.array_equal(g["R"], Rimg) and np.array_equal(g["rphi"], rphi)


def test_trace_image_in_chunks(ctx):
    """more points than one sort chunk (2^23): the pixel sums carry over"""
    m = models.small_disk(nrad=12, ntheta=8, nlam=20, mdust=1e-5)
    nc = m.nt - 1
    R_av = np.sqrt(m.R[:-1] * m.R[1:])
    T = np.maximum((300.0 * R_av[:, None] ** -0.5 * np.ones(nc)[None, :]).ravel(), 3.0)
    ctx.set_model(m)
    g = ctx.trace_image(T, 3.0, math.radians(30.0), npixel=32, nint=800, nphi=45, nr=2, seed=3, linear=False)
    n = (g["info"][0] - 1) * 45 * 800
    assert n > (1 << 23)
    ih, fh, _, _ = H.trace_image(m, T, 3.0, math.radians(30.0), 32, 800, float(m.R[-1]), seed=3, linear=0, nphi=45,
                                 nj0=2)
    assert g["flux"] == fh
    assert np.array_equal(g["image"], ih)


def test_trace_image_rejects_bad_sizes(ctx):
    """sizes outside the documented limits come back as errors before any
    device work; the context stays usable"""
    from mcmax_b200.api import McgError
    m = models.small_disk(nrad=12, ntheta=8, nlam=20, mdust=1e-5)
    ctx.set_model(m)
    T = np.full(m.ncell, 100.0)
    for kw in (dict(npixel=0), dict(npixel=9000), dict(nint=0), dict(Rmax=-1.0), dict(Rmax=0.0)):
        with pytest.raises(McgError):
            ctx.trace_image(T, 3.0, 0.5, **dict(dict(npixel=16, nint=2), **kw))
    g = ctx.trace_image(T, 3.0, 0.5, npixel=16, nint=2)
    assert np.all(np.isfinite(g["image"])) and g["image"].sum() > 0
