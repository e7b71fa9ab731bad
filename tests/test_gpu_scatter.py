"""The ray tracer's scattered light on the GPU (scatfield.cu: TraceMono,
TraceMono.f:583-914, as warp-cooperative packet kernels) against the
oracle's serial restatement on the same Philox streams.  The packets follow
the same paths, so the fields agree to the rounding of the order in which
the lanes' atomics add the deposits (a rare 1-ulp difference between
CUDA's and the C library's acos could move one deposit to a neighbouring
bin; none shows at these sizes).  Spectra and images with the scattered
source then agree to rounding."""
import math

import numpy as np
import pytest

import models
import oracle_ffi as O

pytestmark = pytest.mark.gpu


def _field_close(a, b):
    scale = np.abs(b).max()
    assert np.allclose(a, b, rtol=1e-9, atol=1e-13 * scale), np.abs(a - b).max() / scale


@pytest.mark.parametrize("scat_how", [2, 1])
def test_field_matches_oracle(ctx, scat_how):
    m = models.small_disk(nrad=12, ntheta=8, nlam=24, ngrains=2, ns=2, nf=3, mdust=1e-4, scat_how=scat_how)
    rng = np.random.default_rng(3)
    T = rng.uniform(50.0, 800.0, m.ncell)
    ctx.set_model(m)
    for lam0, ang, nexits in ((1.0, 45.0, 5), (0.3, 80.0, 0), (20.0, 20.0, 3)):
        g, info = ctx.scatter_field(T, lam0, math.radians(ang), nphot=3000, nphot_star=2000, seed=11, nexits=nexits)
        o, oinfo = O.scatter_field(m, T, lam0, math.radians(ang), nphot=3000, nphot_star=2000, seed=11, nexits=nexits)
        assert info["mode"] == scat_how and info["nsub"] == int(oinfo[0])
        assert (info["geometry_failures"], info["interaction_cap"], info["no_start"]) == tuple(int(x) for x in oinfo[1:])
        assert g[..., 0].sum() > 0
        _field_close(g, o)


def test_spectrum_and_image_with_scattered_light_match_oracle(ctx):
    m = models.small_disk(nrad=12, ntheta=8, nlam=24, ngrains=2, ns=2, nf=3, mdust=1e-4)
    T = np.full(m.ncell, 300.0)
    ctx.set_model(m)
    sc = dict(nphot=2000, nphot_star=2000, seed=5, nexits=5)
    lam = np.array([0.4, 1.0, 3.0, 12.0])
    ang = math.radians(60)
    f0, _ = ctx.trace_spectrum(T, lam, ang)
    f1, (nr, bad) = ctx.trace_spectrum(T, lam, ang, scatter=sc)
    o1, onr, obad = O.trace_spectrum(m, T, lam, ang, scatter=sc)
    assert (nr, bad) == (onr, obad) and bad == 0
    assert np.allclose(f1, o1, rtol=1e-9, atol=0)
    assert np.all(f1 > f0)
    r = ctx.trace_image(T, 1.0, ang, npixel=48, nint=20, seed=9, scatter=sc)
    oim, oflux, _, _ = O.trace_image(m, T, 1.0, ang, 48, 20, float(m.R[-1]), seed=9, linear=1, scatter=sc)
    assert abs(r["flux"] / oflux - 1) < 1e-9
    assert np.allclose(r["image"], oim, rtol=1e-8, atol=1e-12 * oim.max())


def test_isotropic_spectrum_caches_grid_wavelength_fields(ctx):
    """isotropic scattering stores one field per grid wavelength
    (TraceMono.f:90-160): the spectrum at wavelengths between two grid
    points interpolates the two fields, as the oracle does"""
    m = models.small_disk(nrad=12, ntheta=8, nlam=24, ngrains=2, ns=2, nf=3, mdust=1e-4, scat_how=1)
    T = np.full(m.ncell, 300.0)
    ctx.set_model(m)
    sc = dict(nphot=2000, nphot_star=1000, seed=8, nexits=5)
    lam = np.sqrt(m.lam[3:7] * m.lam[4:8])
    f1, _ = ctx.trace_spectrum(T, lam, math.radians(30), scatter=sc)
    o1, _, _ = O.trace_spectrum(m, T, lam, math.radians(30), scatter=sc)
    assert np.allclose(f1, o1, rtol=1e-9, atol=0)
