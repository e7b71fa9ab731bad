"""mcg_trace_spectrum on the GPU against the host replay of the same host
logic and per-ray arithmetic, bit for bit (the unit is built with
--fmad=false, the replay with -ffp-contract=off, and the ray set-up and
attenuation use detmath.h)."""
import math

import numpy as np
import pytest

import hostcheck_ffi as H
import models

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
