"""The oracle's scattered-light field of the ray tracer (orc_scatter_field,
the restatement of TraceMono, TraceMono.f:583-914) on CPU, against the
physics it estimates: in an optically thin disk the single-scattered
starlight field of a cell, sum over packets of E x path length, is the
stellar flux at the cell times its volume, Estar V / (4 pi r^2); the
sub-cone grid of a full-Mueller field follows Telescope.f:93-110; and the
scattered light raises the ray-traced flux where the star dominates."""
import math

import numpy as np

import models
import oracle_ffi as O

AU = float(np.float32(1.49598e13))


def _thin(scat_how=1):
    return models.small_disk(nrad=10, ntheta=6, nlam=16, ngrains=2, ns=2, nf=3, mdust=1e-14, scat_how=scat_how)


def test_starlight_field_of_a_thin_disk_is_flux_times_volume():
    m = _thin(1)
    T = np.full(m.ncell, 50.0)
    lam0 = 0.5
    SF, info = O.scatter_field(m, T, lam0, math.radians(45), nphot=0, nphot_star=200000, seed=7, nexits=0)
    assert info.tolist() == [m.nt - 1, 0, 0, 0]
    nc = m.nt - 1
    tot = SF[..., 0].sum(axis=2).reshape(m.nr, nc)           # both sides: sum of E v AU
    l = int(np.searchsorted(m.lam, lam0)) - 1
    w2 = (lam0 - m.lam[l]) / (m.lam[l + 1] - m.lam[l])
    Estar = m.Fstar[l] * (1 - w2) + m.Fstar[l + 1] * w2
    # every packet crosses every shell once, radially far from the star:
    # the shell collects Estar dR (a little more for the slanted paths)
    dR = (m.R[2:] - m.R[1:-1]) * AU
    shell = tot[1:].sum(1) / (Estar * dR)
    assert np.all(shell > 1.0 - 1e-5) and np.all(shell < 1.0 + 2e-4), shell
    # and each cell its share of the shell's volume, within the noise
    V = m.V.reshape(m.nr, nc)
    share = tot[1:] / (Estar * dR[:, None] * V[1:] / V[1:].sum(1, keepdims=True))
    assert np.all(np.abs(share - 1) < 0.1), share


def test_full_mueller_sub_cones():
    m = _thin(2)
    SF, info = O.scatter_field(m, np.full(m.ncell, 50.0), 1.0, math.radians(30), nphot=200, nphot_star=200, seed=1)
    th = np.arccos(np.asarray(m.Theta, float))
    th[0], th[-1] = 0.0, math.pi / 2
    nrg = [max(1, int((th[j] - th[j - 1]) * 270.0 / math.pi)) for j in range(1, m.nt)]
    assert SF.shape == (m.nr, sum(nrg), 2, 91) and int(info[0]) == sum(nrg) and max(nrg) > 1
    assert np.all(SF >= 0) and SF[..., 0].sum() > 0 and SF[..., 1:].sum() > 0
    assert int(info[1]) == 0 and int(info[3]) == 0


def test_scattered_light_adds_to_the_spectrum():
    m = models.small_disk(nrad=12, ntheta=8, nlam=24, ngrains=2, ns=2, nf=3, mdust=1e-4)
    T = np.full(m.ncell, 300.0)
    lam = np.array([0.5, 1.0])
    f0, _, _ = O.trace_spectrum(m, T, lam, math.radians(60))
    f1, _, bad = O.trace_spectrum(m, T, lam, math.radians(60), scatter=dict(nphot=500, nphot_star=500, seed=2))
    assert bad == 0 and np.all(f1 > f0) and np.all(f1 < 2 * f0)
