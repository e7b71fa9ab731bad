"""The surrogate's Mueller matrix from Legendre moments (surrogate_phase.h,
built for the host): the plain clipped series, the delta-M form (Wiscombe
1977) that keeps the asymmetry parameter of forward-peaked grains, and the
constraints of any mixture of spheres.  Moments of exact ComputePart rows
come from the oracle."""
import numpy as np
import pytest

import hostcheck_ffi as H
import oracle_ffi as O

NA, L = 180, 12
TH = np.pi * (np.arange(NA) + 0.5) / NA
MU, W = np.cos(TH), np.sin(TH)
PL = np.zeros((L + 1, NA))
PL[0], PL[1] = 1.0, MU
for _l in range(1, L):
    PL[_l + 1] = ((2 * _l + 1) * MU * PL[_l] - _l * PL[_l - 1]) / (_l + 1)


def moments(F):
    """chi, beta, gamma, delta of an exact row F[6][180], as the surrogate's
    training targets define them"""
    s0 = np.sum(F[0] * W)
    return [np.array([np.sum(F[e] * W * PL[l]) / s0 for l in range(L + 1)]) for e in (0, 1, 3, 4)]


def g_of(f11):
    return np.sum(f11 * MU * W) / np.sum(f11 * W)


def plain_series(chi, beta, gam, dlt):
    """the clipped series without delta-M, restated in NumPy"""
    c2 = (2 * np.arange(L + 1) + 1)[:, None]
    a = np.maximum(np.sum(c2 * chi[:, None] * PL, 0), 0.0)
    b, g, d = (np.sum(c2 * m[:, None] * PL, 0) for m in (beta, gam, dlt))
    c = np.sum(W) / np.sum(a * W)
    a, b, g, d = a * c, b * c, g * c, d * c
    b = np.clip(b, -a, a)
    room, gd = a * a - b * b, g * g + d * d
    s = np.where(gd > room, np.sqrt(np.where(gd > 0, room / np.where(gd > 0, gd, 1.0), 0.0)), 1.0)
    return a, b, g * s, d * s


def check_sphere_constraints(F):
    assert np.all(F[0] >= 0)
    assert np.all(np.abs(F[1]) <= F[0])
    assert np.array_equal(F[2], F[0]) and np.array_equal(F[5], F[3])
    assert np.all(F[1] ** 2 + F[3] ** 2 + F[4] ** 2 <= F[0] ** 2 * (1 + 1e-12) + 1e-300)
    assert abs(np.sum(F[0] * W) / np.sum(W) - 1) < 1e-12


def hg_moments(g, pol=0.3):
    chi = g ** np.arange(L + 1)
    beta = -pol * chi * np.r_[0.0, np.ones(L)] * 0.5
    return chi, beta, chi.copy(), 0.1 * beta


def test_plain_series_is_the_clipped_legendre_sum():
    chi, beta, gam, dlt = hg_moments(0.6)
    F = H.surr_phase(chi, beta, gam, dlt, deltam=0)
    a, b, g, d = plain_series(chi, beta, gam, dlt)
    for got, ref in ((F[0], a), (F[1], b), (F[3], g), (F[4], d)):
        assert np.allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    check_sphere_constraints(F)


# at g = 0.97 the remainder after the delta (g = 0.91) still rings a little
# and is clipped: 0.009 off, against 0.44 for the plain series
@pytest.mark.parametrize("g,tol", [(0.3, 2e-3), (0.8, 2e-3), (0.97, 0.012)])
def test_delta_m_keeps_the_asymmetry_of_a_henyey_greenstein_function(g, tol):
    chi, beta, gam, dlt = hg_moments(g)
    Fd = H.surr_phase(chi, beta, gam, dlt, deltam=1)
    Fp = H.surr_phase(chi, beta, gam, dlt, deltam=0)
    check_sphere_constraints(Fd)
    check_sphere_constraints(Fp)
    assert abs(g_of(Fd[0]) - g) < tol, (g_of(Fd[0]), g)
    if g > 0.9:
        # the clipped series loses most of the forward scattering
        assert g_of(Fp[0]) < g - 0.2


def test_delta_m_on_exact_rows_of_forward_peaked_grains():
    """ComputePart rows (oracle) of large grains at short wavelengths, where
    the plain series loses up to 0.4 of the asymmetry parameter"""
    lam = np.array([0.1, 0.3, 1.0, 3.0, 10.0])
    n, k = 1.7 + 0 * lam, 0.03 + 0 * lam
    dg_dm, dg_plain = [], []
    for amin, amax in ((1.0, 3.0), (10.0, 30.0), (100.0, 300.0)):
        r = O.compute_part(lam, n, k, np.ones(1), np.full(1, 3.0), amin, amax, 3.5, 0.8, True, 0.25, 3, 6)
        for j in range(lam.size):
            F = r["F"][j]
            m = moments(F)
            g0 = g_of(F[0])
            Fd = H.surr_phase(*m, deltam=1)
            check_sphere_constraints(Fd)
            dg_dm.append(abs(g_of(Fd[0]) - g0))
            dg_plain.append(abs(g_of(H.surr_phase(*m, deltam=0)[0]) - g0))
    dg_dm, dg_plain = np.array(dg_dm), np.array(dg_plain)
    assert np.median(dg_dm) < 1e-3 and dg_dm.max() < 0.03, dg_dm
    assert dg_plain.max() > 0.1 and dg_dm.max() < 0.2 * dg_plain.max(), (dg_plain, dg_dm)


def test_delta_fraction_bounds():
    chi = np.r_[1.0, np.full(L, 0.999)]
    F = H.surr_phase(chi, np.zeros(L + 1), chi, np.zeros(L + 1), deltam=1)
    check_sphere_constraints(F)
    # f is capped at 0.99: the first bin holds at least that share of the weight
    assert F[0, 0] * W[0] / np.sum(W) >= 0.99 - 1e-12
    # no delta when the last moments are not positive
    chi = np.r_[1.0, 0.5, 0.2, np.zeros(L - 2)]
    Fd = H.surr_phase(chi, np.zeros(L + 1), chi, np.zeros(L + 1), deltam=1)
    Fp = H.surr_phase(chi, np.zeros(L + 1), chi, np.zeros(L + 1), deltam=0)
    assert np.array_equal(Fd, Fp)


def test_oracle_transport_with_delta_m_matrices_conserves_energy():
    """A delta-M matrix puts a large value in the first angle bin; the
    transport's angle tables take it like any other row: every run ends,
    and the escaping energy is the star's (the model's matrices replaced by
    their delta-M rebuilds from 12 moments)."""
    import models
    from mcmax_b200 import model as M
    m = models.small_disk(nrad=20, ntheta=12, nlam=24, mdust=1e-4, amin=1.0, amax=30.0)
    F = m.F.copy()
    fmax = 0.0
    for c in range(F.shape[0]):
        for l in range(F.shape[1]):
            mom = moments(m.F[c, l])
            chi = mom[0]
            if chi[L - 1] > 0 and chi[L] > 0:
                fmax = max(fmax, min(chi[L] ** 2 / chi[L - 1], chi[L]))
            F[c, l] = H.surr_phase(*mom, deltam=1)
            check_sphere_constraints(F[c, l])
    assert fmax > 0.3  # rows with a strong forward delta are in the model
    out = O.mcradiation(M.Model(**{**m.__dict__, "F": F}), 20000, seed=5)
    assert out["status"] == 0
    nu = m.nu
    dn = np.empty_like(nu)
    dn[0], dn[-1], dn[1:-1] = nu[1] / 2, (nu[-1] - nu[-2]) / 2, (nu[2:] - nu[:-2]) / 2
    cos = np.arange(31) / 30.0
    wang = 1.0 / (cos[1:] - cos[:-1])
    e = out["spec"][:, 1:] / ((-1e23 / dn)[:, None] * wang[None, :])
    assert abs(e.sum() / m.Lstar - 1) < 0.02
    assert np.all(np.isfinite(out["EJv"])) and np.all(out["EJv"] >= 0)
