"""The vertical structure step (DiskStructure, DiskStructure.f:85-468) on
CPU: the host logic of mcg_disk_structure with its kernels replaced by
serial loops over the same per-column and per-cell functions
(tests/native/hostcheck.cpp) against the oracle's restatement in the
reference's loop order (oracle/oracle_dstruct.c), bit for bit, and against
closed forms of hydrostatic equilibrium."""
import math

import numpy as np
import pytest

import hostcheck_ffi as H
import models
import oracle_ffi as O
from mcmax_b200 import model as M
from mcmax_b200.api import shtype_codes

MU, G, KB = float(np.float32(2.3)) * 1.67262158e-24, 6.67300e-8, 1.3806503e-16
SH = 0.05 * math.sqrt(2.0)


@pytest.fixture(scope="module")
def disk():
    m = models.small_disk(nrad=20, ntheta=14, nlam=16, mdust=1e-4, ngrains=2)
    dens = np.maximum(m.dens, 1e-50)
    state = dict(dens=dens.copy(), dens0=dens.copy(), gasdens=dens.copy(), w=m.comp_w.copy(), w0=m.comp_w.copy())
    return m, state


def _st(m, zones, **kw):
    d = dict(nr=m.nr, nt=m.nt, ng=m.ncomp, R=m.R, Theta=m.Theta, V=m.V, Mstar=2.5 * M.MSUN, zones=zones)
    d.update(kw)
    return d


def _temp(m, vertical=0.5):
    nc = m.nt - 1
    R_av = np.sqrt(m.R[:-1] * m.R[1:])
    return np.maximum((300.0 * R_av[:, None] ** -0.5 * (1 + vertical * np.linspace(1, 0, nc))[None, :]).ravel(), 2.7)


def _run(fn, st, T, s):
    return dict(zip(("dens", "dens0", "gasdens", "w", "w0"),
                    fn(st, T, s["dens"], s["dens0"], s["gasdens"], s["w"], s["w0"])))


def _geometry(m):
    nc = m.nt - 1
    R_av = M.AU * 10 ** ((np.log10(m.R[:-1]) + np.log10(m.R[1:])) / 2)
    th = np.arccos((m.Theta[:-1] + m.Theta[1:]) / 2)
    return R_av, th, nc


@pytest.mark.parametrize("fix", [0, 1])
def test_replay_matches_oracle_and_keeps_ring_masses(disk, fix):
    m, s = disk
    st = _st(m, [(0.5, 100.0, SH, 1.0, 1.125, 1.0, fix)])
    T = _temp(m)
    o = _run(O.disk_structure, st, T, s)
    h = _run(H.disk_structure, st, T, s)
    for k in o:
        assert np.array_equal(o[k], h[k]), k
    nc = m.nt - 1
    V = m.V.reshape(m.nr, nc)
    for name, new, old in (("gas", h["gasdens"], s["gasdens"]), ("condensable", h["dens0"], s["dens0"])):
        r = (new.reshape(m.nr, nc) * V).sum(1)[1:] / (old.reshape(m.nr, nc) * V).sum(1)[1:]
        assert np.allclose(r, 1.0, rtol=1e-12, atol=0), name
    assert np.allclose(h["w"].reshape(-1, m.ncomp).sum(1), 1.0, rtol=1e-12)


def test_isothermal_column_is_gaussian(disk):
    """constant T: ln rho = -mu G M z^2 / (2 k T R^3) + const"""
    m, s = disk
    st = _st(m, [(0.5, 100.0, SH, 1.0, 1.125, 1.0, 0)])
    T = np.full(m.ncell, 3000.0)
    h = _run(H.disk_structure, st, T, s)
    R_av, th, nc = _geometry(m)
    gas = h["gasdens"].reshape(m.nr, nc)
    for i in (8, 15, 19):
        z = R_av[i] * np.cos(th)
        lnr = -MU * G * st["Mstar"] * z ** 2 / (2 * KB * 3000.0 * R_av[i] ** 3)
        got = np.log(gas[i] / gas[i, -1])
        ok = gas[i] > 1e-45
        assert ok.sum() >= 3
        err = np.abs(got[ok] - (lnr[ok] - lnr[-1]))
        assert np.all(err < 1e-5 * np.maximum(1.0, np.abs(lnr[ok]))), (i, err)


def test_settling_factor_narrows_a_grain(disk):
    """a grain with scale-height factor f follows the gas profile with z/f"""
    m, s = disk
    gs = np.ones((m.ncomp, m.nr))
    gs[1] = 0.5
    st = _st(m, [(0.5, 100.0, SH, 1.0, 1.125, 1.0, 0)], grain_scale=gs)
    T = np.full(m.ncell, 3000.0)
    o = _run(O.disk_structure, st, T, s)
    h = _run(H.disk_structure, st, T, s)
    for k in o:
        assert np.array_equal(o[k], h[k]), k
    R_av, th, nc = _geometry(m)
    i = 19
    z = R_av[i] * np.cos(th)
    d1 = (h["dens0"] * h["w0"][:, 1]).reshape(m.nr, nc)[i]
    lnr = -MU * G * st["Mstar"] * z ** 2 / (2 * KB * 3000.0 * R_av[i] ** 3 * 0.25)
    ok = d1 > 1e-45
    assert ok.sum() >= 2
    got = np.log(d1[ok] / d1[-1])
    assert np.all(np.abs(got - (lnr[ok] - lnr[-1])) < 1e-5 * np.maximum(1.0, np.abs(lnr[ok])))


def test_fixed_zone_profile(disk):
    """a fixed-structure zone keeps rho ~ r^-p / h exp(-(z/h)^2), h = sh (r/Rsh)^q,
    renormalised per ring (DiskStructure.f:360-386)"""
    m, s = disk
    st = _st(m, [(0.5, 100.0, SH, 1.0, 1.125, 1.0, 1)])
    h = _run(H.disk_structure, st, _temp(m), s)
    R_av, th, nc = _geometry(m)
    i = 10
    rr = R_av[i] * np.sin(th) / M.AU
    zz = R_av[i] * np.cos(th) / M.AU
    hr = SH * rr ** 1.125
    prof = rr ** -1.0 / hr * np.exp(-(zz / hr) ** 2 * (np.arange(nc) != nc - 1))
    prof = prof / (prof * m.V.reshape(m.nr, nc)[i]).sum()
    got = h["gasdens"].reshape(m.nr, nc)[i]
    got = got / (got * m.V.reshape(m.nr, nc)[i]).sum()
    big = prof > 1e-40
    assert np.allclose(got[big], prof[big], rtol=1e-12)


def test_wedge_zone_and_ring_factors(disk):
    m, s = disk
    shs = np.linspace(0.8, 1.2, m.nr)
    st = _st(m, [(0.5, 10.0, -30.0, 1.0, 1.0, 1.0, 1), (10.0, 100.0, SH, 1.0, 1.125, 1.0, 0)], shscale=shs)
    T = _temp(m)
    o = _run(O.disk_structure, st, T, s)
    h = _run(H.disk_structure, st, T, s)
    for k in o:
        assert np.array_equal(o[k], h[k]), k
    R_av, th, nc = _geometry(m)
    inner = np.nonzero((R_av > 0.5 * M.AU) & (R_av < 10 * M.AU))[0][1]
    g = h["gasdens"].reshape(m.nr, nc)[inner]
    open_ = 180 * th[:-1] / np.pi > 30.0
    assert np.allclose(g[:-1][open_], g[-1], rtol=1e-12)
    assert np.all(g[:-1][~open_] < 1e-20 * g[-1])


SHAPES = ("DISK", "ZODI", "HALO", "LOBE", "JET", "SHELL", "CYLI", "CAVITY", "WEDGE", "KEEP")


def _shape_case():
    """one grain of every scale-height type, with the factors the closed
    forms read: HALO a wedge (negative factor), LOBE 30 degrees, JET 20,
    SHELL 2, CYLI 3 AU, CAVITY 0.3, WEDGE 60 degrees"""
    m = models.small_disk(nrad=20, ntheta=14, nlam=16, mdust=1e-4, ngrains=len(SHAPES))
    dens = np.maximum(m.dens, 1e-50)
    w = m.comp_w.copy()
    state = dict(dens=dens.copy(), dens0=dens.copy(), gasdens=dens.copy(), w=w.copy(), w0=w.copy())
    gs = np.ones((m.ncomp, m.nr))
    for k, f in ((2, -0.5), (3, 30.0), (4, 20.0), (5, 2.0), (6, 3.0), (7, 0.3), (8, 60.0)):
        gs[k] = f
    st = _st(m, [(0.5, 100.0, SH, 1.0, 1.125, 1.0, 0)], grain_scale=gs, shtype=np.arange(len(SHAPES), dtype=np.int32))
    return m, state, st, gs


def test_scale_height_types_match_oracle_and_closed_forms():
    """DiskStructure.f:248-344: each grain's new profile along theta is its
    type's closed form, renormalised to the grain's mass in the ring; the
    host logic and the oracle agree bit for bit"""
    m, s, st, gs = _shape_case()
    T = _temp(m)
    o = _run(O.disk_structure, st, T, s)
    h = _run(H.disk_structure, st, T, s)
    for k in o:
        assert np.array_equal(o[k], h[k]), k
    R_av, th, nc = _geometry(m)
    thet = np.arccos(m.Theta[:-1])
    V = m.V.reshape(m.nr, nc)
    grain = (h["dens0"][:, None] * h["w0"]).reshape(m.nr, nc, m.ncomp)
    old = (s["dens"][:, None] * s["w"]).reshape(m.nr, nc, m.ncomp)
    deg = np.degrees(th)
    for i in (5, 12, 19):
        z = R_av[i] * np.cos(th) / M.AU
        rc = R_av[i] * np.sin(th) / M.AU
        expect = {
            1: 0.15 + 0.85 * np.cos(np.pi / 2 - th) ** 28,
            2: np.where(np.pi / 2 - th > 0.5, 0.0, 1.0),
            3: np.exp(-(deg / 30.0) ** 2 / math.log(10.0)),
            4: np.exp(-(np.degrees(thet) / (20.0 * R_av[i] / R_av[-1])) ** 2),
            5: 1.0 + 2.0 * np.sin(th) ** 3,
            6: np.where((z < 3.0) | (np.arange(nc) == nc - 1), 1.0, 0.0),
            7: np.where(np.arange(nc) == nc - 1, 1.0,
                        np.where((np.arange(nc) > 0) & (z < rc ** 2 * 0.3), 1.0, 0.0)),
            8: np.where(deg > 60.0, 1.0, 0.0),
            9: old[i, :, 9],
        }
        for k, e in expect.items():
            e = e * (old[i, :, k] * V[i]).sum() / (e * V[i]).sum()
            got = grain[i, :, k]
            big = e > 1e-30 * e.max()
            assert np.allclose(got[big], e[big], rtol=1e-9), (SHAPES[k], i)
            assert np.all(got[~big] < 1e-20 * e.max()), (SHAPES[k], i)


def test_scale_height_names_map_to_codes():
    from mcmax_b200.api import McgError, shtype_codes
    assert list(shtype_codes(["disk", "ZODI", "Halo", "lobe", "JET", "shell", "CYLI", "CAVITY", "WEDGE", "SPIRAL"],
                             10)) == list(range(10))
    with pytest.raises(McgError):
        shtype_codes(["DISK"], 2)


# ---------------------------------------------------------------- the iteration driver
from mcmax_b200 import structure as S  # noqa: E402


def test_temp_average_and_compare_cells():
    T0 = np.array([10.0, 2.0, 5.0])
    assert np.array_equal(S.temp_average(None, T0, 0.5), T0)
    assert np.allclose(S.temp_average(T0, [20.0, 1.0, 5.0], 0.5), [15.0, 2.35, 5.0])
    nr, nt = 3, 3          # 3 rings x 2 theta cells; ring 0 is left out
    T1 = np.array([1, 1, 10, 10, 20, 20.0])
    T2 = np.array([1, 1, 12, 10, 20, 23.0])
    dT = np.ones(6)
    dT2 = dT.copy()
    dT2[5] = 0.0           # no error estimate: cell left out
    err = S.compare_cells(T1, dT, T2, dT2, nr, nt)
    assert abs(err - (4.0 / 2.0) / (2 * 2 - 1)) < 1e-15


class _FakeRun:
    """packet loop stand-in: the temperatures it returns are set by the
    test; the structure step is the host replay of mcg_disk_structure"""

    def __init__(self, temps):
        self.temps = list(temps)
        self.calls = dict(mc=0, ds=0, diffuse=0)
        self.dens_seen = []
        self.grain_scales = []

    def set_model(self, m):
        self.model = m
        self.dens_seen.append(np.array(m.dens))

    def mcradiation(self, nphot, **kw):
        self.calls["mc"] += 1
        return nphot, dict(Ni=np.full(self.model.ncell, 1000, np.int32))

    def finalize_t(self):
        T = self.temps[min(self.calls["mc"], len(self.temps)) - 1]
        return T.copy(), np.ones_like(T), np.zeros_like(T)

    def diffuse(self, Ni, dT, T, nphotmin, dtmax, factRW):
        self.calls["diffuse"] += 1
        return T, None, (0, 0, 0, 0)

    def disk_structure(self, R, Theta, V, Mstar, zones, Temp, dens, dens0, gasdens, w, w0, shscale=None,
                       grain_scale=None, shtype=None):
        self.calls["ds"] += 1
        self.grain_scales.append(grain_scale)
        st = dict(nr=R.size - 1, nt=Theta.size, ng=np.asarray(w).shape[1], R=R, Theta=Theta, V=V, Mstar=Mstar,
                  zones=zones, shscale=shscale, grain_scale=grain_scale,
                  shtype=None if shtype is None else shtype_codes(shtype, np.asarray(w).shape[1]))
        out = H.disk_structure(st, Temp, dens, dens0, gasdens, np.ravel(w), np.ravel(w0))
        ncell = np.asarray(dens).size
        return out[0], out[1], out[2], out[3].reshape(ncell, -1), out[4].reshape(ncell, -1)


def _driver_model():
    m = models.small_disk(nrad=20, ntheta=14, nlam=16, mdust=1e-4, ngrains=2)
    return M.Model(**dict(m.__dict__, dens=np.maximum(m.dens, 1e-50).copy(), comp_w=m.comp_w.copy()))


def test_iterations_stop_after_two_agreeing_passes():
    m = _driver_model()
    T = _temp(m)
    fake = _FakeRun([T])
    zones = [(0.5, 100.0, SH, 1.0, 1.125, 1.0, 0)]
    r = S.iterate(fake, m, zones, 2.5 * M.MSUN, 1000)
    # pass 1 has no previous temperatures (errT 0), pass 2 agrees, then one last run
    assert [h["niter"] for h in r["history"]] == [1, 2]
    assert fake.calls == dict(mc=3, ds=2, diffuse=3)
    assert not np.array_equal(fake.dens_seen[1], fake.dens_seen[0])
    assert np.array_equal(m.dens, r["state"]["dens"])


def test_iterations_stop_at_maxiter():
    m = _driver_model()
    T = _temp(m)
    fake = _FakeRun([T, T + 10.0, T, T + 10.0, T, T + 10.0])
    r = S.iterate(fake, m, [(0.5, 100.0, SH, 1.0, 1.125, 1.0, 0)], 2.5 * M.MSUN, 1000, maxiter=3)
    assert [h["niter"] for h in r["history"]] == [1, 2, 3, 4]
    assert all(h["errT"] > 3.0 for h in r["history"][1:])
    assert fake.calls["mc"] == 5 and fake.calls["ds"] == 4
    # the structure temperature averages the passes with weight f_weight = 0.5
    assert np.allclose(r["Temp"], 0.5 * (0.5 * (0.5 * T + 0.5 * (T + 10)) + 0.5 * T) + 0.5 * (T + 10), rtol=1e-12)


def test_thin_temperatures_follow_determine_t():
    """OpticallyThin's cell temperatures: the absorbed dilute stellar field
    inverted on each cell's Planck-mean table with determineT's bracket and
    T^4 interpolation; the oracle's determineT on the same table gives the
    same bits"""
    m = _driver_model()
    Kp, kps = S.planck_means(m)
    T = S.thin_temperature(m, Kp, kps)
    w = m.comp_w.reshape(m.ncell, m.ncomp)
    nc = m.nt - 1
    R = np.asarray(m.R)
    for c in range(0, m.ncell, 7):
        i = c // nc
        r = (R[1] if i == 0 else R[i]) * M.AU
        W = 0.5 * (1.0 - math.sqrt(1.0 - (m.Rstar_cm / r) ** 2))
        E = 0.0
        for k in range(m.ncomp):
            E = E + kps[k] * w[c, k]
        E = W * E * m.Lstar / (math.pi * m.Rstar_cm ** 2) / w[c].sum()
        kp = np.zeros(S.TMAX + 1)
        for k in range(m.ncomp):
            kp = kp + Kp[k] * w[c, k]
        kp = np.ascontiguousarray(kp)
        assert T[c] == O.load().orc_determine_t(O.P(kp), E, 100.0), c
    # hotter inside, and below the star
    Tr = T.reshape(m.nr, nc)[:, -1]
    assert np.all(np.diff(Tr[1:]) < 0) and Tr[1] < m.Tstar


def test_thin_temperature_of_a_grey_grain():
    """with a wavelength-independent opacity, sum Kp(T) = W sum Kpabsstar
    gives int B(T) = W int B(Tstar) on the grid: T = W^(1/4) Tstar where
    the grid holds both Planck curves"""
    m = _driver_model()
    m = M.Model(**dict(m.__dict__, Kabs=np.ones_like(m.Kabs)))
    T = S.thin_temperature(m).reshape(m.nr, m.nt - 1)
    R = np.asarray(m.R)
    for i in (3, 8, 15):
        W = 0.5 * (1.0 - math.sqrt(1.0 - (m.Rstar_cm / (R[i] * M.AU)) ** 2))
        assert abs(T[i, 0] / (W ** 0.25 * m.Tstar) - 1.0) < 0.02, (i, T[i, 0], W ** 0.25 * m.Tstar)


def test_thin_start_runs_three_structure_passes():
    m = _driver_model()
    T = _temp(m)
    fake = _FakeRun([T])
    zones = [(0.5, 100.0, SH, 1.0, 1.125, 1.0, 0)]
    thin = S.thin_temperature(m)
    st = S.thin_start(fake, m, zones, 2.5 * M.MSUN)
    assert fake.calls["ds"] == 3 and np.array_equal(st["Temp"], thin)
    assert np.array_equal(m.dens, st["state"]["dens"])
    # the ring masses survive the passes
    V = m.V.reshape(m.nr, -1)
    d0 = _driver_model().dens.reshape(m.nr, -1)
    d1 = m.dens.reshape(m.nr, -1)
    assert np.allclose((d1 * V).sum(1)[1:], (d0 * V).sum(1)[1:], rtol=1e-10)
    fake2 = _FakeRun([T])
    r = S.iterate(fake2, _driver_model(), zones, 2.5 * M.MSUN, 1000, thin=True)
    assert fake2.calls["ds"] == 3 + len(r["history"])


def test_mp_settling_factors():
    """MPSettling's factor h / sqrt(1 + h^2), h = (1/3)^(1/4) sqrt(alpha /
    (Omega tau_f)), tau_f = rho_grain rv / (c_s rho_gas) at the midplane:
    near 1 for small grains, small for large ones"""
    m = _driver_model()
    st = S.initial_state(m)
    T = _temp(m)
    nr, nc = m.nr, m.nt - 1
    rho = np.array([3.0, 3.0])
    rv = np.array([1e-5, 1e-1])
    alpha = np.full(nr, 1e-3)
    sc = S.mp_settling(m, st, T, 2.5 * M.MSUN, rho, rv, alpha)
    assert sc.shape == (m.ncomp, nr) and np.all(sc[:, 0] == 1.0)
    assert np.all(sc[0, 1:] > 0.9) and np.all(sc[1, 1:] < sc[0, 1:])
    R_av = M.AU * 10.0 ** ((np.log10(m.R[:-1]) + np.log10(m.R[1:])) / 2.0)
    d = st["dens"].reshape(nr, nc)
    for i in (3, 10):
        cs = math.sqrt(1.3806503e-16 * T.reshape(nr, nc)[i, -1] / (float(np.float32(2.3)) * 1.66053886e-24))
        tauf = rho[1] * rv[1] / (cs * d[i, -1] * 100.0)
        om = math.sqrt(6.672e-8 * 2.5 * M.MSUN / R_av[i] ** 3)
        h = (1.0 / 3.0) ** 0.25 * math.sqrt(1e-3 / (om * tauf))
        assert abs(sc[1, i] / (h / math.sqrt(1 + h * h)) - 1) < 1e-10


def test_settling_factors_reach_each_structure_pass():
    m = _driver_model()
    T = _temp(m)
    seen = []

    class Fake(_FakeRun):
        def disk_structure(self, *a, **kw):
            seen.append(a[12] if len(a) > 12 else kw.get("grain_scale"))
            return super().disk_structure(*a, **kw)

    fake = Fake([T])
    zones = [(0.5, 100.0, SH, 1.0, 1.125, 1.0, 0)]
    settling = dict(rho=np.array([3.0, 3.0]), rv=np.array([1e-5, 1e-2]), alpha=np.full(m.nr, 1e-4))
    S.iterate(fake, m, zones, 2.5 * M.MSUN, 1000, thin=True, settling=settling)
    assert len(seen) == fake.calls["ds"] and all(g is not None and g.shape == (2, m.nr) for g in seen)
    assert all(np.all(g[1, 1:] < g[0, 1:]) for g in seen)


def test_fixed_settling_factors_match_the_start_settling():
    """FixedMPSettling's factors from the structure state equal those the
    fixed-zone settling of the deck set-up applies (the same surface
    density and grain stopping parameter); larger grains settle more"""
    m = _driver_model()
    st = S.initial_state(m)
    nr, nc = m.nr, m.nt - 1
    rho = np.array([3.0, 2.0])
    rv = np.array([1e-5, 1e-2])
    sc = S.fixed_settling(m, st, rho, rv, 1e-4)
    assert sc.shape == (m.ncomp, nr) and np.all(sc[:, 0] == 1.0)
    assert np.all(sc[1, 1:] < sc[0, 1:])
    V = m.V.reshape(nr, nc)
    d = st["dens"].reshape(nr, nc)
    for i in (4, 11):
        sigma = (d[i] * 100.0 * V[i]).sum() / (math.pi * (m.R[i + 1] ** 2 - m.R[i] ** 2) * M.AU ** 2)
        for k in range(2):
            hH = (1.0 / 3.0) ** 0.25 * math.sqrt(1e-4 * sigma / (math.sqrt(2 * math.pi) * rho[k] * rv[k]))
            assert abs(sc[k, i] / (hH / math.sqrt(1 + hH * hH)) - 1) < 1e-12


def test_fixed_settling_and_shapes_reach_each_structure_pass():
    m = _driver_model()
    T = _temp(m)
    fake = _FakeRun([T])
    zones = [(0.5, 100.0, SH, 1.0, 1.125, 1.0, 0)]
    fixed = dict(rho=np.array([3.0, 3.0]), rv=np.array([1e-5, 1e-2]), alpha=1e-4)
    passes = []
    S.iterate(fake, m, zones, 2.5 * M.MSUN, 1000, thin=True, fixed=fixed, shtype=["DISK", "DISK"], maxiter=2,
              epsiter=0.0, on_pass=lambda n, res, t: passes.append(n))
    assert len(fake.grain_scales) == fake.calls["ds"] == 3 + 3
    assert all(g is not None and np.all(g[1, 1:] < g[0, 1:]) for g in fake.grain_scales)
    assert passes == [1000] * fake.calls["mc"] and fake.calls["mc"] == 4
