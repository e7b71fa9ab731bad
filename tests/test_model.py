"""Host-side set-up: keyword decks, refractive-index regridding, grids,
densities and size distributions."""
import math
import os

import numpy as np
import pytest

from mcmax_b200 import model as M


def test_parse_deck_surface():
    txt = """* a comment line
Tstar=10000   * inline
rstar = 2.5
computepart01:file='dust.lnk'
scattype='FULL'
NRAD=100
"""
    d = M.parse_deck(txt, overrides=["nrad=200", "factrw=5"])
    assert d["tstar"] == "10000" and d["rstar"] == "2.5"
    assert d["computepart01:file"] == "dust.lnk"
    assert d["scattype"] == "FULL"
    assert d["nrad"] == "200" and M.deck_value(d, "factrw", 10.0) == 5.0
    assert M.deck_value(d, "missing", 3.0) == 3.0


def test_readrefind_regrid_and_extrapolation(tmp_path):
    p = tmp_path / "a.lnk"
    p.write_text("0.1 1.5 0.1\n1.0 1.6 0.05\n10.0 1.8 0.02\n")
    grid = np.array([0.05, 0.1, 0.5, 1.0, 5.0, 10.0, 100.0])
    n, k = M.readrefind(str(p), grid)
    assert n[0] == 1.5 and k[0] == 0.1          # below the table: first row
    assert n[3] == 1.6 and abs(k[3] - 0.05) < 1e-15
    assert 1.5 < n[2] < 1.6                     # log-log interpolation
    assert n[-1] == n[-2] and abs(k[-1] - k[-2] * 10 / 100) < 1e-15  # dielectric extrapolation


def test_particle_file(tmp_path):
    (tmp_path / "a.lnk").write_text("0.1 1.5 0.1\n10 1.6 0.05\n")
    pf = tmp_path / "part.in"
    pf.write_text("* sizes\n5\n20\n'a.lnk'\n1.0 3.0\n")
    ns, nf, mats = M.read_particle_file(str(pf))
    assert ns == 5 and nf == 20 and mats[0][1:] == (1.0, 3.0)
    assert mats[0][0].endswith("a.lnk")


def test_spatial_grid_and_density():
    R, Th, thet, ST = M.spatial_grid(2.5 * M.RSUN, 0.5, 100.0, 20, 12)
    assert R.size == 22 and Th.size == 13
    assert Th[0] == 1.0 and Th[-1] == 0.0 and np.all(np.diff(Th) < 0)
    assert np.all(np.diff(R) > 0) and abs(R[1] - 0.5) < 1e-12 and abs(R[-1] - 100) < 1e-9
    dens, V = M.zones_density(R, Th, thet, [dict(rin=0.5, rout=100, mdust=1e-5, denspow=1, sh=0.07, rsh=1,
                                                 shpow=1.125)])
    mass = (dens[1:] * V[1:]).sum()
    assert abs(mass / (1e-5 * M.MSUN) - 1) < 1e-6
    assert np.all(dens[0] == 1e-60)
    # cells cover one hemisphere and count its mirror (Init.f:3073): the
    # volumes add up to the full spherical shell
    vol = V.sum()
    full = 4 * math.pi / 3 * (R[-1] ** 3 - R[0] ** 3) * M.AU ** 3
    assert abs(vol / full - 1) < 1e-12


def test_mrn_abundances():
    bins = M.grain_bins(0.1, 1.0, 20)
    assert abs(bins[0][0] - 0.1) < 1e-15 and abs(bins[-1][1] - 1.0) < 1e-12
    rg = [math.sqrt(a * b) * 1e-4 for a, b in bins]
    w = M.mrn_abundances(rg, 0.1e-4, 1e-4, 3.5)
    assert abs(w.sum() - 1) < 1e-9 and np.all(w > 0)
    assert w[-1] > w[0]  # a^-3.5: mass in the large grains


def test_settling_conserves_each_grain_mass_and_settles_large_grains():
    R, Th, thet, ST = M.spatial_grid(2.5 * M.RSUN, 0.5, 100.0, 24, 16)
    zone = dict(rin=0.5, rout=100, mdust=1e-3, denspow=1.0, sh=0.05 * math.sqrt(2.0), rsh=1.0, shpow=1.125)
    dens, V = M.zones_density(R, Th, thet, [zone])
    ng = 5
    w = np.tile(np.full(ng, 1.0 / ng), (dens.shape[0], dens.shape[1], 1))
    rv = np.array([1e-6, 1e-5, 1e-4, 1e-3, 1e-2])
    d2, w2 = M.fixed_mp_settling(R, Th, 16, dens, V, w, np.full(ng, 3.0), rv, 1e-3, zone)
    assert np.allclose(w2.sum(2), 1.0)
    for ii in range(ng):
        m0 = (dens[1:] * V[1:] * w[1:, :, ii]).sum()
        m1 = (d2[1:] * V[1:] * w2[1:, :, ii]).sum()
        assert abs(m1 / m0 - 1) < 1e-12
    i = 12
    nc = w2.shape[1]
    # an upper cell that still holds dust: the big grains have left it
    upper = [j for j in range(nc - 3) if d2[i, j] * w2[i, j, 0] > 1e-40][-1]
    assert w2[i, upper, -1] < 0.1 * w2[i, upper, 0]
    assert w2[i, nc - 1, -1] > w2[i, nc - 1, 0]   # and collect at the midplane


def test_grain_rv_and_theta_centres():
    assert abs(M.grain_rv(0.5, 0.5, 3.5, 1) - 0.5e-4) < 1e-16
    rv = M.grain_rv(0.1, 1.0, 3.5, 5)
    assert 0.1e-4 < rv < 1.0e-4
    th = M.theta_centres(60)
    assert th.size == 60 and np.all(np.diff(th) > 0) and th[-1] < math.pi / 2


def test_learned_deck_parts():
    lam, _ = M.wavelength_grid(0.1, 3000.0, 12)
    parts, bins = M.learned_disk_parts(lam, ngrains=5)
    assert len(parts) == 15 and len(bins) == 5
    assert abs(bins[0][0] - 0.01) < 1e-12 and abs(bins[-1][1] - 1000.0) < 1e-9
    assert {p["porosity"] for p in parts} == {0.0, 0.2, 0.4}


def test_deck_model_builds_the_disk_model_of_its_keywords(tmp_path):
    import oracle_ffi as O
    lam_tab = np.geomspace(0.05, 5000.0, 80)
    n, k = M.synthetic_lnk(lam_tab, 0.03)
    (tmp_path / "syn.lnk").write_text("".join("%g %g %g\n" % t for t in zip(lam_tab, n, k)))
    (tmp_path / "dust.particle").write_text("2\n3\n'syn.lnk'\n1.0 3.0\n")
    deck = tmp_path / "disk.in"
    deck.write_text("""* a passive disk
tstar=10000
rstar=2.5
startype='PLANCK'
rin=0.5
rout=100
nrad=12
ntheta=8
lam1=0.1
lam2=3000
nlam=20
denstype='ZONES'
zone1:rin=0.5
zone1:rout=100
zone1:mdust=1d-5
zone1:denspow=1
zone1:sh=0.0707
zone1:rsh=1
zone1:shpow=1.125
scattype='FULL'
computepart01:file='dust.particle'
amin=0.1
computepart01:amax=1.0
computepart01:ngrains=3
computepart01:fmax=0.8
computepart01:porosity=0.25
randomwalk=.true.
factrw=5
idum=-7
""")

    def oracle_parts(parts):
        return [O.compute_part(p["lam"], p["e1"][0], p["e2"][0], p["frac"], p["rho"], p["amin"], p["amax"],
                               p["apow"], p["fmax"], p["blend"], p["porosity"], p["ns"], p["nf"]) for p in parts]

    m, run = M.deck_model(None, str(deck), overrides=["maxinteract=20000"], compute_parts=oracle_parts)
    assert (m.nr, m.nt, m.nlam, m.ncomp, m.scat_how) == (13, 9, 20, 3, 2)
    zones = run.pop("zones")
    assert zones == [(0.5, 100.0, 0.0707, 1.0, 1.125, 1.0, False)]
    assert abs(run.pop("Mstar") / (2.5 * M.MSUN) - 1) < 1e-15
    assert run == dict(seed=7, randomwalk=True, factRW=5.0, maxinteract=20000, maxruntime=-1.0, nruns=1, nphotdiffuse=25,
                       dtdiffuse=1.0, maxiter=10, epsiter=3.0, incangle=45.0, outputfits=False, posangle=0.0,
                       iterate=True, thin_start=True, settling=None, fixed=None, vis_norm_fov=True)
    # interstellar reddening of the observed fluxes is not built: the deck is refused
    with pytest.raises(ValueError, match="reddening"):
        M.deck_model(None, str(deck), overrides=["av=1.5"], compute_parts=oracle_parts)
    assert np.allclose(m.comp_w.sum(1), 1.0)
    ref = M.disk_model(None, nrad=12, ntheta=8, nlam=20, lam2=3000.0, mdust=1e-5, sh=0.0707, ngrains=3,
                       opacities=(m.Kabs, m.Ksca, m.F))
    for key in ("R", "Theta", "dens", "V", "comp_w", "lam", "BB", "Fstar"):
        assert np.allclose(getattr(m, key), getattr(ref, key), rtol=1e-12, atol=0), key
    assert abs(m.Lstar / ref.Lstar - 1) < 1e-12
    with pytest.raises(ValueError):
        M.deck_model(None, str(deck), overrides=["scattype='ANISOTROPIC'"], compute_parts=oracle_parts)


def test_read_star_bins_and_interpolates(tmp_path):
    lam = M.wavelength_grid(0.1, 100.0, 30)[0]
    fine = np.geomspace(0.05, 50.0, 4000)
    f = lambda x: x ** -2.0 * np.exp(-0.05 / x)
    (tmp_path / "star.dat").write_text("* a spectrum\n" + "".join("%.9e %.9e\n" % (x, f(x)) for x in fine))
    got = M.read_star(str(tmp_path / "star.dat"), lam)
    inside = lam < 30.0
    # bin averages of a smooth spectrum sampled densely: close to its value
    assert np.allclose(got[inside], f(lam[inside]), rtol=0.03)
    # beyond the file: lambda^-2 from the last point
    beyond = lam > 50.0 * 1.0001
    assert np.allclose(got[beyond], f(fine[-1]) * fine[-1] ** 2 / lam[beyond] ** 2, rtol=1e-9)
    # a coarse file: a bin holding one of its points takes that point's value,
    # a bin holding none the log-log interpolation between its points
    coarse = np.geomspace(0.05, 50.0, 7)
    (tmp_path / "coarse.dat").write_text("".join("%.12e %.12e\n" % (x, x ** -3.0) for x in coarse))
    got = M.read_star(str(tmp_path / "coarse.dat"), lam)
    interp = np.isclose(got, lam ** -3.0, rtol=1e-9)
    point = np.array([np.any(np.isclose(g, coarse ** -3.0, rtol=1e-9)) for g in got])
    assert np.all((interp | point)[lam < 50.0])
    assert interp.sum() >= 15 and point.sum() >= 4


def test_deck_model_file_star(tmp_path):
    import oracle_ffi as O
    lam_tab = np.geomspace(0.05, 5000.0, 80)
    n, k = M.synthetic_lnk(lam_tab, 0.03)
    (tmp_path / "syn.lnk").write_text("".join("%g %g %g\n" % t for t in zip(lam_tab, n, k)))
    (tmp_path / "dust.particle").write_text("1\n1\n'syn.lnk'\n1.0 3.0\n")
    fine = np.geomspace(0.05, 5000.0, 3000)
    (tmp_path / "spec.dat").write_text("".join("%.9e %.9e\n" % (x, x ** -2 * np.exp(-0.3 / x)) for x in fine))
    deck = tmp_path / "d.in"
    deck.write_text("startype='FILE'\nstarfile='spec.dat'\nlstar=20\nnrad=8\nntheta=6\nnlam=15\n"
                    "zone1:rin=1\nzone1:rout=50\nzone1:fix=.true.\ncomputepart01:file='dust.particle'\n")

    def oracle_parts(parts):
        return [O.compute_part(p["lam"], p["e1"][0], p["e2"][0], p["frac"], p["rho"], p["amin"], p["amax"],
                               p["apow"], p["fmax"], p["blend"], p["porosity"], p["ns"], p["nf"]) for p in parts]

    m, run = M.deck_model(None, str(deck), compute_parts=oracle_parts)
    Lsun = M.luminosity(5778.0, M.RSUN)
    # the reference's luminosity unit is per steradian over pi: sigma T^4 R^2,
    # as the integral of Fstar = pi R^2 B_nu is for a Planck star
    assert abs(Lsun / (5.6704e-5 * 5778.0 ** 4 * M.RSUN ** 2) - 1) < 1e-3
    assert abs(m.Lstar / (20 * Lsun) - 1) < 1e-14
    assert abs(M.integrate(m.nu, m.Fstar) / m.Lstar - 1) < 1e-12
    with pytest.raises(ValueError):
        M.deck_model(None, str(deck), overrides=["startype='KURUCZ'"], compute_parts=oracle_parts)


def test_deck_model_file_density_restarts_from_denstemp(tmp_path):
    import oracle_ffi as O
    from mcmax_b200 import outputs as OUT
    lam_tab = np.geomspace(0.05, 5000.0, 80)
    n, k = M.synthetic_lnk(lam_tab, 0.03)
    (tmp_path / "syn.lnk").write_text("".join("%g %g %g\n" % t for t in zip(lam_tab, n, k)))
    (tmp_path / "dust.particle").write_text("1\n1\n'syn.lnk'\n1.0 3.0\n")
    common = "rin=0.5\nrout=100\nnlam=15\ncomputepart01:file='dust.particle'\n"
    (tmp_path / "a.in").write_text(common + "nrad=14\nntheta=10\nzone1:rin=0.5\nzone1:rout=100\nzone1:fix=.true.\n"
                                   "zone1:mdust=1d-4\n")

    def oracle_parts(parts):
        return [O.compute_part(p["lam"], p["e1"][0], p["e2"][0], p["frac"], p["rho"], p["amin"], p["amax"],
                               p["apow"], p["fmax"], p["blend"], p["porosity"], p["ns"], p["nf"]) for p in parts]

    a, _ = M.deck_model(None, str(tmp_path / "a.in"), compute_parts=oracle_parts)
    T = np.linspace(20, 900, a.ncell)
    OUT.write_denstemp(str(tmp_path / "denstemp.dat"), a, T)
    (tmp_path / "b.in").write_text(common + "denstype='FILE'\ndensfile='denstemp.dat'\n")
    b, run = M.deck_model(None, str(tmp_path / "b.in"), compute_parts=oracle_parts)
    assert (b.nr, b.nt) == (a.nr, a.nt) and run["zones"] == []
    nc = a.nt - 1
    assert np.array_equal(b.dens.reshape(b.nr, nc)[1:], a.dens.reshape(a.nr, nc)[1:])
    assert np.allclose(b.R, a.R, rtol=1e-12) and np.allclose(b.Theta, a.Theta, rtol=0, atol=1e-14)
    assert np.allclose(b.V, a.V, rtol=1e-10)


def test_deck_model_file_density_from_fits(tmp_path):
    import oracle_ffi as O
    from mcmax_b200 import outputs as OUT
    lam_tab = np.geomspace(0.05, 5000.0, 80)
    n, k = M.synthetic_lnk(lam_tab, 0.03)
    (tmp_path / "syn.lnk").write_text("".join("%g %g %g\n" % t for t in zip(lam_tab, n, k)))
    (tmp_path / "dust.particle").write_text("1\n1\n'syn.lnk'\n1.0 3.0\n")
    common = "rin=0.5\nrout=100\nnlam=12\ncomputepart01:file='dust.particle'\n"
    (tmp_path / "a.in").write_text(common + "nrad=9\nntheta=8\nzone1:rin=0.5\nzone1:rout=100\nzone1:fix=.true.\n")

    def oracle_parts(parts):
        return [O.compute_part(p["lam"], p["e1"][0], p["e2"][0], p["frac"], p["rho"], p["amin"], p["amax"],
                               p["apow"], p["fmax"], p["blend"], p["porosity"], p["ns"], p["nf"]) for p in parts]

    a, _ = M.deck_model(None, str(tmp_path / "a.in"), compute_parts=oracle_parts)
    OUT.write_denstemp_fits(str(tmp_path / "denstemp.fits.gz"), a, np.full(a.ncell, 50.0))
    (tmp_path / "b.in").write_text(common + "denstype='FILE'\ndensfile='denstemp.fits.gz'\noutputfits=.true.\n")
    b, run = M.deck_model(None, str(tmp_path / "b.in"), compute_parts=oracle_parts)
    nc = a.nt - 1
    assert run["outputfits"] is True
    assert np.array_equal(b.dens.reshape(b.nr, nc)[1:], a.dens.reshape(a.nr, nc)[1:])
    assert np.allclose(b.R, a.R, rtol=1e-12)


def test_deck_grains_from_particle_fits_and_opacity_tables(tmp_path):
    import oracle_ffi as O
    from mcmax_b200 import particle_fits as PF
    lam_tab = np.geomspace(0.05, 5000.0, 80)
    n, k = M.synthetic_lnk(lam_tab, 0.03)
    (tmp_path / "syn.lnk").write_text("".join("%g %g %g\n" % t for t in zip(lam_tab, n, k)))
    (tmp_path / "dust.particle").write_text("2\n2\n'syn.lnk'\n1.0 3.0\n")
    common = "rin=0.5\nrout=100\nnrad=8\nntheta=6\nnlam=14\nzone1:rin=0.5\nzone1:rout=100\nzone1:fix=.true.\n"
    (tmp_path / "a.in").write_text(common + "computepart01:file='dust.particle'\ncomputepart01:amin=0.2\n"
                                   "computepart01:amax=0.8\n")

    def oracle_parts(parts):
        return [O.compute_part(p["lam"], p["e1"][0], p["e2"][0], p["frac"], p["rho"], p["amin"], p["amax"],
                               p["apow"], p["fmax"], p["blend"], p["porosity"], p["ns"], p["nf"]) for p in parts]

    a, _ = M.deck_model(None, str(tmp_path / "a.in"), compute_parts=oracle_parts)
    # the particle cache file of that grain, and an opacity table of it
    res = dict(kabs=a.Kabs[0], ksca=a.Ksca[0], kext=a.Kabs[0] + a.Ksca[0], F=a.F[0], rho_av=2.25)
    PF.write_particle_fits(str(tmp_path / "p.fits.gz"), a.lam, res, 0.2, 0.8, 3.5, 0.0, True, 0.25, [1.0], [3.0],
                           ["syn.lnk"], 2)
    (tmp_path / "o.dat").write_text("".join("%.17e %.17e %.17e %.17e\n" % (l, ka + ks, ka, ks)
                                            for l, ka, ks in zip(a.lam, a.Kabs[0], a.Ksca[0])))
    with open(tmp_path / "q.dat", "w") as f:    # the ASCII particle format: 8 values per line for the matrices
        for li, l in enumerate(a.lam):
            f.write("%.17e %.17e %.17e %.17e\n" % (l, a.Kabs[0][li] + a.Ksca[0][li], a.Kabs[0][li], a.Ksca[0][li]))
            for e in range(6):
                row = a.F[0][li, e]
                for c0 in range(0, 180, 8):
                    f.write(" ".join("%.17e" % x for x in row[c0:c0 + 8]) + "\n")
    (tmp_path / "b.in").write_text(common + "fitspart01='p.fits.gz'\nopac02='o.dat'\npart3='q.dat'\nabun01=3\n"
                                   "abun02=1\n")
    b, _ = M.deck_model(None, str(tmp_path / "b.in"), compute_parts=oracle_parts)
    assert b.ncomp == 3 and np.allclose(b.comp_w[0], [0.6, 0.2, 0.2])
    assert np.array_equal(b.Kabs[2], a.Kabs[0]) and np.allclose(b.F[2], a.F[0], rtol=1e-12, atol=1e-300)
    assert np.array_equal(b.Kabs[0], a.Kabs[0]) and np.array_equal(b.Ksca[1], a.Ksca[0])
    assert np.allclose(b.F[0], a.F[0], rtol=1e-12, atol=1e-300)
    s = np.sin(np.pi * (np.arange(1, 181) - 0.5) / 180.0)
    assert np.allclose((b.F[1][:, 0, :] * s).sum(1), s.sum(), rtol=1e-13)      # the normalised Rayleigh matrix
    assert np.allclose(b.bins[0], (0.2, 0.8), rtol=1e-7)      # R_MIN, R_MAX of the file (single precision)


def test_rayleigh_scattype_matrices_for_file_grains(tmp_path):
    from mcmax_b200 import particle_fits as PF
    th = (np.arange(1, 181) - 0.5) * np.pi / 180.0
    hg = lambda g: (1 - g * g) / (1 - 2 * g * np.cos(th) + g * g) ** 1.5 / 2
    # the one-degree bin average is the closed form to second order in the bin width
    assert np.allclose([PF.hg_binned(0.5, x) for x in th], hg(0.5), rtol=2e-3)
    lam = M.wavelength_grid(0.1, 1000.0, 10)[0]
    res = dict(kabs=np.linspace(1, 2, 10), ksca=np.linspace(2, 3, 10), kext=np.linspace(3, 5, 10),
               F=np.ones((10, 6, 180)), rho_av=3.0)
    PF.write_particle_fits(str(tmp_path / "p.fits"), lam, res, 0.1, 1.0, 3.5, 0.0, False, 0.0, [1.0], [3.0], ["x"], 1)
    r = PF.read_particle_fits(str(tmp_path / "p.fits"), lam, matrix=PF.rayleigh_hg_matrix(0.5, pmax=0.3))
    s = np.sin(th)
    F11 = r["F"][3, 0]
    assert np.allclose(F11 / F11[0], np.array([PF.hg_binned(0.5, x) for x in th]) / PF.hg_binned(0.5, th[0]),
                       rtol=1e-12)
    assert abs((F11 * s).sum() / s.sum() - 1) < 1e-13
    c = np.cos(th)
    assert np.allclose(r["F"][3, 1], -0.3 * F11 * (1 - c * c) / (1 + c * c), rtol=1e-12)
    ray = PF.read_particle_fits(str(tmp_path / "p.fits"), lam, matrix=PF.rayleigh_hg_matrix())
    assert np.allclose(ray["F"][0, 0] / ray["F"][0, 0][0], ((1 + c * c) / 2) / ((1 + c[0] ** 2) / 2), rtol=1e-12)


def _analytic_deck(tmp_path, body):
    import oracle_ffi as O
    lam_tab = np.geomspace(0.05, 5000.0, 80)
    n, k = M.synthetic_lnk(lam_tab, 0.03)
    (tmp_path / "syn.lnk").write_text("".join("%g %g %g\n" % t for t in zip(lam_tab, n, k)))
    (tmp_path / "dust.particle").write_text("1\n1\n'syn.lnk'\n1.0 3.0\n")
    deck = tmp_path / "d.in"
    deck.write_text("rin=0.1\nrout=1000\nnrad=30\nntheta=20\nlam1=0.1\nlam2=3000\nnlam=25\n"
                    "computepart01:file='dust.particle'\n" + body)

    def oracle_parts(parts):
        return [O.compute_part(p["lam"], p["e1"][0], p["e2"][0], p["frac"], p["rho"], p["amin"], p["amax"],
                               p["apow"], p["fmax"], p["blend"], p["porosity"], p["ns"], p["nf"]) for p in parts]

    return str(deck), oracle_parts


def _cells(m):
    nc = m.nt - 1
    dens = m.dens.reshape(m.nr, nc)
    V = m.V.reshape(m.nr, nc)
    R_av = M.AU * 10.0 ** ((np.log10(m.R[:-1]) + np.log10(m.R[1:])) / 2.0)
    th = np.arccos((m.Theta[:-1] + m.Theta[1:]) / 2.0)
    return dens, V, R_av[:, None] * np.sin(th)[None, :] / M.AU, R_av[:, None] * np.cos(th)[None, :] / M.AU


def test_pascucci_density_has_the_midplane_optical_depth(tmp_path):
    """the benchmark disk: rho ~ (r/rd)^-1 exp(-pi/4 (z/h)^2), h = rd/4
    (r/rd)^1.125, scaled so that the midplane's radial optical depth at
    0.55 micron, from rin to rout, is tau550"""
    deck, parts = _analytic_deck(tmp_path, "denstype='PASCUCCI'\ntau550=100\n")
    m, run = M.deck_model(None, deck, compute_parts=parts)
    dens, V, r, z = _cells(m)
    rd = 500.0
    h = rd / 4.0 * (r / rd) ** 1.125
    shape = (r / rd) ** -1.0 * np.exp(-(math.pi / 4.0) * (z / h) ** 2)
    sel = dens[1:] > 1e-40          # cells above the 1e-60 floor
    ratio = dens[1:][sel] / shape[1:][sel]
    assert np.allclose(ratio, ratio[0], rtol=1e-12)
    # the midplane tau of the closed form: Kext550 * scale * rd * ln(rout/rin)
    k550 = np.interp(0.55, m.lam, m.Kabs[0] + m.Ksca[0])
    tau = k550 * ratio[0] * M.AU * rd * math.log(1000.0 / 0.1)
    assert abs(tau / 100.0 - 1.0) < 1e-3, tau
    assert run["zones"] == []


@pytest.mark.parametrize("kind", ["MIN", "PARAMETERIZED", "PINTE"])
def test_gaussian_disks_hold_the_dust_mass(kind, tmp_path):
    deck, parts = _analytic_deck(tmp_path, "denstype='%s'\nmdust=2d-4\nsh1au=0.05\nshpow=1.2\ndenspow=0.8\n"
                                           "rexp=100\n" % kind)
    m, _ = M.deck_model(None, deck, compute_parts=parts)
    dens, V, r, z = _cells(m)
    assert abs((dens[1:] * V[1:]).sum() / (2e-4 * M.MSUN) - 1.0) < 1e-12
    if kind == "MIN":
        f = r ** -0.8 * np.exp(-(z / (0.05 * r ** 1.2)) ** 2) * r ** -1.2
        sel = dens[1:] > 1e-40
        ratio = dens[1:][sel] / f[1:][sel]
        assert np.allclose(ratio, ratio[0], rtol=1e-10)
    if kind == "PINTE":
        # outside rexp: 1e-60 times the mass scaling, as the reference scales every cell
        assert np.all(dens[1:][r[1:] >= 100.0] < 1e-55) and np.any(dens[1:][r[1:] < 100.0] > 1e-30)


def test_shell_and_wedge_densities(tmp_path):
    deck, parts = _analytic_deck(tmp_path, "denstype='SHELL'\ndenspow=2\nmdust=1d-5\n")
    m, _ = M.deck_model(None, deck, compute_parts=parts)
    dens, V, r, z = _cells(m)
    R_av = M.AU * 10.0 ** ((np.log10(m.R[:-1]) + np.log10(m.R[1:])) / 2.0)
    assert np.allclose(dens[1:] * (R_av[1:, None] / M.AU) ** 2, dens[1, 0] * (R_av[1] / M.AU) ** 2, rtol=1e-12)
    deck, parts = _analytic_deck(tmp_path, "denstype='WEDGE'\nwedgeopen=20\n")
    m, _ = M.deck_model(None, deck, compute_parts=parts)
    dens, V, r, z = _cells(m)
    thet = np.asarray(m.thet)
    lo = 90.0 - np.degrees(thet[1:])      # elevation of a cell's lower edge above the midplane
    assert np.all(dens[1:, lo > 20.5] <= 1e-60)          # at the floor
    assert np.all(dens[1:, -1] > 1e-40)
    with pytest.raises(ValueError):
        M.deck_model(None, deck, overrides=["denstype='PRODIMO'"], compute_parts=parts)
    with pytest.raises(ValueError):
        M.deck_model(None, deck, overrides=["zone1:rin=1"], compute_parts=parts)


@pytest.mark.parametrize("kind", ["POW", "SIMILARITY", "DOUBLEPOW", "DOUBLEPOWSIM"])
def test_power_law_densities(kind, tmp_path):
    """the radial power laws start from (AU/R)^(denspow+1), independent of
    theta, scaled to mdust; their vertical structure comes from the
    optically thin start"""
    deck, parts = _analytic_deck(tmp_path, "denstype='%s'\nmdust=1d-4\ndenspow=1.5\ndenspow2=3\nrpow2=30\n"
                                           "rexp=50\n" % kind)
    m, run = M.deck_model(None, deck, compute_parts=parts)
    dens, V, r, z = _cells(m)
    assert abs((dens[1:] * V[1:]).sum() / (1e-4 * M.MSUN) - 1.0) < 1e-12
    assert np.all(dens[1:] == dens[1:, :1])
    R_av = 10.0 ** ((np.log10(m.R[:-1]) + np.log10(m.R[1:])) / 2.0)
    f = R_av ** -2.5
    if kind == "SIMILARITY":
        f = f * np.exp(-(R_av / 50.0) ** 0.5)        # gamma_exp defaults to 2 - denspow
    if kind in ("DOUBLEPOW", "DOUBLEPOWSIM"):
        f = np.where(R_av < 30.0, (30.0 / R_av) ** 2.5, (30.0 / R_av) ** 4.0)
        if kind == "DOUBLEPOWSIM":
            f = np.where(R_av < 30.0, f, f * np.exp(-(R_av / 50.0) ** 0.5))
    ratio = dens[1:, 0] / f[1:]
    assert np.allclose(ratio, ratio[0], rtol=1e-10)
    assert run["thin_start"] and not run["iterate"] and run["zones"] == []


def test_massloss_and_infall_densities(tmp_path):
    """MASSLOSS at constant speed is Mdot / (gas2dust 4 pi R^2 v); INFALL far
    outside its disk radius tends to free fall, Minfall / (4 pi sqrt(2 G
    Mstar R^3)) / gas2dust, whatever the angle"""
    yr = 365.25 * 24 * 3600.0
    deck, parts = _analytic_deck(tmp_path, "denstype='MASSLOSS'\nmdot=1d-6\nvexp=15\n")
    m, _ = M.deck_model(None, deck, compute_parts=parts)
    dens, V, r, z = _cells(m)
    R_av = M.AU * 10.0 ** ((np.log10(m.R[:-1]) + np.log10(m.R[1:])) / 2.0)
    want = 1e-6 * M.MSUN / yr / (100.0 * 4.0 * math.pi * R_av ** 2 * 15e5)
    assert np.allclose(dens[1:], want[1:, None], rtol=1e-12)
    deck, parts = _analytic_deck(tmp_path, "denstype='INFALL'\nmdot=1d-6\nrexp=0.5\nmstar=1\n")
    m, _ = M.deck_model(None, deck, compute_parts=parts)
    dens, V, r, z = _cells(m)
    R_av = M.AU * 10.0 ** ((np.log10(m.R[:-1]) + np.log10(m.R[1:])) / 2.0)
    ff = 1e-6 * M.MSUN / yr / (4.0 * math.pi * np.sqrt(2.0 * 6.673e-8 * M.MSUN * R_av ** 3)) / 100.0
    far = R_av / M.AU > 200.0
    assert np.allclose(dens[far], ff[far, None], rtol=0.05)
    # nearer in, the flow piles up toward the midplane
    i = int(np.searchsorted(R_av / M.AU, 1.0))
    assert dens[i, -1] > dens[i, 0]


def test_regridlog_follows_the_reference_reader(tmp_path):
    p = tmp_path / "s.dat"
    p.write_text("# r sigma\n1.0 10.0\n2.0 5.0\n4.0 0.0\n8.0 1.0\n")
    grid = np.array([0.5, 1.0, 1.5, 3.0, 6.0, 16.0, 32.0])
    y = M.regridlog(str(p), grid)
    assert y[0] == 10.0 and y[1] == 10.0                     # at or below the first x
    assert abs(y[2] - 10.0 * 1.5 ** -1.0) < 1e-12            # log-log inside: Sigma ~ 1/r here
    # an entry <= 0 is read as 1e-50 of the one before
    assert abs(math.log10(y[3] / 5.0) - math.log10(5e-50 / 5.0) * math.log10(3.0 / 2.0) / math.log10(2.0)) < 1e-9
    assert y[5] == y[4] * 6.0 / 16.0 or abs(y[5] / (1.0 * 8.0 / 16.0) - 1) < 1e-12
    assert abs(y[6] / y[5] - 0.5) < 1e-12                    # beyond the table: 1/r from the last point


def test_surface_density_file(tmp_path):
    r = np.geomspace(0.05, 2000.0, 60)
    (tmp_path / "sigma.dat").write_text("".join("%.8e %.8e\n" % (a, 100.0 * a ** -1.0) for a in r))
    (tmp_path / "gas.dat").write_text("".join("%.8e %.8e\n" % (a, 1e4 * a ** -1.0) for a in r))
    deck, parts = _analytic_deck(tmp_path, "denstype='SURFFILE'\ndensfile='sigma.dat'\nmdust=1d-4\n"
                                           "gasdensfile='gas.dat'\n")
    m, run = M.deck_model(None, deck, compute_parts=parts)
    dens, V, r_, z_ = _cells(m)
    assert abs((dens[1:] * V[1:]).sum() / (1e-4 * M.MSUN) - 1.0) < 1e-12
    R = np.asarray(m.R)
    R_av = 10.0 ** ((np.log10(R[:-1]) + np.log10(R[1:])) / 2.0)
    # each ring's mass goes as Sigma(R_av) (R_i+1^2 - R_i^2), spread evenly over its cells
    ringmass = (dens * V).sum(1)[1:]
    want = R_av[1:] ** -1.0 * (R[2:] ** 2 - R[1:-1] ** 2)
    assert np.allclose(ringmass / want, ringmass[0] / want[0], rtol=1e-7)   # the table has 9 digits
    assert np.allclose(dens[1:], dens[1:, :1], rtol=1e-12)
    gas = m.gasdens.reshape(m.nr, -1)
    want_gas = 1e4 * R_av[1:, None] ** -1.0 * math.pi * (R[2:] ** 2 - R[1:-1] ** 2)[:, None] * M.AU ** 2 / V[1:] / \
        (m.nt - 1) / 100.0
    assert np.allclose(gas[1:], want_gas, rtol=1e-7)
    assert run["thin_start"] and not run["iterate"]


def test_shell_density_file(tmp_path):
    r = np.geomspace(0.05, 2000.0, 40)
    (tmp_path / "shell.dat").write_text("".join("%.12e %.12e\n" % (a, 1e-18 * a ** -2.0) for a in r))
    deck, parts = _analytic_deck(tmp_path, "denstype='SHELLFILE'\ndensfile='shell.dat'\nmdust=1d-4\n")
    m, run = M.deck_model(None, deck, compute_parts=parts)
    dens, V, _, _ = _cells(m)
    R = np.asarray(m.R)
    R_av = 10.0 ** ((np.log10(R[:-1]) + np.log10(R[1:])) / 2.0)
    # the table's values, not scaled to mdust
    assert np.allclose(dens[1:], 1e-18 * R_av[1:, None] ** -2.0, rtol=1e-9)
    assert not run["thin_start"]


def test_meixner_shell(tmp_path):
    """at the inner radius the profile is 1 + A (1 - cos theta)^F; with
    C = 0 it falls as r^-B times the equatorial factor"""
    deck, parts = _analytic_deck(tmp_path, "denstype='MEIXNER'\nmdust=1d-5\nmeixc=0\nmeixrin=1\n")
    m, _ = M.deck_model(None, deck, compute_parts=parts)
    dens, V, _, _ = _cells(m)
    R = np.asarray(m.R)
    ra = 10.0 ** ((np.log10(R[:-1]) + np.log10(R[1:])) / 2.0)
    th = np.arccos((m.Theta[:-1] + m.Theta[1:]) / 2.0)
    f = (ra[:, None] / 1.0) ** -2.0 * (1.0 + 8.0 * (1.0 - np.cos(th))[None, :]
                                        * np.exp(-(ra[:, None] / 1800.0) ** 3 + (1.0 / 1800.0) ** 3))
    sel = ra[1:] > 1.0
    ratio = dens[1:][sel] / f[1:][sel]
    assert np.allclose(ratio, ratio[0, 0], rtol=1e-10)
    assert np.all(dens[1:][~sel] < 1e-55)
    assert abs((dens[1:] * V[1:]).sum() / (1e-5 * M.MSUN) - 1) < 1e-12


def test_meixner_timeshift_moves_the_grid_and_the_profile(tmp_path):
    """timeshift t [yr] at vexp1 v [km/s]: the grid's inner and outer radii
    move out by t v 0.210944839 AU (Init.f:1634-1636), the profile is
    evaluated at r - t v 0.210944839 AU with the shell's inner radius kept
    at the unshifted rin (Init.f:1528, 3231); meixd <= 0 takes meixe
    (Init.f:1529)"""
    deck, parts = _analytic_deck(tmp_path, "denstype='MEIXNER'\nmdust=1d-5\nmeixd=-1\ntimeshift=100\n"
                                           "vexp1=15\n")
    m, _ = M.deck_model(None, deck, compute_parts=parts)
    shift = 100.0 * 15.0 * 0.210944839
    R = np.asarray(m.R)
    assert abs(R[1] / (0.1 + shift) - 1) < 1e-12
    assert abs(R[-1] / (1000.0 + shift) - 1) < 1e-12
    dens, V, _, _ = _cells(m)
    ra = 10.0 ** ((np.log10(R[:-1]) + np.log10(R[1:])) / 2.0)
    th = np.arccos((m.Theta[:-1] + m.Theta[1:]) / 2.0)
    rr = (ra[1:] - 100.0 * 15e5 * 0.210944839e-5)[:, None]   # the disk's rings (not the star cell)
    st, ct = np.sin(th)[None, :], np.cos(th)[None, :]
    D = E = 3.0
    f = (rr / 0.1) ** (-2.0 * (1.0 + 2.0 * st * np.exp(-(rr / 1800.0) ** D + (0.1 / 1800.0) ** D)))
    f = f * (1.0 + 8.0 * (1.0 - ct) * np.exp(-(rr / 1800.0) ** E + (0.1 / 1800.0) ** E)) * (rr / ra[1:, None]) ** 2
    ratio = dens[1:] / f
    assert np.all(rr > 0.1)
    assert np.allclose(ratio, ratio[0, 0], rtol=1e-10)
    assert abs((dens[1:] * V[1:]).sum() / (1e-5 * M.MSUN) - 1) < 1e-12
