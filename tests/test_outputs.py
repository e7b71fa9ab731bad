"""The reference's output files written from library results: denstemp.dat
(format 5) round trip, and the MCSpec file names and columns."""
import math
import os

import numpy as np

import models
from mcmax_b200 import model as M
from mcmax_b200 import outputs as OUT


def test_denstemp_round_trip(tmp_path):
    m = models.small_disk()
    rng = np.random.default_rng(2)
    T = rng.uniform(10, 1500, m.ncell)
    p = os.path.join(tmp_path, "denstemp.dat")
    OUT.write_denstemp(p, m, T)
    d = OUT.read_denstemp(p)
    nr, nc = m.nr, m.nt - 1
    assert d["dens"].shape == (nr - 1, nc) and d["ngrains"] == m.ncomp
    assert np.array_equal(d["T"], T.reshape(nr, nc)[1:])
    assert np.array_equal(d["dens"], m.dens.reshape(nr, nc)[1:])
    assert np.array_equal(d["comp"], m.comp_w.reshape(nr, nc, m.ncomp)[1:])
    assert np.allclose(d["gasdens"], 100.0 * d["dens0"], rtol=1e-15)
    assert np.all(np.diff(d["r_av"]) > 0) and np.all(np.diff(d["theta_av"]) > 0)
    assert abs(d["r_av"][0] / M.AU - math.sqrt(m.R[1] * m.R[2])) < 1e-9 * d["r_av"][0] / M.AU


def test_mcspec_names_and_columns(tmp_path):
    names = [OUT.mcspec_name(j) for j in range(1, 31)]
    assert names[0] == "MCSpec89.0.dat" and names[-1] == "MCSpec10.5.dat"
    assert len(set(names)) == 30
    m = models.small_disk()
    ns = m.nlam * 31
    rng = np.random.default_rng(1)
    res = dict(spec=rng.uniform(0, 1, ns), scatspec=rng.uniform(0, 0.1, ns), ispec=rng.integers(0, 50, ns))
    OUT.write_mcspec(str(tmp_path), m, res, distance_pc=140.0)
    a = np.loadtxt(os.path.join(tmp_path, names[5]))
    assert a.shape == (m.nlam, 6)
    d2 = (140.0 * OUT.PARSEC) ** 2
    sp = res["spec"].reshape(m.nlam, 31)[:, 6]
    assert np.allclose(a[:, 0], m.lam) and np.allclose(a[:, 1], sp / d2, rtol=1e-15)
    n = res["ispec"].reshape(m.nlam, 31)[:, 6]
    ok = n > 0
    assert np.allclose(a[ok, 2], sp[ok] / np.sqrt(n[ok]) / d2, rtol=1e-14)
    assert os.path.exists(os.path.join(tmp_path, "MCSpec.dat"))


def test_spectrum_file(tmp_path):
    lam = np.geomspace(0.1, 1000.0, 12)
    Fstar = lam ** -2.0 * np.exp(-0.5 / lam)
    lo = OUT.spectrum_wavelengths(lam, 0.2, 500.0)
    assert lo[0] == 0.2 and lo[-1] == 500.0 and np.all(np.diff(lo) > 0) and lo.size == 2 + np.sum((lam > 0.2) & (lam < 500))
    flux = np.linspace(1.0, 2.0, lo.size)
    path = OUT.write_spectrum(str(tmp_path), 45.0, lo, flux, lam, Fstar, distance_pc=100.0)
    assert os.path.basename(path) == "spectrum45.0.dat"
    rows = np.loadtxt(path)
    d2 = (100.0 * OUT.PARSEC) ** 2
    assert np.allclose(rows[:, 0], lo) and np.allclose(rows[:, 1], 1e23 * flux / d2, rtol=1e-15)
    assert np.all(rows[:, 2] == 0.0)
    # the reference's star column: the abscissa at the ends, the last-interval power law inside
    p = math.log10(Fstar[-1] / Fstar[-2]) / math.log10(lam[-1] / lam[-2])
    inner = Fstar[-2] * (lo[1:-1] / lam[-2]) ** p
    assert np.allclose(rows[1:-1, 3], 1e23 * inner / d2, rtol=1e-12)
    p2 = OUT.write_spectrum(str(tmp_path), 7.5, lo, flux, lam, Fstar, star_column="interpolated", flag="_b")
    assert os.path.basename(p2) == "spectrum07.5_b.dat"
    r2 = np.loadtxt(p2)
    assert np.allclose(r2[1:-1, 3], 1e23 * np.exp(np.interp(np.log(lo[1:-1]), np.log(lam), np.log(Fstar))) / d2)
    # full Mueller scattering: a fifth column for the Q flux
    p3 = OUT.write_spectrum(str(tmp_path), 30.0, lo, flux, lam, Fstar, polarised=True)
    r3 = np.loadtxt(p3)
    assert rows.shape[1] == 4 and r3.shape == (lo.size, 5)
    assert np.all(r3[:, 4] == 0.0) and np.array_equal(r3[:, :4], rows[:, :4])


def test_denstemp_fits_round_trip(tmp_path):
    m = models.small_disk(nrad=10, ntheta=8, nlam=12, mdust=1e-5)
    T = np.linspace(10.0, 500.0, m.ncell)
    p = OUT.write_denstemp_fits(str(tmp_path / "denstemp.fits"), m, T)
    assert p.endswith(".fits.gz") and os.path.exists(p)
    d = OUT.read_denstemp_fits(p)
    OUT.write_denstemp(str(tmp_path / "denstemp.dat"), m, T)
    t = OUT.read_denstemp(str(tmp_path / "denstemp.dat"))
    for k in ("dens", "T", "gasdens", "dens0", "comp"):
        assert np.array_equal(d[k], t[k]), k
    assert np.allclose(d["r_av"], t["r_av"], rtol=1e-15) and np.array_equal(d["theta_av"], t["theta_av"])
    from mcmax_b200 import particle_fits as PF
    hdr = PF._read_hdus(PF._open(p))[0][0]
    assert (hdr["NR"], hdr["NTHETA"], hdr["NGRAINS"], hdr["NHDU"]) == (m.nr - 1, m.nt - 1, m.ncomp, 5)
    assert hdr["HDU 3"] == "COMP"


def test_image_file_names_follow_the_reference_formats():
    deg = lambda a: math.pi * a / 180.0
    assert OUT.image_name("AI", deg(45.0), 0.6, 50.0) == "ImageAI_i45.0_l00000.60_fov00100.0.fits"
    assert OUT.rimage_name(deg(30.0), 1234.5678, "_x") == "RImage_i30.0_l01234.57_x.dat"
    # tenths of 9.95 and up carry into the tens (angle and field of view)
    assert OUT._angle_tag(deg(39.97)) == "40.0"
    assert OUT._fov_tag(99.97 / 2.0) == "00100.0"
    # a value that does not fit f4.2 prints as asterisks, as Fortran does
    assert OUT._lam_tag(9.999) == "0000****"


def test_image_fits_round_trip(tmp_path):
    im = np.arange(12.0 * 12.0).reshape(12, 12) * 1e-3
    p = OUT.write_image_fits(str(tmp_path / "ImageAI_x.fits"), im, 25.0, rscale=0.01, scaletype=2)
    raw = open(p, "rb").read()
    assert len(raw) % 2880 == 0
    hdr, back = OUT.read_image_fits(p)
    assert np.array_equal(back, im)
    assert hdr["NAXIS1"] == 12 and hdr["BITPIX"] == -64
    assert hdr["CRPIX1"] == 0.5 and abs(hdr["CRVAL2"] + 0.25) < 1e-12 and abs(hdr["CDELT1"] - 0.5 / 12) < 1e-12
    assert hdr["CTYPE2"].strip() == "Y [arcsec]"


def test_rimage_profile(tmp_path):
    """running trapezoid flux per image radius, the total on the last row,
    the intensity at column nphi/2 times the pixel scaling"""
    R = np.array([0.0, 1.0, 2.5, 4.0])
    rphi = np.outer([4.0, 3.0, 2.0, 1.0], np.ones(6)) * 1e-10
    d = 140.0 * OUT.PARSEC
    p = OUT.write_rimage(str(tmp_path / "RImage.dat"), R, rphi, 1.0, 1.0, d, 10.0, 100)
    rows = np.loadtxt(p)
    AU = M.AU
    ring = [(R[i + 1] - R[i]) * math.pi * AU ** 2 * (R[i] * rphi[i, 0] + R[i + 1] * rphi[i + 1, 0])
            for i in range(3)]
    assert rows.shape == (4, 3)
    assert np.allclose(rows[:, 0], R)
    assert np.allclose(rows[:3, 1], np.cumsum(ring) * 1e23 / d ** 2, rtol=1e-12)
    assert rows[3, 1] == rows[2, 1]
    scaling = 1e23 / d ** 2 * 10.0 ** 2 * AU ** 2 / 100 ** 2
    assert np.allclose(rows[:, 2], scaling * rphi[:, 2], rtol=1e-12)


def test_visibility_of_a_uniform_disk():
    """a face-on disk of constant intensity out to R: V = |2 J1(x) / x|,
    x = k R with k = 2 pi b / lambda in rad per AU at the distance; V = 1
    at zero baseline"""
    from scipy.special import j1
    R = np.linspace(0.0, 10.0, 201)
    rphi = np.ones((R.size, 45))
    d = 140.0 * OUT.PARSEC
    for b in (0.0, 20.0, 60.0, 120.0):
        V, ph = OUT.visibility(R, rphi, b, 0.3, 2.0, d)
        k = 2.0 * math.pi * b / (2.0 * 140.0) * 1e6 * math.pi / (180.0 * 3600.0)
        x = k * 10.0
        want = 1.0 if b == 0.0 else abs(2.0 * j1(x) / x)
        assert abs(V - want) < 2e-3, (b, V, want)
    # a telescope taper (diameter d) only lowers the long-baseline response
    V1, _ = OUT.visibility(R, rphi, 60.0, 0.3, 2.0, d, diam=8.0)
    assert 0.0 <= V1 <= 1.0 + 1e-12


def test_observation_vis_norm_fov(tmp_path):
    """vis_norm_fov: the input deck's value unless the observation file sets
    it for all observations or for one (Telescope.f:657, 1023, 1176)"""
    p = tmp_path / "obs.out"
    p.write_text("nphi=30\nvis_norm_fov=.false.\n*****\ntype='VISIBILITY'\n"
                 "type='VISIBILITY'\nvis_norm_fov=.true.\n")
    lam = np.geomspace(0.1, 1000.0, 20)
    obs = OUT.read_observations(str(p), lam, rout=100.0)
    assert [o["vis_norm_fov"] for o in obs] == [False, True]
    p.write_text("*****\ntype='VISIBILITY'\n")
    assert OUT.read_observations(str(p), lam, vis_norm_fov=False)[0]["vis_norm_fov"] is False
    assert OUT.read_observations(str(p), lam)[0]["vis_norm_fov"] is True
