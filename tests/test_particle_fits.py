"""The particle cache (particleNNNN.fits.gz) on CPU: the FITS container,
the keyword check that decides a cache hit, the wavelength regridding of
ReadParticleFits, and ComputePart reading a cached bin instead of
computing it.  ComputePart results come from the oracle."""
import gzip
import math
import os

import numpy as np
import pytest

import oracle_ffi as O
from mcmax_b200 import api
from mcmax_b200 import model as M
from mcmax_b200 import particle_fits as PF


def _result(lam, seed=0):
    rng = np.random.default_rng(seed)
    nlam = lam.size
    kabs = rng.uniform(10, 1e4, nlam)
    ksca = rng.uniform(10, 1e4, nlam)
    F = rng.uniform(0.1, 2.0, (nlam, 6, 180))
    s = np.sin(math.pi * (np.arange(1, 181) - 0.5) / 180.0)
    F *= (s.sum() / (F[:, 0] * s).sum(1))[:, None, None]
    return dict(kabs=kabs, ksca=ksca, kext=kabs + ksca, F=F, rho_av=2.7)


GRAIN = dict(amin=0.1, amax=1.0, apow=3.5, fmax=0.8, blend=True, porosity=0.25, frac=[0.7, 0.3], rho=[3.0, 1.8],
             lnkfiles=["/data/a.lnk", "/data/b.lnk"], ns=20)


def test_fits_container_layout(tmp_path):
    lam = np.geomspace(0.1, 3000, 37)
    path = str(tmp_path / "particle0001.fits")
    PF.write_particle_fits(path, lam, _result(lam), **GRAIN)
    raw = open(path, "rb").read()
    assert len(raw) % 2880 == 0
    cards = [raw[k:k + 80].decode() for k in range(0, 2880, 80)]
    assert cards[0] == "SIMPLE  =                    T" + cards[0][30:]
    assert cards[1].startswith("BITPIX  =                  -64")
    assert cards[3].startswith("NAXIS1  =                   37")
    assert any(c.startswith("FILE02  = '/data/b.lnk'") for c in cards)
    assert any(c.startswith("N_RADII =                   20") for c in cards)
    (h0, a), (h1, m) = PF._read_hdus(raw)
    assert a.shape == (4, 37) and m.shape == (180, 6, 37)
    assert h1["XTENSION"] == "IMAGE" and h1["NAXIS3"] == 180
    assert np.array_equal(a[0], lam)
    # the data is big-endian IEEE double, Fortran order: wavelength fastest
    hdr_len = 2880 * (1 + (len([c for c in cards if c.strip()]) * 80) // 2880)
    first = np.frombuffer(raw[hdr_len:hdr_len + 8], ">f8")[0]
    assert first == lam[0]
    a1, a2, a3 = h0["A1"], h0["A2"], h0["A3"]
    assert abs(math.sqrt(a2) * 1e-4 / M.grain_rv(0.1, 1.0, 3.5, 20) - 1) < 1e-6
    assert a1 ** 2 < a2 and a2 ** 1.5 < a3


def test_round_trip_on_the_same_grid(tmp_path):
    lam = np.geomspace(0.1, 3000, 50)
    res = _result(lam, 3)
    path = str(tmp_path / "p.fits.gz")
    PF.write_particle_fits(path, lam, res, **GRAIN)
    assert open(path, "rb").read(2) == b"\x1f\x8b"
    back = PF.read_particle_fits(path, lam)
    for k in ("kabs", "ksca", "kext"):
        assert np.array_equal(back[k], res[k]), k
    assert np.allclose(back["F"], res["F"], rtol=1e-13, atol=0)
    assert back["rho_av"] == np.float32(2.7)


def test_regridding_interpolates_and_extrapolates(tmp_path):
    coarse = np.geomspace(0.5, 100, 12)
    res = _result(coarse, 5)
    path = str(tmp_path / "p.fits")
    PF.write_particle_fits(path, coarse, res, **GRAIN)
    fine = np.geomspace(0.2, 1000, 70)
    back = PF.read_particle_fits(path, fine)
    below = fine <= coarse[0]
    inside = (fine > coarse[0]) & (fine <= coarse[-1])
    above = fine > coarse[-1]
    assert np.all(back["kabs"][below] == res["kabs"][0])
    assert np.allclose(back["kabs"][inside], np.interp(fine[inside], coarse, res["kabs"]), rtol=1e-12)
    assert np.allclose(back["kext"][inside], np.interp(fine[inside], coarse, res["kext"]), rtol=1e-12)
    last = np.flatnonzero(inside)[-1]
    assert np.allclose(back["ksca"][above], back["ksca"][last] * (fine[last] / fine[above]) ** 4, rtol=1e-12)
    assert np.allclose(back["kabs"][above], back["kabs"][last] * (fine[last] / fine[above]) ** 2, rtol=1e-12)
    assert np.allclose(back["kext"][above], back["kabs"][above] + back["ksca"][above], rtol=1e-14)
    s = np.sin(math.pi * (np.arange(1, 181) - 0.5) / 180.0)
    assert np.allclose((back["F"][:, 0] * s).sum(1), s.sum(), rtol=1e-13)


def test_keyword_check_decides_a_cache_hit(tmp_path):
    lam = np.geomspace(0.1, 3000, 20)
    path = str(tmp_path / "particle0001.fits.gz")
    PF.write_particle_fits(path, lam, _result(lam), **GRAIN)
    g = dict(GRAIN)
    assert PF.check_particle_file(path, **g)
    assert PF.check_particle_file(path, **dict(g, ns=10))          # fewer sizes than cached: still a hit
    for change in (dict(ns=40), dict(amin=0.11), dict(amax=2.0), dict(apow=3.0), dict(fmax=0.7),
                   dict(porosity=0.3), dict(frac=[0.5, 0.5]), dict(rho=[3.0, 2.0]),
                   dict(lnkfiles=["/data/a.lnk", "/data/c.lnk"])):
        assert not PF.check_particle_file(path, **dict(g, **change)), change
    # the power does not matter for one size, the porosity not for unblended grains
    PF.write_particle_fits(path, lam, _result(lam), **dict(g, ns=1, blend=False))
    assert PF.check_particle_file(path, **dict(g, ns=1, blend=False, apow=2.0, porosity=0.5))
    assert not PF.check_particle_file(str(tmp_path / "missing.fits"), **g)
    # the fractions are compared after normalisation, as the reference stores them
    assert PF.check_particle_file(path, **dict(g, ns=1, blend=False, frac=[1.4, 0.6]))


def test_long_file_names_continue_over_cards(tmp_path):
    lam = np.geomspace(0.1, 3000, 20)
    long = ["/very/long/" + "d" * 150 + "/it's.lnk", "/data/b.lnk"]
    path = str(tmp_path / "p.fits")
    PF.write_particle_fits(path, lam, _result(lam), **dict(GRAIN, lnkfiles=long))
    raw = open(path, "rb").read()
    assert raw.count(b"CONTINUE  '") >= 2
    hdr = PF._read_hdus(raw)[0][0]
    assert hdr["FILE01"] == long[0] and hdr["FILE02"] == long[1]
    assert PF.check_particle_file(path, **dict(GRAIN, lnkfiles=long))


def test_file_names():
    assert PF.particle_file_name("d", 3) == os.path.join("d", "particle0003.fits.gz")
    assert PF.particle_file_name("d", 12, iopac=2, gz=False) == os.path.join("d", "particle0012_02.fits")
    assert PF.particle_file_name("", 1, frac=[0.25, 0.75], abun_in_name=2) == "particle0001_f0.25_f0.75.fits.gz"
    assert PF.particle_file_name("", 1, frac=[0.5], abun_in_name=1, iopac=3) == "particle0001_f0.5_03.fits.gz"


class _OracleContext:
    def __init__(self):
        self.calls = 0

    def compute_part_batch(self, parts):
        self.calls += 1
        out = []
        for p in parts:
            r = O.compute_part(p["lam"], p["e1"][0], p["e2"][0], p["frac"], p["rho"], p["amin"], p["amax"],
                               p["apow"], p["fmax"], p["blend"], p["porosity"], p["ns"], p["nf"])
            r.setdefault("mscale", 1.0)
            r.setdefault("rscale", 1.0)
            for k in ("n_dhs", "n_mie", "n_dhs_fail"):
                r.setdefault(k, 0)
            out.append(r)
        return out


def test_compute_part_reads_its_cache(tmp_path):
    lam_tab = np.geomspace(0.05, 5000.0, 60)
    n, k = M.synthetic_lnk(lam_tab, 0.03)
    (tmp_path / "syn.lnk").write_text("".join("%g %g %g\n" % t for t in zip(lam_tab, n, k)))
    (tmp_path / "dust.particle").write_text("3\n2\n'syn.lnk'\n1.0 3.0\n")
    lam = np.geomspace(0.2, 1000, 16)
    cache = str(tmp_path / "cache")
    ctx = _OracleContext()
    args = (str(tmp_path / "dust.particle"), 0.1, 1.0, 3.5, 0.8, True, 0.25, None, 1, -1.0, "FILE", 1, lam)
    p1 = api.ComputePart(ctx, api.Particle(lam.size), 1, *args, particledir=cache)
    assert ctx.calls == 1 and os.path.exists(os.path.join(cache, "particle0001.fits.gz"))
    p2 = api.ComputePart(ctx, api.Particle(lam.size), 1, *args, particledir=cache)
    assert ctx.calls == 1                                            # read, not computed
    assert np.array_equal(p2.Kabs, p1.Kabs) and np.array_equal(p2.Ksca, p1.Ksca)
    assert np.allclose(p2.F, p1.F, rtol=1e-12, atol=1e-300)
    assert abs(p2.rv[0] / p1.rv[0] - 1) < 1e-6
    # another grain is computed and cached as the next index
    args2 = (str(tmp_path / "dust.particle"), 0.1, 2.0, 3.5, 0.8, True, 0.25, None, 1, -1.0, "FILE", 1, lam)
    api.ComputePart(ctx, api.Particle(lam.size), 2, *args2, particledir=cache)
    assert ctx.calls == 2 and os.path.exists(os.path.join(cache, "particle0002.fits.gz"))
    # the first grain is found again under index 2's lookup (particle0001 .. particle0002)
    api.ComputePart(ctx, api.Particle(lam.size), 2, *args, particledir=cache)
    assert ctx.calls == 2


def test_nspike_flattens_the_forward_peak(tmp_path):
    lam = np.geomspace(0.1, 3000, 8)
    res = _result(lam, 9)
    res["F"][:, 0, :5] *= 50.0          # a forward spike
    path = str(tmp_path / "p.fits")
    PF.write_particle_fits(path, lam, res, **GRAIN)
    plain = PF.read_particle_fits(path, lam)
    flat = PF.read_particle_fits(path, lam, nspike=4)
    s = np.sin(np.pi * (np.arange(1, 181) - 0.5) / 180.0)
    for j in range(lam.size):
        F11 = flat["F"][j, 0]
        assert np.allclose(F11[:4], F11[0]) and abs((F11 * s).sum() / s.sum() - 1) < 1e-13
        # the removed forward part leaves Ksca, the extinction follows
        assert flat["ksca"][j] < plain["ksca"][j] and abs(flat["kext"][j] - flat["kabs"][j] - flat["ksca"][j]) < 1e-9 * flat["kext"][j]
    mixed = PF.read_particle_fits(path, lam, wasym2=0.3, asym2=0.6)
    hg = np.array([PF.hg_binned(0.6, x) for x in (np.arange(1, 181) - 0.5) * np.pi / 180.0])
    assert np.allclose(mixed["F"][2, 0], 0.7 * plain["F"][2, 0] + 0.3 * hg, rtol=1e-12)
