"""The command-line runner's wiring on CPU: deck keywords reach the packet
loop's run parameters, the result files are written and read back.  The
context is a stand-in that records the calls; the transport itself is
covered by the GPU tests."""
import os

import numpy as np

import oracle_ffi as O
from mcmax_b200 import model as M
from mcmax_b200 import outputs, run as R

DECK = """tstar=5000
rstar=2
rin=1
rout=50
nrad=6
ntheta=6
lam1=0.2
lam2=1000
nlam=12
zone1:rin=1
zone1:rout=50
zone1:mdust=1d-6
zone1:fix=.true.
scattype='ISOTROPIC'
computepart01:file='dust.particle'
computepart01:amin=0.1
computepart01:amax=0.5
computepart01:ngrains=2
maxinteract=5000
nruns=2
idum=-11
"""


def _oracle_parts(parts):
    return [O.compute_part(p["lam"], p["e1"][0], p["e2"][0], p["frac"], p["rho"], p["amin"], p["amax"],
                           p["apow"], p["fmax"], p["blend"], p["porosity"], p["ns"], p["nf"]) for p in parts]


class FakeContext:
    def __init__(self, device=0):
        self.calls = []
        self.closed = False

    def compute_part_batch(self, parts):
        return _oracle_parts(parts)

    def set_model(self, m):
        self.model = m

    def mcradiation(self, nphot, **run):
        self.calls.append(dict(nphot=nphot, **run))
        m = self.model
        rng = np.random.default_rng(0)
        ns = (m.nlam, 31)
        return nphot, dict(spec=rng.uniform(1e20, 1e21, ns), scatspec=np.zeros(ns),
                           ispec=rng.integers(1, 100, ns).astype(np.int32), Ni=np.full(m.ncell, 7, np.int32))

    def diffuse(self, Ni, dT, T, nphotmin, dtmax, factRW):
        self.diffuse_args = (int(Ni[0]), nphotmin, dtmax, factRW)
        T = np.array(T)
        T[-1] = 555.0
        return T, np.full(T.size, np.nan), (1, 5, 1, 0)

    def finalize_t(self):
        T = np.linspace(20.0, 900.0, self.model.ncell)
        return T, 0 * T, 0 * T

    def trace_spectrum(self, T, lam_obs, angle, nphi=45, nr=2, Rfix=(), scatter=None):
        self.trace_args = (angle, nphi, nr, tuple(Rfix))
        self.scatter_args = scatter
        return np.full(len(lam_obs), 1e20), (100, 0)

    def disk_structure(self, R, Theta, V, Mstar, zones, Temp, dens, dens0, gasdens, w, w0, shscale=None,
                       grain_scale=None, shtype=None):
        self.structure_calls = getattr(self, "structure_calls", 0) + 1
        self.structure_zones = zones
        self.grain_scales = getattr(self, "grain_scales", []) + [grain_scale]
        return (np.array(dens), np.array(dens0), np.array(gasdens), np.array(w), np.array(w0))

    def trace_image(self, T, lam0, angle, npixel=500, nint=1000, Rmax=None, pa=0.0, nphi=45, nr=2, Rfix=(),
                    seed=42, lam_path=None, scatter=None):
        self.image_args = dict(lam0=lam0, angle=angle, npixel=npixel, nint=nint, Rmax=Rmax, pa=pa, nphi=nphi, nr=nr,
                               seed=seed, lam_path=lam_path, scatter=scatter)
        self.image_calls = getattr(self, "image_calls", []) + [self.image_args]
        R = np.linspace(0.0, 50.0, 11)
        return dict(image=np.full((npixel, npixel), 2.0), flux=1.0, R=R, rphi=np.ones((R.size, nphi)),
                    info=(R.size, 0))

    def close(self):
        self.closed = True


def _write_inputs(d):
    lam_tab = np.geomspace(0.05, 5000.0, 60)
    n, k = M.synthetic_lnk(lam_tab, 0.03)
    (d / "syn.lnk").write_text("".join("%g %g %g\n" % t for t in zip(lam_tab, n, k)))
    (d / "dust.particle").write_text("1\n1\n'syn.lnk'\n1.0 3.0\n")
    (d / "disk.in").write_text(DECK)
    return str(d / "disk.in")


def test_command_line_runs_the_deck_and_writes_result_files(tmp_path):
    deck = _write_inputs(tmp_path)
    out = tmp_path / "out"
    made = []

    def factory(device):
        made.append(FakeContext(device))
        return made[-1]

    r = R.main([deck, "2e4", "-o", str(out), "-s", "randomwalk=.true.", "-s", "factrw=4",
                "--precision", "fp64", "--spectrum", "30", "--spectrum-nphi", "20"], context=factory)
    ctx = made[0]
    assert ctx.closed
    assert ctx.calls == [dict(nphot=20000, precision="fp64", seed=11, randomwalk=True, factRW=4.0,
                              maxinteract=5000, maxruntime=-1.0, nruns=2)]
    assert ctx.diffuse_args == (7, 25, 1.0, 4.0) and r["diffused"] == (1, 5, 1, 0)
    # a deck with zones starts from three structure passes (a fixed zone's
    # profile rebuilt at the cell centres), as the reference's Init does
    assert ctx.structure_calls == 3 and ctx.structure_zones == [(1.0, 50.0, 0.01, 1.0, 1.1, 1.0, True)]
    assert len(r["files"]) == 33 and all(os.path.exists(f) for f in r["files"])
    assert os.path.basename(r["files"][-1]) == "spectrum30.0.dat"
    assert made[0].trace_args[1:] == (20, 2, ()) and abs(made[0].trace_args[0] - np.radians(30)) < 1e-15
    d = outputs.read_denstemp(str(out / "denstemp.dat"))
    m = r["model"]
    assert d["T"].shape == (m.nr - 1, m.nt - 1)
    assert np.allclose(d["T"].ravel(), r["T"].reshape(m.nr, m.nt - 1)[1:].ravel(), rtol=1e-15)
    assert np.allclose(d["dens"].ravel(), m.dens.reshape(m.nr, m.nt - 1)[1:].ravel(), rtol=1e-15)
    assert np.allclose(d["comp"].sum(-1), 1.0)
    # isotropic scattering: the phase matrices are unit, sizes from the deck
    assert m.scat_how == 1 and m.bins[0][0] == 0.1 and abs(m.bins[-1][1] - 0.5) < 1e-12


def test_observation_files_drive_spectra(tmp_path):
    deck = _write_inputs(tmp_path)
    (tmp_path / "Spectrum.out").write_text("nphi=30\nnrad=1\nnphot=300\n*****\ntype='SPECTRUM'\ninc=60\n"
                                           "flag='_a'\n"
                                           "type='IMAGE'\nlam=0.6\nnpix=16\nnint=3\nnphotstar=70\nnexits=0\n"
                                           "type='SPECTRUM'\nlam1=1\nlam2=100\nnlam=5\n"
                                           "type='LINE'\n")
    made = []

    def factory(device):
        made.append(FakeContext(device))
        return made[-1]

    r = R.main([deck, "1e3", str(tmp_path / "Spectrum.out"), "-o", str(tmp_path / "o")], context=factory)
    names = [os.path.basename(f) for f in r["files"] if "spectrum" in f]
    assert names == ["spectrum60.0_a.dat", "spectrum45.0.dat"]
    assert r["skipped"] == ["LINE"]
    images = [os.path.basename(f) for f in r["files"] if "Image" in f]
    assert images == ["RImage_i45.0_l00000.60.dat", "ImageAI_i45.0_l00000.60_fov00100.0.fits"]
    a = made[0].image_args
    rout = float(r["model"].R[-1])
    assert (a["lam0"], a["npixel"], a["nint"], a["Rmax"], a["nphi"], a["nr"], a["pa"]) == (0.6, 16, 3, rout, 30, 1, 0.0)
    hdr, im = outputs.read_image_fits(str(tmp_path / "o" / images[1]))
    d = 100.0 * outputs.PARSEC
    assert im.shape == (16, 16) and np.allclose(im, 2.0 * 1e23 / d ** 2, rtol=1e-15)
    assert abs(hdr["CRVAL1"] / -rout - 1) < 1e-10 and abs(hdr["CDELT2"] / (2 * rout / 16) - 1) < 1e-10
    assert hdr["CTYPE1"].strip() == "X [AU]"
    rows = np.loadtxt(str(tmp_path / "o" / "spectrum45.0.dat"))
    assert rows.shape[0] == 5 and np.allclose(rows[[0, -1], 0], [1.0, 100.0])
    assert made[0].trace_args[1:3] == (30, 1)
    # the observations' scattered-light packets (Telescope.f:943-973)
    assert made[0].scatter_args == dict(nphot=300, nphot_star=1000, seed=11, nexits=5)
    assert a["scatter"] == dict(nphot=300, nphot_star=70, seed=11, nexits=0)


def test_command_line_arguments():
    a = R.parse_args(["x.in", "1e6"])
    assert (a.nphot, a.outdir, a.overrides, a.precision, a.opacity) == (1000000, ".", [], "mixed", "dhs")
    a = R.parse_args(["x.in", "300", "obs.out", "-o", "o", "-s", "a=1", "-s", "b=2", "--opacity", "surrogate"])
    assert (a.nphot, a.outdir, a.overrides, a.opacity, a.observations) == (300, "o", ["a=1", "b=2"], "surrogate",
                                                                            ["obs.out"])


def test_power_law_deck_starts_from_the_thin_structure(tmp_path):
    deck = _write_inputs(tmp_path)
    made = []

    def factory(device):
        made.append(FakeContext(device))
        return made[-1]

    body = open(deck).read().replace("zone1:rin=1\nzone1:rout=50\nzone1:mdust=1d-6\nzone1:fix=.true.\n", "")
    (tmp_path / "pow.in").write_text(body + "denstype='POW'\nmdust=1d-6\n")
    r = R.main([str(tmp_path / "pow.in"), "1e3", "-o", str(tmp_path / "o")], context=factory)
    # three structure passes before the one packet run, no zones
    assert made[0].structure_calls == 3 and made[0].structure_zones == []
    assert len(made[0].calls) == 1 and r["structure"] is None


def test_ifu_observation_writes_one_image_per_wavelength(tmp_path):
    deck = _write_inputs(tmp_path)
    (tmp_path / "ifu.out").write_text("type='IFU'\nlam1=1\nlam2=100\nnlam=3\nnpix=8\nnint=2\nfov=40\n")
    made = []

    def factory(device):
        made.append(FakeContext(device))
        return made[-1]

    r = R.main([deck, "1e3", str(tmp_path / "ifu.out"), "-o", str(tmp_path / "o")], context=factory)
    names = [os.path.basename(f) for f in r["files"] if "Image" in f]
    assert names == ["ImageAI_i45.0_l00001.00_fov00040.0.fits", "ImageAI_i45.0_l00010.00_fov00040.0.fits",
                     "ImageAI_i45.0_l00100.00_fov00040.0.fits"]
    calls = made[0].image_calls
    assert [c["lam0"] for c in calls] == [1.0, 10.0, 100.0]
    assert all(c["lam_path"] == 0.55 and c["Rmax"] == 20.0 and c["npixel"] == 8 for c in calls)
    assert len({c["seed"] for c in calls}) == 3


def test_visibility_observation(tmp_path):
    deck = _write_inputs(tmp_path)
    (tmp_path / "vis.out").write_text("type='VISIBILITY'\nlam1=1\nlam2=100\nnlam=3\nbase1=50\nbase2=200\n"
                                      "angle2=30\n")
    made = []

    def factory(device):
        made.append(FakeContext(device))
        return made[-1]

    r = R.main([deck, "1e3", str(tmp_path / "vis.out"), "-o", str(tmp_path / "o")], context=factory)
    path = [f for f in r["files"] if os.path.basename(f).startswith("visibility")]
    assert [os.path.basename(p) for p in path] == ["visibility45.0.dat"]
    rows = np.loadtxt(path[0])
    assert rows.shape == (3, 2 + 2 + 2)
    assert np.all((rows[:, 2:4] >= 0.0) & (rows[:, 2:4] <= 1.0 + 1e-12))
    head = open(path[0]).read().splitlines()[:4]
    assert head[3].startswith("# column   4 and   6: vis and phase for: baseline    200.000, angle     30.000")
    assert all(c["lam_path"] == 0.55 and c["npixel"] == 1 for c in made[0].image_calls)


def test_basevis_observation(tmp_path):
    deck = _write_inputs(tmp_path)
    (tmp_path / "bv.out").write_text("type='BASEVIS'\nlam1=2\nlam2=2\nlam3=10\nbase1=10\nbase2=110\nangle3=45\n")
    made = []

    def factory(device):
        made.append(FakeContext(device))
        return made[-1]

    r = R.main([deck, "1e3", str(tmp_path / "bv.out"), "-o", str(tmp_path / "o")], context=factory)
    path = [f for f in r["files"] if os.path.basename(f).startswith("basevis")]
    assert [os.path.basename(p) for p in path] == ["basevis45.0.dat"]
    rows = np.loadtxt(path[0])
    assert rows.shape == (100, 2 + 3 + 3)
    assert rows[0, 0] == 10.0 and rows[-1, 0] == 110.0
    # the same wavelength twice is traced once
    calls = made[0].image_calls
    assert [c["lam0"] for c in calls] == [2.0, 10.0] and all(c["lam_path"] == 2.0 for c in calls)
    head = open(path[0]).read().splitlines()
    assert head[4].startswith("# column   5 and   8: vis and phase for wavelength     10.000, angle     45.000")


def test_image_in_arcsec(tmp_path):
    """scaletype 2: the field of view in arcsec becomes AU at the distance
    (100 pc), the header counts arcsec and the image is in mJy/arcsec^2"""
    deck = _write_inputs(tmp_path)
    (tmp_path / "im.out").write_text("type='IMAGE'\nlam=1\nnpix=10\nnint=2\nfov=0.4\nscaletype=2\n")
    made = []

    def factory(device):
        made.append(FakeContext(device))
        return made[-1]

    r = R.main([deck, "1e3", str(tmp_path / "im.out"), "-o", str(tmp_path / "o")], context=factory)
    a = made[0].image_args
    assert abs(a["Rmax"] - 0.4 * 100.0 / 2.0) < 1e-9
    fits = [f for f in r["files"] if os.path.basename(f).startswith("ImageAI")]
    hdr, im = outputs.read_image_fits(fits[0])
    assert hdr["CTYPE1"].strip() == "X [arcsec]" and abs(hdr["CDELT1"] - 0.4 / 10) < 1e-12
    d = 100.0 * outputs.PARSEC
    zscale = 1e3 * (10 / 0.4) ** 2
    assert np.allclose(im, 2.0 * 1e23 * zscale / d ** 2, rtol=1e-12)


def test_fixed_settling_deck_starts_with_settled_structure_passes(tmp_path):
    """fixmpset: the optically thin start runs (Init.f:3923-3927) and every
    structure pass gets FixedMPSettling's factors (DiskStructure.f:108)"""
    deck = _write_inputs(tmp_path)
    made = []

    def factory(device):
        made.append(FakeContext(device))
        return made[-1]

    R.main([deck, "1e3", "-o", str(tmp_path / "o"), "-s", "fixmpset=.true.", "-s", "alphaturb=1d-3"], context=factory)
    ctx = made[0]
    assert ctx.structure_calls == 3
    assert all(g is not None and g.shape[0] == 2 and np.all((g[:, 1:] > 0) & (g[:, 1:] <= 1)) for g in ctx.grain_scales)
