"""The full-model driver (mcmax_b200.full_model) on CPU: its arguments and
the agreement statistics on constructed inputs."""
import numpy as np

from mcmax_b200 import full_model as F
from mcmax_b200.model import Model


def test_defaults_are_the_full_model():
    a = F.parse_args([])
    assert (a.nrad, a.ntheta, a.nlam, a.nphot, a.passes, a.alpha, a.npix) == (300, 200, 300, 10 ** 9, 5, 1e-4, 512)
    assert a.angle_list == [20.0, 45.0, 80.0] and a.lam_list == [1.0, 10.0, 100.0]
    assert (a.scatter_nphot, a.scatter_nstar) == (1000, 1000)


def test_agreement_statistics():
    m = Model(nr=4, nt=4, ncomp=1)
    nc = m.nt - 1
    T = np.full(m.ncell, 100.0)
    Nabs = np.full(m.ncell, 5000)
    Nabs[-1] = 10
    ref = dict(model=m, T=T, Nabs=Nabs, spectra={20.0: np.array([1.0, 2.0, 1e-9])},
               images={(20.0, 10.0): np.array([[1.0, 2.0], [0.0, 4.0]])})
    T2 = T.copy()
    T2[nc] = 103.0
    other = dict(model=m, T=T2, Nabs=Nabs, spectra={20.0: np.array([1.01, 2.1, 5.0])},
                 images={(20.0, 10.0): np.array([[1.0, 2.2], [9.0, 4.0]])})
    ag = F.agreement(ref, other)
    assert ag["cells_nabs_ge_1e3"] == m.ncell - nc - 1
    assert abs(ag["T_within_1pct"] - (1 - 1 / ag["cells_nabs_ge_1e3"])) < 1e-12
    s = ag["spectra"]["20.0"]
    assert s["wavelengths"] == 2 and s["within_2pct"] == 0.5
    im = ag["images"]["20_deg_10_um"]
    assert im["bright_pixels"] == 3 and abs(im["bright_within_5pct"] - 2 / 3) < 1e-12
    assert abs(im["total_flux_ratio"] - 16.2 / 7.0) < 1e-12
