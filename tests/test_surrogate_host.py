"""Host-side pieces of the opacity surrogate: the training box and its
normalisation, the Sobol sampler, folding the output standardisation into
the last layer (checked with the NumPy network reference), the committed
weights file, and the correction of the network's opacities by ComputePart
at a subset of the wavelengths."""
import os

import numpy as np
import pytest

import mlp_ref as R
from mcmax_b200 import surrogate as S


def test_sobol_samples_fill_the_box_and_normalise_to_unit_cube():
    s = S.sobol_samples(4096, seed=4)
    x = S.normalize(s)
    assert x.shape == (4096, 6) and x.min() >= -1.0 - 1e-6 and x.max() <= 1.0 + 1e-6
    assert np.all(np.abs(x.mean(0)) < 0.05)
    assert s[:, 0].min() >= 0.01 * (1 - 1e-9) and s[:, 0].max() <= 1000.0 * (1 + 1e-9)


def test_fold_output_scaling_matches_rescaled_outputs():
    p = R.init(seed=3)
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, (64, R.IN)).astype(np.float32)
    mean = rng.normal(0, 3, R.OUT).astype(np.float32)
    # exact arithmetic: any scale folds into the output layer
    std = rng.uniform(0.1, 5, R.OUT).astype(np.float32)
    y0, _, _ = R.forward(p, x, emulate=False)
    y1, _, _ = R.forward(S.fold_output_scaling(p, mean, std), x, emulate=False)
    assert np.allclose(y1, y0 * std + mean, rtol=1e-5, atol=1e-5)
    # with the kernels' BF16 weights: power-of-two scales fold exactly
    std2 = (2.0 ** np.round(np.log2(std))).astype(np.float32)
    y0, _, _ = R.forward(p, x)
    y1, _, _ = R.forward(S.fold_output_scaling(p, mean, std2), x)
    assert np.allclose(y1, y0 * std2 + mean, rtol=1e-6, atol=1e-5)


def test_committed_weights_file():
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    p, info = S.load(os.path.join(here, "mcmax_b200", "data", "surrogate_nf20.npz"))
    assert p.shape == (R.NP,) and np.all(np.isfinite(p))
    assert int(info["nf"]) == S.NF_TRAIN and float(info["rho"]) == S.RHO_TRAIN
    assert float(info["bins_median_dex_kabs"]) < 0.01


def test_correction_wavelengths_include_both_ends():
    idx = S.correction_wavelengths(200, 10)
    assert idx[0] == 0 and idx[-1] == 199 and np.all(np.diff(idx) > 0) and idx.size == 21
    assert np.array_equal(S.correction_wavelengths(7, 1), np.arange(7))


def test_correct_with_exact_removes_a_smooth_error():
    lam = np.geomspace(0.1, 3000.0, 200)
    ll = np.log10(lam)
    exact_abs = 10.0 ** (2.0 - 0.5 * ll + 0.3 * np.sin(ll))
    exact_sca = 10.0 ** (1.0 - 1.5 * np.tanh(ll))
    parts = [dict(lam=lam), dict(lam=lam), dict(lam=lam)]
    used = np.array([1, 0, 1], np.int32)
    err = 0.01 * np.cos(0.7 * ll)          # smooth log error of the network
    res = [dict(kabs=exact_abs * 10 ** err, ksca=exact_sca * 10 ** -err, F=np.ones((200, 6, 180)))
           for _ in parts]
    res[1] = dict(kabs=exact_abs * 2.0, ksca=exact_sca * 2.0)   # a bin the network did not serve: untouched
    idx = S.correction_wavelengths(200, 10)
    exact = [dict(kabs=exact_abs[idx], ksca=exact_sca[idx]) for _ in (0, 2)]
    out = S.correct_with_exact(res, used, parts, exact, idx)
    for k in (0, 2):
        for key, ref in (("kabs", exact_abs), ("ksca", exact_sca)):
            d = np.abs(np.log10(out[k][key] / ref))
            assert np.all(d[idx] < 1e-12)                 # exact at the evaluated wavelengths
            assert d.max() < 2e-4                          # interpolation error of a smooth error
        assert np.allclose(out[k]["kext"], out[k]["kabs"] + out[k]["ksca"], rtol=1e-15)
    assert np.array_equal(out[1]["kabs"], exact_abs * 2.0)
    with pytest.raises(ValueError):
        S.correct_with_exact(res, used, parts, exact[:1], idx)
