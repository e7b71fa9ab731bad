"""Host-side pieces of the opacity surrogate: the training box and its
normalisation, the Sobol sampler, folding the output standardisation into
the last layer (checked with the NumPy network reference), and the
committed weights file."""
import os

import numpy as np

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
