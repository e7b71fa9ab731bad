"""Train the opacity surrogate on the GPU and write its weights.

    python -m mcmax_b200.train_surrogate --samples 2000000 --out surrogate.npz

Samples: a scrambled Sobol sequence over the training box (see surrogate.py);
targets: ComputePart on the GPU for each sample (one grain size, nf = 20,
material density 3 g/cm^3); training: the tensor-core forward/backward
kernels with Adam.  Prints the held-out error of the network and its error
on the learned-opacities deck's 150 grain bins (200 wavelengths) against the
DHS kernels: kappa_abs and kappa_sca in dex, and the polarisation elements
F33 and F34 as the median of |F_net - F_DHS| / F11_DHS over the angles."""
import argparse
import json
import time

import numpy as np

from . import api
from . import surrogate as S


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--samples", type=int, default=1 << 21)
    ap.add_argument("--test", type=int, default=20_000)
    ap.add_argument("--epochs", type=int, default=300)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--pol-weight", type=float, default=float(S.OUT_WEIGHT[27]),
                    help="loss weight of the F33 and F34 moments")
    ap.add_argument("--out", default="surrogate.npz")
    a = ap.parse_args()
    ctx = api.Context(0)
    t0 = time.perf_counter()
    X = S.sobol_samples(a.samples, seed=a.seed)
    T = S.targets(ctx, X)
    t_targets = time.perf_counter() - t0
    w = S.OUT_WEIGHT.copy()
    w[27:53] = a.pol_weight
    params, info = S.train(ctx, X, T, epochs=a.epochs, batch=a.batch, lr=a.lr, lr_min=a.lr * 1e-2, seed=a.seed,
                           weights=w)
    Xt = S.sobol_samples(a.test, seed=a.seed + 1000)
    Tt = S.targets(ctx, Xt)
    Y = ctx.mlp_forward(S.normalize(Xt))
    err = np.abs(Y - Tt)
    info.update(targets_s=t_targets, test_n=a.test,
                test_median_dex_kabs=float(np.median(err[:, 0])), test_p95_dex_kabs=float(np.percentile(err[:, 0], 95)),
                test_median_dex_ksca=float(np.median(err[:, 1])), test_p95_dex_ksca=float(np.percentile(err[:, 1], 95)),
                test_median_g=float(np.median(err[:, 2])))
    from . import model as M
    lam, _ = M.wavelength_grid(0.1, 3000.0, 200)
    parts, _ = M.learned_disk_parts(lam)
    got, used = S.compute_part_surrogate(ctx, parts, params)
    ref = ctx.compute_part_batch(parts)
    lk = np.concatenate([np.log10(g["kabs"] / r["kabs"]) for g, r in zip(got, ref)])
    ls = np.concatenate([np.log10(g["ksca"] / r["ksca"]) for g, r in zip(got, ref)])
    f33 = np.concatenate([(np.abs(g["F"][:, 3] - r["F"][:, 3]) / r["F"][:, 0]).ravel() for g, r in zip(got, ref)])
    f34 = np.concatenate([(np.abs(g["F"][:, 4] - r["F"][:, 4]) / r["F"][:, 0]).ravel() for g, r in zip(got, ref)])
    info.update(bins_served=int(np.sum(used)), bins_median_dex_kabs=float(np.median(np.abs(lk))),
                bins_median_dex_ksca=float(np.median(np.abs(ls))), bins_median_f33_rel=float(np.median(f33)),
                bins_median_f34_rel=float(np.median(f34)), kappa_weight=float(w[0]), pol_weight=float(a.pol_weight))
    S.save(a.out, params, info)
    print(json.dumps({k: (v.tolist() if isinstance(v, np.ndarray) else v) for k, v in info.items()}))


if __name__ == "__main__":
    main()
