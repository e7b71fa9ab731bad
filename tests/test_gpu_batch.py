"""Several models in one launch (mcg_add_model / mcg_mcradiation_batch).

A model's packets keep their Philox streams inside a batch, so with one
thread (serial packet order) every model sees the same packets as in its
own single-model run.  The batched and single-model kernels are compiled
separately with FMA contraction on, so a rounding difference can tip one
comparison of one packet: the check is agreement of every counter and
accumulator total to a fraction of a percent, not bit identity.  Parallel
batches (autotuned shape, CUDA-graph replay) conserve each model's energy."""
import numpy as np
import pytest

import models
from test_gpu_transport import _energy_out

pytestmark = pytest.mark.gpu


def _three():
    return [models.small_disk(nrad=12, ntheta=8, nlam=24, ngrains=2, ns=2, nf=3),
            models.small_disk(nrad=20, ntheta=12, nlam=30, mdust=1e-4),
            models.small_disk(nrad=16, ntheta=10, nlam=24, ngrains=2, ns=2, nf=3, mdust=1e-3, scat_how=1)]


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_serial_batch_equals_single_runs(ctx, prec):
    ms = _three()
    ids = [ctx.add_model(m) for m in ms]
    nphot, seeds = [300, 200, 250], [5, 6, 7]
    n_out, outs, _ = ctx.mcradiation_batch(ids, nphot, seeds, precision=prec, maxinteract=20000, threads=1)
    assert n_out == nphot
    for m, n, s, b in zip(ms, nphot, seeds, outs):
        ctx.set_model(m)
        _, a = ctx.mcradiation(n, seed=s, precision=prec, maxinteract=20000, threads=1)
        for k in (0, 1, 2, 3, 8, 9):
            assert abs(int(a["counters"][k]) - int(b["counters"][k])) <= 0.005 * int(a["counters"][k]) + 3, k
        for k in ("EJv", "Eabs", "spec"):
            assert abs(b[k].sum() / a[k].sum() - 1) < 0.01, k


def test_parallel_batch_conserves_energy_with_graph_and_autotune(ctx):
    ms = _three()
    ids = [ctx.add_model(m) for m in ms]
    nphot = [20000, 30000, 10000]
    for call in range(2):  # the second call replays the captured graph
        _, outs, info = ctx.mcradiation_batch(ids, nphot, [11 + call, 12 + call, 13 + call], precision="mixed",
                                              maxinteract=100000, autotune=True, use_graph=True)
        assert info["block"] in (128, 256) and info["chunk"] >= 1 and info["device_ms"] > 0
        for m, n, o in zip(ms, nphot, outs):
            c = o["counters"]
            assert int(c[9]) + int(c[7]) + int(c[11]) == n
            assert abs(_energy_out(m, o) / m.Lstar - 1) < 0.03


def test_batch_rejects_bad_arguments(ctx):
    from mcmax_b200.api import McgError
    m = _three()[0]
    i = ctx.add_model(m)
    with pytest.raises(McgError):
        ctx.mcradiation_batch([i, i], [10, 10], [1, 2])
    with pytest.raises(McgError):
        ctx.mcradiation_batch([i + 1000], [10], [1])
