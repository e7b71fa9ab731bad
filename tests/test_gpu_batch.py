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


def test_uneven_models_with_random_walk_match_their_single_runs(ctx):
    """Four models of uneven grids and disk masses, the random walk on (a
    uniform mixture's thick cells share one diffusion row), in one parallel
    launch: each model's packets are accounted for, its energy is conserved,
    and its absorbed energy and SED agree with its own single-model run."""
    ms = [models.small_disk(nrad=12, ntheta=8, nlam=24, ngrains=2, ns=2, nf=3, mdust=1e-3),
          models.small_disk(nrad=24, ntheta=14, nlam=24, ngrains=2, ns=2, nf=3, mdust=1e-2),
          models.small_disk(nrad=16, ntheta=20, nlam=24, ngrains=2, ns=2, nf=3, mdust=1e-4),
          models.small_disk(nrad=30, ntheta=10, nlam=24, ngrains=2, ns=2, nf=3, mdust=3e-3)]
    ids = [ctx.add_model(m) for m in ms]
    nphot = [40000, 60000, 30000, 50000]
    run = dict(precision="mixed", randomwalk=True, factRW=10.0, maxinteract=100000)
    _, outs, info = ctx.mcradiation_batch(ids, nphot, [31, 32, 33, 34], autotune=False, use_graph=False, **run)
    assert info["device_ms"] > 0
    rw_steps = 0
    for m, n, o, s in zip(ms, nphot, outs, (41, 42, 43, 44)):
        c = o["counters"]
        assert int(c[9]) + int(c[7]) + int(c[11]) == n
        assert int(c[11]) == 0
        rw_steps += int(c[4])
        assert abs(_energy_out(m, o) / m.Lstar - 1) < 0.03
        ctx.set_model(m)
        _, a = ctx.mcradiation(n, seed=s, **run)
        assert abs(o["EJv"].sum() / a["EJv"].sum() - 1) < 0.05
        # escaping energy in three inclination ranges (the raw SED total is
        # weighted by 1/dnu and so dominated by the few far-infrared
        # packets), within 4 sigma of the packets' Poisson noise in the range
        eo, ea = _energy_by_inclination(m, o), _energy_by_inclination(m, a)
        no, na = _packets_by_inclination(o), _packets_by_inclination(a)
        tol = 4.0 * np.sqrt(1.0 / np.maximum(no, 1) + 1.0 / np.maximum(na, 1)) + 0.01
        assert np.all(np.abs(eo / ea - 1) < tol), (eo, ea, no, na)
    assert rw_steps > 0


def _packets_by_inclination(out, groups=3):
    return np.asarray(out["ispec"], float).reshape(-1, 31)[:, 1:].sum(0).reshape(groups, -1).sum(1)


def _energy_by_inclination(m, out, groups=3):
    e = _energy_out(m, {"spec": out["spec"]}, per_bin=True)
    return e.sum(0).reshape(groups, -1).sum(1)
