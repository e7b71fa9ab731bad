"""The GPU packet loop against the oracle (the CPU restatement of the
reference loop, MCRadiation.f:320-648 with Radiation.f and RandomWalk.f) at
the benchmark decks:

* the plain-method deck as specified: nr 100 x ntheta 60, nlam 100 from 0.1
  to 3000 micron, Mdust 1e-5 Msun, MRN 0.1-1 micron in 20 bins with DHS
  fmax 0.8 and full Mueller scattering, 1e6 packets per run;
* the precision deck's grid: nr 200 x ntheta 120, nlam 200, Mdust 1e-3 Msun,
  random walk (factRW 10), 3e5 packets per run.

Four independent seeds on each side.  Per-cell temperatures (the post-run
determineT of Main.f:498-549) agree within 3 sigma of the combined Monte
Carlo noise, sigma from the seeds' scatter, with no systematic shift; the
SEDs (MCRadiation.f:581-646) agree within 3 sigma in the bins with S/N > 50
and within 2 % where the noise makes 2 % a 3-sigma difference.  The GPU runs
use the library's default launch, which keeps at most one packet in flight
per 1333 packets of the run (the regime of a 1e8-packet run on the whole
GPU); more packets in flight at once move the Bjorkman-Wood temperatures of
optically thick cells away from the serial order.  The oracle runs the seeds
in parallel threads (the C calls release the interpreter lock)."""
import math
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import models
import oracle_ffi as O

pytestmark = pytest.mark.gpu
SEEDS_ORACLE = (101, 102, 103, 104)
SEEDS_GPU = (201, 202, 203, 204)


def _temperatures(m, tab, EJv):
    """determineT per cell from EJv / V (Main.f:503-513), the oracle's
    restatement on the cell's Planck-mean table"""
    L = O.load()
    kp = tab["KpCell"]
    uniform = kp.shape[0] == 1
    T = np.zeros(m.ncell)
    for c in range(m.ncell):
        row = np.ascontiguousarray(kp[0 if uniform else c])
        T[c] = max(L.orc_determine_t(O.P(row), EJv[c] / m.V[c], 100.0), 1.0)
    return T


def _oracle_runs(m, n, run):
    tab = O.transport_tables(m, randomwalk=run.get("randomwalk", False), factRW=run.get("factRW", 10.0),
                             lazy_kd=True)
    with ThreadPoolExecutor(len(SEEDS_ORACLE)) as ex:
        outs = list(ex.map(lambda s: O.mcradiation(m, n, seed=s, tables=tab, **run), SEEDS_ORACLE))
    for o in outs:
        assert o["status"] == 0
    T = np.array([_temperatures(m, tab, o["EJv"]) for o in outs])
    return dict(T=T, Nabs=np.array([o["Nabs"] for o in outs]),
                spec=np.array([o["spec"].reshape(m.nlam, 31) for o in outs]),
                ispec=np.array([o["ispec"].reshape(m.nlam, 31) for o in outs]))


def _gpu_runs(ctx, m, n, prec, run):
    ctx.set_model(m)
    T, Nabs, spec, ispec = [], [], [], []
    for s in SEEDS_GPU:
        n_out, g = ctx.mcradiation(n, seed=s, precision=prec, **run)
        assert n_out == n
        t, _, _ = ctx.finalize_t()
        T.append(t)
        Nabs.append(g["Nabs"])
        spec.append(g["spec"])
        ispec.append(g["ispec"])
    return dict(T=np.array(T), Nabs=np.array(Nabs), spec=np.array(spec), ispec=np.array(ispec))


def _compare(m, ref, gpu):
    """The statistics the assertions use (and that the design notes quote).
    sigma of a mean is the seeds' scatter over sqrt(seeds) on each side (for
    the SED at least the Poisson error of the bin's packet count)."""
    nc = m.nt - 1
    disk = np.arange(m.ncell) >= nc
    na = ref["Nabs"].mean(0)
    sel = disk & (na >= 30)
    k = len(SEEDS_ORACLE)
    mr, mg = ref["T"].mean(0), gpu["T"].mean(0)
    sig = np.sqrt((ref["T"].var(0, ddof=1) + gpu["T"].var(0, ddof=1)) / k) + 1e-9 * mr
    zs = (mg - mr) / sig
    well = disk & (na >= 1e3)
    rel = mg[well] / mr[well] - 1
    out = {"cells_compared": int(sel.sum()), "T_within_3sigma": float(np.mean(np.abs(zs[sel]) < 3)),
           "T_mean_signed_z": float(np.mean(zs[sel])),
           "cells_nabs_ge_1e3": int(well.sum()), "T_median_rel_nabs_ge_1e3": float(np.median(rel)),
           "T_p99_abs_rel_nabs_ge_1e3": float(np.percentile(np.abs(rel), 99))}
    for tag, sl in (("bins", lambda a: a[:, :, 1:]), ("lam", lambda a: a[:, :, 1:].sum(2))):
        A, B = sl(ref["spec"]), sl(gpu["spec"])
        NA, NB = sl(ref["ispec"]).sum(0), sl(gpu["ispec"]).sum(0)
        ma, mb = A.mean(0), B.mean(0)
        ok = (NA > 2500) & (NB > 2500) & (ma > 0)          # S/N > 50 on both sides
        mas = np.where(ma > 0, ma, 1.0)
        s = np.maximum(np.sqrt((A.var(0, ddof=1) + B.var(0, ddof=1)) / k) / mas,
                       np.sqrt(1.0 / np.maximum(NA, 1) + 1.0 / np.maximum(NB, 1)))
        r = mb / mas - 1
        tight = ok & (s < 0.02 / 3)                          # where 2 % is at least 3 sigma
        out["sed_%s_sn50" % tag] = int(ok.sum())
        out["sed_%s_within_3sigma" % tag] = float(np.mean(np.abs(r[ok]) < 3 * s[ok])) if ok.any() else None
        out["sed_%s_tight" % tag] = int(tight.sum())
        out["sed_%s_tight_within_2pct" % tag] = float(np.mean(np.abs(r[tight]) < 0.02)) if tight.any() else None
        out["sed_%s_tight_worst" % tag] = float(np.abs(r[tight]).max()) if tight.any() else None
    return zs[sel], rel, out


def _check(stats, z):
    assert stats["cells_compared"] > 100
    # 4 seeds a side: the scatter estimates follow a t distribution with 6
    # degrees of freedom, so about 97.6 % of the cells fall within 3 sigma
    # (independent oracle seeds: 97 %); the default launch's packets in
    # flight leave about 95 %
    assert stats["T_within_3sigma"] > 0.94, np.sort(np.abs(z))[-10:]
    # no systematic shift: independent oracle seeds give a mean signed z of
    # about +-0.2; a temperature bias of a few tenths of a sigma over all
    # cells shows up here long before it shows in the 3-sigma count
    assert abs(stats["T_mean_signed_z"]) < 0.35, stats
    # SED (wavelength, inclination) bins with S/N > 50: within 3 sigma
    if stats["sed_bins_sn50"]:
        assert stats["sed_bins_within_3sigma"] > 0.95, stats
    # inclination-summed SED where 2 % is a 3-sigma difference: within 2 %
    # (a residual of about 1-2 % remains in the near- and mid-infrared of the
    # hottest dust, from the packets in flight at once)
    if stats["sed_lam_tight"]:
        assert stats["sed_lam_tight_within_2pct"] >= 0.9, stats
        assert stats["sed_lam_tight_worst"] < 0.03, stats


PLAIN = dict(nrad=100, ntheta=60, nlam=100, ngrains=20, ns=5, nf=20, mdust=1e-5)
PRECISION_GRID = dict(nrad=200, ntheta=120, nlam=200, ngrains=20, ns=5, nf=20, mdust=1e-3)
RUN_PRECISION = dict(randomwalk=True, factRW=10.0, maxinteract=100000)


@pytest.fixture(scope="module")
def plain_oracle():
    m = models.small_disk(**PLAIN)
    return m, _oracle_runs(m, 1_000_000, {})


@pytest.fixture(scope="module")
def precision_oracle():
    m = models.small_disk(**PRECISION_GRID)
    return m, _oracle_runs(m, 300_000, RUN_PRECISION)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_plain_deck_matches_oracle(ctx, plain_oracle, prec):
    m, ref = plain_oracle
    gpu = _gpu_runs(ctx, m, 1_000_000, prec, {})
    z, rel, stats = _compare(m, ref, gpu)
    print("plain deck", prec, stats)
    _check(stats, z)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_precision_grid_matches_oracle(ctx, precision_oracle, prec):
    m, ref = precision_oracle
    gpu = _gpu_runs(ctx, m, 300_000, prec, RUN_PRECISION)
    z, rel, stats = _compare(m, ref, gpu)
    print("precision grid", prec, stats)
    _check(stats, z)
