"""GPU packet loop through the C-ABI against the oracle.

Reference-order FP64 kernel with one thread: bit for bit the oracle's
serial loop.  Parallel runs (all three forms): statistical agreement of the
per-cell temperatures and energy bookkeeping."""
import numpy as np
import pytest

import models
import oracle_ffi as O

pytestmark = pytest.mark.gpu
KEYS = ("EJv", "EJv2", "Eabs", "T", "Ni", "spec", "scatspec", "ispec")


@pytest.mark.parametrize("scat_how,rw,mdust,maxint", [(2, False, 1e-5, 0), (1, False, 1e-5, 0), (0, False, 1e-5, 0),
                                                      (2, True, 1e-2, 0), (2, False, 1e-4, 500)])
def test_serial_replay_bit_exact(ctx, scat_how, rw, mdust, maxint):
    m = models.small_disk(mdust=mdust, scat_how=scat_how)
    ctx.set_model(m)
    o = O.mcradiation(m, 150, seed=9, randomwalk=rw, maxinteract=maxint)
    _, g = ctx.mcradiation(150, seed=9, randomwalk=rw, maxinteract=maxint, threads=1, precision="exact")
    assert list(o["counters"][:12]) == list(g["counters"][:12])
    for k in KEYS:
        assert np.array_equal(o[k], g[k]), k


def _energy_out(m, out, per_bin=False):
    # escaping luminosity from the SED bins: spec = wangle*E*wlam with
    # wlam = -1e23/dnu; undo the weights
    nu = m.nu
    dn = np.empty_like(nu)
    dn[0] = nu[1] / 2
    dn[-1] = (nu[-1] - nu[-2]) / 2
    dn[1:-1] = (nu[2:] - nu[:-2]) / 2
    wlam = -1e23 / dn
    cos = np.arange(31) / 30.0
    wang = np.ones(31)
    wang[1:] = 1 / (cos[1:] - cos[:-1])
    e = out["spec"][:, 1:] / (wlam[:, None] * wang[None, 1:])
    return e if per_bin else e.sum()


@pytest.mark.parametrize("prec", ["exact", "fp64", "mixed"])
def test_energy_conservation(ctx, prec):
    m = models.small_disk()
    ctx.set_model(m)
    n, g = ctx.mcradiation(20000, seed=4, precision=prec, maxinteract=100000)
    c = g["counters"]
    escaped = int(c[9])
    killed = int(c[7]) + int(c[11])
    assert escaped + killed == 20000
    # escaping energy = packets that left * E (E = Lstar/N, boosted by the roulette)
    assert abs(_energy_out(m, g) / m.Lstar - 1) < 0.02


@pytest.mark.parametrize("prec", ["exact", "fp64", "mixed"])
def test_temperatures_statistically_match_oracle(ctx, prec):
    """Per-cell temperature of a parallel GPU run vs the serial oracle:
    cells with many packets agree within 3 sigma of the combined MC noise
    (sigma from the independent-seed scatter of the oracle)."""
    m = models.small_disk(nrad=12, ntheta=8, nlam=24, ngrains=2, ns=2, nf=3)
    N = 4000
    ctx.set_model(m)
    tab = O.transport_tables(m)
    L = O.load()
    kp = np.ascontiguousarray(tab["KpCell"][0])

    def temps(EJv):
        return np.array([L.orc_determine_t(O.P(kp), EJv[c] / m.V[c], 100.0) for c in range(m.ncell)])

    ref = np.array([temps(O.mcradiation(m, N, seed=100 + s, tables=tab, maxinteract=100000)["EJv"])
                    for s in range(4)])
    gpu = []
    for s in range(4):
        ctx.mcradiation(N, seed=200 + s, precision=prec, maxinteract=100000)
        T, dT, dE = ctx.finalize_t()
        gpu.append(T)
    gpu = np.array(gpu)
    i = np.arange(m.ncell) // (m.nt - 1)
    sel = i > 0
    mr, mg = ref.mean(0)[sel], gpu.mean(0)[sel]
    sr, sg = ref.std(0, ddof=1)[sel], gpu.std(0, ddof=1)[sel]
    sig = np.sqrt((sr ** 2 + sg ** 2) / 4) + 1e-3 * mr
    z = np.abs(mr - mg) / sig
    assert np.mean(z < 3) > 0.95, np.sort(z)[-5:]
    well = sr < 0.02 * mr  # cells the oracle resolves to 2 %
    assert well.sum() > 10
    assert np.all(np.abs(mg / mr - 1)[well] < 0.1)


def test_finalize_matches_oracle_determine_t(ctx):
    m = models.small_disk()
    ctx.set_model(m)
    _, g = ctx.mcradiation(2000, seed=3, precision="exact")
    T, dT, dE = ctx.finalize_t()
    tab = O.transport_tables(m)
    L = O.load()
    kp = np.ascontiguousarray(tab["KpCell"][0])
    nc = m.nt - 1
    for c in range(nc, m.ncell, 7):
        ref = L.orc_determine_t(O.P(kp), g["EJv"][c] / m.V[c], g["T"][c])
        ref = max(ref, 1.0)
        assert T[c] == ref


def test_nruns_concurrent_subruns(ctx):
    m = models.small_disk()
    ctx.set_model(m)
    n, a = ctx.mcradiation(6000, seed=8, nruns=3, precision="fp64", maxinteract=100000)
    assert n == 6000
    c = a["counters"]
    assert int(c[9]) + int(c[7]) == 6000
    assert abs(_energy_out(m, a) / m.Lstar - 1) < 0.03


def test_invalid_run_arguments(ctx):
    from mcmax_b200.api import McgError
    m = models.small_disk()
    ctx.set_model(m)
    for kw in (dict(nphot=0), dict(nphot=10, maxinteract=1), dict(nphot=10, randomwalk=True, factRW=0.0)):
        n = kw.pop("nphot")
        with pytest.raises(McgError):
            ctx.mcradiation(n, **kw)


def test_settled_mixture_fast_forms_match_reference_order(ctx):
    """Per-cell grain mixtures (vertical settling, three compositions): the
    GPU-ordered kernels, which scan each cell's re-emission spectrum and
    component list in blocks, agree with the reference-order kernel within
    the Monte Carlo noise of independent seeds."""
    from mcmax_b200 import model as M
    m, _, _ = M.learned_disk_model(ctx, opacity="dhs", nrad=16, ntheta=10, nlam=24, ngrains=3, ns=2, nf=4,
                                   mdust=1e-4)
    assert not np.allclose(m.comp_w[m.nt - 2], m.comp_w[(m.nt - 1) * 5 + 1])  # mixtures differ by cell
    ctx.set_model(m)
    N = 20000

    def temps(prec, seeds):
        out = []
        for s in seeds:
            ctx.mcradiation(N, seed=s, precision=prec, maxinteract=100000)
            T, _, _ = ctx.finalize_t()
            out.append(T)
        return np.array(out)

    ref = temps("exact", range(300, 304))
    i = np.arange(m.ncell) // (m.nt - 1)
    sel = i > 0
    mr, sr = ref.mean(0)[sel], ref.std(0, ddof=1)[sel]
    for prec in ("fp64", "mixed"):
        g = temps(prec, range(400, 404))
        mg, sg = g.mean(0)[sel], g.std(0, ddof=1)[sel]
        z = np.abs(mr - mg) / (np.sqrt((sr ** 2 + sg ** 2) / 4) + 1e-3 * mr)
        assert np.mean(z < 3) > 0.95, (prec, np.sort(z)[-5:])


@pytest.mark.parametrize("prec", ["exact", "fp64", "mixed"])
def test_absorption_events_per_cell(ctx, prec):
    """Nabs counts the absorption events of each cell: they add up to the
    run's absorption counter, and only cells with matter absorb."""
    m = models.small_disk()
    ctx.set_model(m)
    _, g = ctx.mcradiation(5000, seed=21, precision=prec, maxinteract=100000, nruns=2)
    assert int(g["Nabs"].sum()) == int(g["counters"][2]) > 0
    star_cells = np.arange(m.ncell) < (m.nt - 1)
    assert g["Nabs"][star_cells].sum() == 0


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_maxruntime_shrinks_the_run(ctx, prec):
    """maxruntime (MCRadiation.f:323-342): a run that would take longer
    starts over with NphotTot (maxruntime / t) (0.5 i / Nphot) packets, and
    the packets of the run that finished are all accounted for."""
    m = models.small_disk()
    ctx.set_model(m)
    n0 = 4_000_000
    _, full = ctx.mcradiation(n0, seed=22, precision=prec, maxinteract=100000)
    # packets start at a steady rate until the counter runs out, then the
    # tail finishes: a limit of a tenth of the time half the packets took
    # stops the run with far fewer than 90 % of the packets started
    limit = full["progress_ms"][0] * 1e-3 / 10.0
    n, g = ctx.mcradiation(n0, seed=22, precision=prec, maxinteract=100000, maxruntime=limit)
    assert 10 <= n < n0 // 4, (n, limit)
    c = g["counters"]
    assert int(c[9]) + int(c[7]) + int(c[11]) == n
    # an unlimited run is left alone
    n2, _ = ctx.mcradiation(20000, seed=23, precision=prec, maxinteract=100000, maxruntime=1e6)
    assert n2 == 20000


def test_single_precision_t4_replays_the_oracle(ctx):
    """mcg_run.t4_single: the reference's single-precision real(i)**4 in
    increaseT and determineT (Radiation.f:551, 584, 698); the serial replay
    and the post-run temperatures equal the oracle's with the same switch,
    bit for bit, and differ from the FP64 form by under 1e-6"""
    import oracle_ffi as OF
    m = models.small_disk(mdust=1e-4)
    ctx.set_model(m)
    L = OF.load()
    L.orc_set_t4_single(1)
    try:
        o = O.mcradiation(m, 150, seed=9)
    finally:
        L.orc_set_t4_single(0)
    _, g = ctx.mcradiation(150, seed=9, threads=1, precision="exact", t4_single=True)
    assert list(o["counters"][:12]) == list(g["counters"][:12])
    for k in KEYS:
        assert np.array_equal(o[k], g[k]), k
    Ts, _, _ = ctx.finalize_t()
    _, g64 = ctx.mcradiation(150, seed=9, threads=1, precision="exact")
    T64, _, _ = ctx.finalize_t()
    ok = (T64 > 1.0) & (Ts > 1.0)
    rel = np.abs(Ts[ok] / T64[ok] - 1)
    assert rel.max() < 1e-6 and np.any(Ts[ok] != T64[ok])
