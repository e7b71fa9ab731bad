"""mcg_diffuse and mcg_disk_structure on the GPU against the host replays
of the same logic and per-element arithmetic (bit for bit: the library
builds both units with --fmad=false, the replay with -ffp-contract=off, and
the structure step takes exp and log from detmath.h), mcg_disk_structure
against the oracle's restatement of DiskStructure bit for bit, and
mcg_diffuse against the oracle's dense DGESV form to rounding."""
import numpy as np
import pytest

import hostcheck_ffi as H
import models
import oracle_ffi as O

pytestmark = pytest.mark.gpu


def test_diffuse_matches_replay_and_oracle(ctx):
    m = models.small_disk(nrad=24, ntheta=16, nlam=24, mdust=1e-3)
    tb = O.transport_tables(m, randomwalk=True, factRW=10.0)
    nc = m.nt - 1
    rng = np.random.default_rng(1)
    R_av = np.sqrt(m.R[:-1] * m.R[1:])
    T = (400.0 * R_av[:, None] ** -0.5 * (1 + 0.3 * np.linspace(1, 0, nc))[None, :]
         * rng.uniform(0.9, 1.1, (m.nr, nc))).ravel()
    Ni = np.full(m.ncell, 1000, np.int32)
    thick = tb["thick"].reshape(m.nr, nc)
    Ni.reshape(m.nr, nc)[thick == 1] = rng.integers(0, 20, int(thick.sum()))
    dT = 0.05 * T
    ctx.set_model(m)
    Tg, Eg, counts = ctx.diffuse(Ni, dT, T)
    Th, Eh, sh = H.diffuse(m, tb, Ni, dT, T)
    assert counts == tuple(int(x) for x in sh[:4])
    assert counts[2] > 30 and counts[3] == 0
    assert np.array_equal(Tg, Th)
    assert np.array_equal(np.isnan(Eg), np.isnan(Eh)) and np.array_equal(Eg[~np.isnan(Eg)], Eh[~np.isnan(Eh)])
    To, _, _, so = O.diffuse(m, tb, Ni, dT, T)
    assert np.max(np.abs(Tg / To - 1)) < 1e-12


def test_disk_structure_matches_replay_and_oracle(ctx):
    from mcmax_b200 import model as M
    m = models.small_disk(nrad=20, ntheta=14, nlam=16, mdust=1e-4, ngrains=2)
    nc = m.nt - 1
    R_av = np.sqrt(m.R[:-1] * m.R[1:])
    Temp = np.maximum((300.0 * R_av[:, None] ** -0.5 * (1 + 0.5 * np.linspace(1, 0, nc))[None, :]).ravel(), 2.7)
    dens = np.maximum(m.dens, 1e-50)
    w = m.comp_w.copy()
    gs = np.ones((m.ncomp, m.nr))
    gs[1] = 0.7
    zones = [(0.5, 10.0, 0.0707, 1.0, 1.125, 1.0, 1), (10.0, 100.0, 0.0707, 1.0, 1.125, 1.0, 0)]
    got = ctx.disk_structure(m.R, m.Theta, m.V, 2.5 * M.MSUN, zones, Temp, dens, dens, dens, w, w, grain_scale=gs)
    st = dict(nr=m.nr, nt=m.nt, ng=m.ncomp, R=m.R, Theta=m.Theta, V=m.V, Mstar=2.5 * M.MSUN, zones=zones,
              grain_scale=gs)
    ref = H.disk_structure(st, Temp, dens, dens, dens, w.ravel(), w.ravel())
    orc = O.disk_structure(st, Temp, dens, dens, dens, w.ravel(), w.ravel())
    for a, b, c, name in zip(got, ref, orc, ("dens", "dens0", "gasdens", "w", "w0")):
        assert np.array_equal(np.ravel(a), np.ravel(b)), name
        assert np.array_equal(np.ravel(a), np.ravel(c)), name


def test_scale_height_types_match_oracle(ctx):
    """a grain of every scale-height type (DiskStructure.f:248-344): the
    device against the oracle bit for bit"""
    from test_dstruct import SHAPES, _shape_case, _temp
    m, s, st, gs = _shape_case()
    T = _temp(m)
    got = ctx.disk_structure(m.R, m.Theta, m.V, st["Mstar"], st["zones"], T, s["dens"], s["dens0"], s["gasdens"],
                             s["w"], s["w0"], grain_scale=gs, shtype=list(SHAPES))
    orc = O.disk_structure(st, T, s["dens"], s["dens0"], s["gasdens"], s["w"].ravel(), s["w0"].ravel())
    for a, c, name in zip(got, orc, ("dens", "dens0", "gasdens", "w", "w0")):
        assert np.array_equal(np.ravel(a), np.ravel(c)), name
