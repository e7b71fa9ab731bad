"""mcg_diffuse on the GPU against the host replay of the same logic and
per-element arithmetic (bit for bit: the library builds the unit with
--fmad=false, the replay with -ffp-contract=off), and against the oracle's
dense DGESV form to rounding."""
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
