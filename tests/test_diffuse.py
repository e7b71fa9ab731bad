"""Diffuse (Diffusion.f:9-330) on CPU: the host logic of mcg_diffuse with
its kernels replaced by serial loops over the same per-element functions
(tests/native/hostcheck.cpp) against the oracle's restatement on the dense
system with DGESV's elimination (oracle/oracle_diffuse.c)."""
import numpy as np
import pytest

import hostcheck_ffi as H
import models
import oracle_ffi as O


@pytest.fixture(scope="module")
def thick_disk():
    m = models.small_disk(nrad=24, ntheta=16, nlam=24, mdust=1e-3)
    tb = O.transport_tables(m, randomwalk=True, factRW=10.0)
    assert tb["thick"].sum() > 40
    return m, tb


def _fields(m, tb, seed=1):
    nc = m.nt - 1
    rng = np.random.default_rng(seed)
    R_av = np.sqrt(m.R[:-1] * m.R[1:])
    T = (400.0 * R_av[:, None] ** -0.5 * (1 + 0.3 * np.linspace(1, 0, nc))[None, :]
         * rng.uniform(0.9, 1.1, (m.nr, nc))).ravel()
    Ni = np.full(m.ncell, 1000, np.int32)
    thick = tb["thick"].reshape(m.nr, nc)
    Ni.reshape(m.nr, nc)[thick == 1] = rng.integers(0, 20, int(thick.sum()))
    return T, 0.05 * T, Ni


def test_band_solution_matches_the_dense_dgesv_form(thick_disk):
    m, tb = thick_disk
    T, dT, Ni = _fields(m, tb)
    To, Eo, _, so = O.diffuse(m, tb, Ni, dT, T)
    Th, Eh, sh = H.diffuse(m, tb, Ni, dT, T)
    assert list(sh[:4]) == list(so), (sh, so)
    assert so[0] > 30 and so[2] > 30
    changed = To != T
    assert changed.sum() == so[2]
    # two stable eliminations of one M-matrix: equal to rounding
    assert np.max(np.abs(Th / To - 1)) < 1e-12
    same = np.floor(Th) == np.floor(To)
    assert np.array_equal(np.isnan(Eh), np.isnan(Eo))
    assert np.array_equal(Eh[same & ~np.isnan(Eh)], Eo[same & ~np.isnan(Eo)])
    # a diffused temperature lies between its neighbours' extremes
    assert np.all(Th[changed] > 0.5 * T.min()) and np.all(Th[changed] < 2 * T.max())


def test_uniform_temperature_is_a_fixed_point(thick_disk):
    m, tb = thick_disk
    _, _, Ni = _fields(m, tb)
    T = np.full(m.ncell, 321.0)
    Th, Eh, sh = H.diffuse(m, tb, Ni, 0.05 * T, T)
    assert sh[2] > 0
    # zero row sums: a constant T^4 solves every stencil row
    assert np.max(np.abs(Th / 321.0 - 1)) < 1e-12


def test_nothing_to_diffuse_leaves_everything_alone(thick_disk):
    m, tb = thick_disk
    T, dT, Ni = _fields(m, tb)
    Ni[:] = 10 ** 6
    Th, Eh, sh = H.diffuse(m, tb, Ni, dT, T)
    To, Eo, _, so = O.diffuse(m, tb, Ni, dT, T)
    assert list(sh[:4]) == [0, 0, 0, 0] == list(so)
    assert np.array_equal(Th, T) and np.all(np.isnan(Eh))


def test_error_criterion_and_empty_thin_cells(thick_disk):
    """dT/T above dtmax selects thick cells whatever their count; a thin
    cell that saw at most one packet is selected too"""
    m, tb = thick_disk
    nc = m.nt - 1
    T, dT, Ni = _fields(m, tb, seed=3)
    Ni[:] = 1000
    thick = tb["thick"].reshape(m.nr, nc)
    ii, jj = np.nonzero(thick[3:-3, 2:] == 1)
    sel = (ii[::5] + 3) * nc + (jj[::5] + 2)
    dT[sel] = 2.0 * T[sel]
    thin = 10 * nc + 5
    assert thick.ravel()[thin] == 0
    Ni[thin] = 0
    To, Eo, _, so = O.diffuse(m, tb, Ni, dT, T, dtmax=1.0)
    Th, Eh, sh = H.diffuse(m, tb, Ni, dT, T, dtmax=1.0)
    assert list(sh[:4]) == list(so)
    assert so[0] == sel.size + 1
    assert Th[thin] != T[thin]
    assert np.max(np.abs(Th / To - 1)) < 1e-12


@pytest.mark.parametrize("nb,w", [(1, 1), (7, 2), (60, 5), (300, 17)])
def test_band_elimination_against_numpy(nb, w):
    """random stencil rows of the Diffuse shape (zero row sums, negative
    centre) with identity rows mixed in, against a dense solve"""
    rng = np.random.default_rng(nb * 31 + w)
    coef = np.zeros((nb, 5))
    coef[:, 0] = 1.0
    rhs = rng.uniform(1e8, 1e10, nb)
    A = np.eye(nb)
    for r in range(nb):
        nbrs = [(1, r - w), (2, r + w), (3, r - 1), (4, r + 1)]
        if rng.random() < 0.4 or not all(0 <= c < nb for _, c in nbrs):
            continue
        q = rng.uniform(1e-20, 1e-17, 4)
        coef[r, 1:] = q
        coef[r, 0] = -q.sum()
        rhs[r] = 0.0
        A[r] = 0.0
        A[r, r] = coef[r, 0]
        for (s, c), v in zip(nbrs, q):
            A[r, c] += v
    code, x = H.band_solve(nb, w, coef, rhs)
    assert code == 0
    ref = np.linalg.solve(A, rhs)
    assert np.max(np.abs(x - ref) / np.abs(ref)) < 1e-10
