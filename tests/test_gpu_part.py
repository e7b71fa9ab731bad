"""GPU ComputePart (DHS/Mie kernels through the C-ABI) against the oracle and
the golden fixtures: bit-exact FP64 opacity tables."""
import os

import numpy as np
import pytest

import oracle_ffi as O
from golden.make_golden import PART_CASES, part_inputs

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden.npz"))


@pytest.mark.parametrize("case", PART_CASES, ids=[c[0] for c in PART_CASES])
def test_compute_part_bit_exact_golden(ctx, case):
    p = part_inputs(case)
    r = ctx.compute_part_batch([p])[0]
    for k in ("kabs", "ksca", "kext", "F"):
        assert np.array_equal(r[k], GOLD["part_%s_%s" % (case[0], k)]), k
    assert [r["n_dhs"], r["n_dhs_fail"]] == list(GOLD["part_%s_counts" % case[0]])


def test_batch_equals_single_calls(ctx):
    ps = [part_inputs(c) for c in PART_CASES]
    batch = ctx.compute_part_batch(ps)
    for p, b in zip(ps, batch):
        s = ctx.compute_part_batch([p])[0]
        for k in ("kabs", "ksca", "kext", "F"):
            assert np.array_equal(s[k], b[k])


def test_random_parts_bit_exact(ctx):
    rng = np.random.default_rng(21)
    from mcmax_b200 import model as M
    for t in range(4):
        nlam = int(rng.integers(8, 20))
        lam, _ = M.wavelength_grid(0.1, float(10 ** rng.uniform(1, 3.5)), nlam)
        n, k = M.synthetic_lnk(lam, float(10 ** rng.uniform(-2.5, -0.5)))
        amin = float(10 ** rng.uniform(-2, 0.5))
        amax = amin * float(10 ** rng.uniform(0.1, 1.5))
        fmax = float(rng.choice([0.0, 0.3, 0.8]))
        blend = bool(rng.integers(0, 2))
        por = float(rng.uniform(0, 0.6)) if blend else 0.0
        ns, nf = int(rng.integers(1, 4)), int(rng.integers(1, 6))
        r = ctx.compute_part_batch([dict(lam=lam, e1=[n], e2=[k], frac=[1.0], rho=[3.0], amin=amin, amax=amax,
                                         apow=3.5, fmax=fmax, porosity=por, blend=blend, ns=ns, nf=nf)])[0]
        o = O.compute_part(lam, n, k, [1.0], [3.0], amin, amax, 3.5, fmax, blend, por, ns, nf)
        for key in ("kabs", "ksca", "kext", "F"):
            assert np.array_equal(o[key], r[key]), (t, key)
        assert o["rho_av"] == r["rho_av"]


def test_invalid_part_reports_error(ctx):
    from mcmax_b200.api import McgError
    lam = np.array([1.0, 2.0, 3.0])
    with pytest.raises(McgError):
        ctx.compute_part_batch([dict(lam=lam, e1=[lam], e2=[lam], frac=[1.0], rho=[0.0], amin=0.1, amax=1.0,
                                     apow=3.5, fmax=0.5, ns=1, nf=2)])
    with pytest.raises(McgError):
        ctx.compute_part_batch([dict(lam=lam, e1=[lam], e2=[lam], frac=[1.0], rho=[3.0], amin=-1.0, amax=1.0,
                                     apow=3.5, fmax=0.5, ns=1, nf=2)])
