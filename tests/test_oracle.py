"""The CPU oracle (oracle/) against published values, limits and
identities of the reference's algorithms, and against the golden fixtures."""
import math
import os

import numpy as np
import pytest

import oracle_ffi as O
from golden.make_golden import PART_CASES, part_inputs

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden.npz"))


def test_mie_bohren_huffman_known_answer():
    # Bohren & Huffman (1983) appendix A: m = 1.55, x = 2 pi 0.525/0.6328
    e, cs, ce, f = O.mie(0.525, 0.6328, 1.55, 0.0)
    g = math.pi * 0.525 ** 2
    assert e == 0
    assert abs(cs / g - 3.10543) < 5e-6
    assert abs(ce / g - 3.10543) < 5e-6


def test_dmilay_backscatter_known_answer():
    # same case through the coated-sphere code with core = shell material:
    # QBS is |S(180)|^2/(pi x^2), so 4 pi QBS = Bohren & Huffman's Qback 2.92534
    wv = 2 * math.pi / 0.6328
    e, q, _ = O.dmilay(0.3, 0.525, wv, 1.55, 0.0, 1.55, 0.0)
    assert e == 0
    assert abs(q[0] - 3.10543) < 5e-6 and abs(q[1] - 3.10543) < 5e-6
    assert abs(4 * math.pi * q[2] - 2.92534) < 5e-5


@pytest.mark.parametrize("m_re,m_im,x", [(1.5, 0.0, 3.0), (1.7, 0.05, 12.0), (2.2, 0.4, 40.0), (1.33, 1e-3, 80.0)])
def test_coated_sphere_with_identical_core_is_homogeneous(m_re, m_im, x):
    lam = 1.0
    rad = x * lam / (2 * math.pi)
    wv = 2 * math.pi / lam
    e, q, _ = O.dmilay(0.6 * rad, rad, wv, m_re, -m_im, m_re, -m_im)
    e2, cs, ce, _ = O.mie(rad, lam, m_re, m_im)
    g = math.pi * rad * rad
    assert e == 0 and e2 == 0
    # the two series truncate differently (DMiLay: |a_n|^2 < 1e-14, Mie: term < 1e-8)
    assert abs(q[1] - cs / g) < 1e-6 * max(1.0, q[1])
    assert abs(q[0] - ce / g) < 1e-6 * max(1.0, q[0])


def test_vacuum_core_limit():
    # a vanishing vacuum core leaves the homogeneous shell (DMiLay vs Mie)
    lam, rad = 1.0, 0.8
    wv = 2 * math.pi / lam
    e, q, _ = O.dmilay(1e-4 * rad, rad, wv, 1.6, -0.02)
    e2, cs, ce, _ = O.mie(rad, lam, 1.6, 0.02)
    g = math.pi * rad * rad
    assert abs(q[1] - cs / g) / (cs / g) < 1e-6


def test_bruggeman_identities():
    # one material: the effective medium is the material itself
    a, b = O.blender([1.7], [0.1], [1.0])
    assert abs(a - 1.7) < 1e-12 and abs(b - 0.1) < 1e-12
    # zero porosity with vacuum: unchanged
    a, b = O.blender([1.7, 1.0], [0.1, 0.0], [1.0, 0.0])
    assert abs(a - 1.7) < 1e-12 and abs(b - 0.1) < 1e-12
    # symmetric in the order of the components
    a1, b1 = O.blender([1.7, 1.0], [0.1, 0.0], [0.6, 0.4])
    a2, b2 = O.blender([1.0, 1.7], [0.0, 0.1], [0.4, 0.6])
    assert abs(a1 - a2) < 1e-12 and abs(b1 - b2) < 1e-12
    # porous material is optically thinner
    assert 1.0 < a1 < 1.7 and 0.0 < b1 < 0.1


@pytest.mark.parametrize("case", PART_CASES, ids=[c[0] for c in PART_CASES])
def test_compute_part_against_golden(case):
    p = part_inputs(case)
    r = O.compute_part(p["lam"], p["e1"], p["e2"], p["frac"], p["rho"], p["amin"], p["amax"], p["apow"], p["fmax"],
                       p["blend"], p["porosity"], p["ns"], p["nf"])
    for k in ("kabs", "ksca", "kext", "F"):
        assert np.array_equal(r[k], GOLD["part_%s_%s" % (case[0], k)]), k
    # invariants of ComputePart.f:407-445
    assert np.allclose(r["kext"], r["kabs"] + r["ksca"], rtol=1e-12)
    sinw = np.sin(np.pi * (np.arange(1, 181) - 0.5) / 180)
    norm = (r["F"][:, 0, :] * sinw).sum(1) / sinw.sum()
    assert np.all(np.abs(norm - 1) < 1e-9)
    assert np.all(r["F"][:, 0, :] >= 0)
    assert np.all(np.abs(r["F"][:, 1, :]) <= r["F"][:, 0, :] * (1 + 1e-9) + 1e-12)


def test_planck_table():
    lam = np.array([0.1, 1.0, 10.0, 1000.0])
    BB = O.bb_table(lam)
    assert BB.shape == (4, O.TT) and np.all(BB[:, 0] == 0)
    # Rayleigh-Jeans limit at long wavelength: 2 k T nu^2 / c^2
    nu = 2.9979e10 / (1000.0 * 1e-4)
    rj = 2 * 1.3807e-16 * 5000 * nu ** 2 / 2.9979e10 ** 2
    x = 6.6261e-27 * nu / (1.3807e-16 * 5000)
    assert abs(BB[3, 5000] / rj - (1 - x / 2)) < 1e-5
    assert np.all(np.diff(BB[:, 1:], axis=1) >= 0)  # increasing in T


def _kp_table():
    T = np.arange(O.TT, dtype=float)
    kp = 1e-10 * np.maximum(T, 0.5) ** 4 * (1 + 1e-4 * T)
    return np.ascontiguousarray(kp)


def test_temperature_inversions_agree():
    L = O.load()
    kp = _kp_table()
    rng = np.random.default_rng(3)
    for E in kp[1] * 10 ** rng.uniform(0, 15, 300):
        if E > kp[-1]:
            continue
        Td = L.orc_determine_t(O.P(kp), E, 1.0)
        Ti = L.orc_increase_t(O.P(kp), E, 0.0)
        assert abs(Td - Ti) <= 1e-9 * Td
        i = int(Td)
        assert kp[i] <= E * (1 + 1e-12) and E <= kp[min(i + 1, O.TMAX)] * (1 + 1e-12)
    assert L.orc_determine_t(O.P(kp), kp[1] * 0.5, 5.0) == 1.0
    assert L.orc_determine_t(O.P(kp), kp[-1] * 2, 5.0) == O.TMAX - 1


def test_ran1_sequence_properties():
    import ctypes as C
    L = O.load()
    idum = C.c_int32(-42)
    iv = (C.c_int32 * 32)()
    iy = C.c_int32(0)
    xs = np.array([L.orc_ran1(C.byref(idum), iv, C.byref(iy)) for _ in range(20000)])
    assert np.all((xs > 0) & (xs < 1))
    assert abs(xs.mean() - 0.5) < 0.01 and abs(xs.var() - 1 / 12) < 0.003


def test_single_precision_t4_interpolation():
    """orc_set_t4_single: determineT and increaseT interpolate T^4 between the
    bracketing steps with the reference's single-precision real(i)**4"""
    import oracle_ffi as OF
    L = OF.load()
    iT = np.arange(0, 10001, dtype=float)
    kp = np.ascontiguousarray(1e-3 * iT ** 4 + 1e-6 * iT)
    P = OF.P
    E1 = 0.37 * kp[1234] + 0.63 * kp[1235]
    t64 = L.orc_determine_t(P(kp), E1, 100.0)
    L.orc_set_t4_single(1)
    try:
        t32 = L.orc_determine_t(P(kp), E1, 100.0)
        u32 = L.orc_increase_t(P(kp), E1, 1000.0)
    finally:
        L.orc_set_t4_single(0)
    a = np.float32(1234.0) ** 2
    a = a * a
    b = np.float32(1235.0) ** 2
    b = b * b
    expect = (float(a) + (float(np.float32(b - a)) * (E1 - kp[1234])) / (kp[1235] - kp[1234])) ** 0.25
    assert abs(t32 / expect - 1) < 1e-15 and t32 == u32
    assert t32 != t64 and abs(t32 / t64 - 1) < 1e-7
