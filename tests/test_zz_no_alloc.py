"""mcg_compute_part_static: ComputePart with all device working memory in
the library's static array, for host programs that must not call cudaMalloc
(a driver whose device memory is already owned by its own pool allocator, or
code that cannot afford cudaFree's device-wide wait).

Called through the C-ABI with ctypes, it must give the same opacity tables,
bit for bit, as mcg_compute_part on the same bin, on consecutive calls that
reuse the array: first a bin that fits in one pass, then one that is split
into several wavelength chunks.  Repeated calls must leave the device's free
memory where it was.  A bin whose single wavelength needs more than the
array holds is refused before anything runs on the GPU.

The file name sorts last so that a run stopping at the first failure has run
every other test first."""
import ctypes as C

import numpy as np
import pytest

from golden.make_golden import PART_CASES, part_inputs
from mcmax_b200 import _ffi
from mcmax_b200 import model as M

pytestmark = pytest.mark.gpu
NA = _ffi.NANG


def _call(lib, h, fn, p):
    lam = np.ascontiguousarray(p["lam"], dtype=np.float64)
    e1 = np.ascontiguousarray(np.atleast_2d(p["e1"]), dtype=np.float64)
    e2 = np.ascontiguousarray(np.atleast_2d(p["e2"]), dtype=np.float64)
    frac = np.ascontiguousarray(np.atleast_1d(p["frac"]), dtype=np.float64)
    rho = np.ascontiguousarray(np.atleast_1d(p["rho"]), dtype=np.float64)
    nlam = lam.size
    pin = _ffi.PartIn(nlam, _ffi.ptr(lam), e1.shape[0], _ffi.ptr(e1), _ffi.ptr(e2), _ffi.ptr(frac), _ffi.ptr(rho),
                      float(p["amin"]), float(p["amax"]), float(p["apow"]), float(p["fmax"]),
                      float(p.get("porosity", 0.0)), float(p.get("normalize_abun", -1.0)),
                      int(bool(p.get("blend", False))), int(p["ns"]), int(p["nf"]))
    o = dict(kabs=np.zeros(nlam), ksca=np.zeros(nlam), kext=np.zeros(nlam), F=np.zeros((nlam, 6, NA)))
    pout = _ffi.PartOut()
    for k in ("kabs", "ksca", "kext", "F"):
        setattr(pout, k, _ffi.ptr(o[k]))
    st = getattr(lib, fn)(h, C.byref(pin), C.byref(pout))
    o.update(status=st, rho_av=pout.rho_av, mscale=pout.mscale, rscale=pout.rscale,
             counts=(pout.n_dhs, pout.n_mie, pout.n_dhs_fail))
    return o


def _chunked_bin():
    # 60 wavelengths x 10 sizes x 20 filling fractions: 200 coated-sphere
    # samples per wavelength, ~1.2 MB of working memory per wavelength, so
    # the 64 MiB array takes the bin in several wavelength chunks
    lam, _ = M.wavelength_grid(0.1, 1000.0, 60)
    n, k = M.synthetic_lnk(lam, 0.03)
    return dict(lam=lam, e1=[n], e2=[k], frac=[1.0], rho=[3.0], amin=0.1, amax=2.0, apow=3.5, fmax=0.8,
                porosity=0.25, blend=True, ns=10, nf=20)


@pytest.fixture(scope="module")
def handle():
    lib = _ffi.load()
    h = C.c_void_p()
    assert lib.mcg_create(C.byref(h), 0) == _ffi.MCG_OK
    yield lib, h
    lib.mcg_destroy(h)


def test_static_matches_allocating_entry_point_on_consecutive_calls(handle):
    lib, h = handle
    bins = [part_inputs(PART_CASES[0]), _chunked_bin()]
    for p in bins:
        ref = _call(lib, h, "mcg_compute_part", p)
        assert ref["status"] == _ffi.MCG_OK, lib.mcg_last_error(h)
        got = _call(lib, h, "mcg_compute_part_static", p)
        assert got["status"] == _ffi.MCG_OK, lib.mcg_last_error(h)
        for key in ("kabs", "ksca", "kext", "F"):
            assert np.array_equal(ref[key], got[key]), key
        for key in ("rho_av", "mscale", "rscale", "counts"):
            assert ref[key] == got[key], key
    # the same bin again: the array still holds the previous call's data
    again = _call(lib, h, "mcg_compute_part_static", bins[0])
    ref0 = _call(lib, h, "mcg_compute_part", bins[0])
    for key in ("kabs", "ksca", "kext", "F"):
        assert np.array_equal(ref0[key], again[key]), key


def _device_free_bytes():
    """Free device memory of the current context (cuMemGetInfo of the
    driver API; the library's calls made its device's primary context
    current on this thread)."""
    drv = C.CDLL("libcuda.so.1")
    free, total = C.c_size_t(), C.c_size_t()
    assert drv.cuMemGetInfo_v2(C.byref(free), C.byref(total)) == 0
    return free.value


def test_static_calls_leave_device_memory_unchanged(handle):
    # the premise of the entry point: no device allocation.  A first pass
    # over both bins loads the kernels and looks up the array's address;
    # after it, the device's free memory must be the same before and after
    # further calls (an allocation that is still held, or a cached buffer,
    # would lower it)
    lib, h = handle
    bins = [part_inputs(PART_CASES[0]), _chunked_bin()]
    for p in bins:
        assert _call(lib, h, "mcg_compute_part_static", p)["status"] == _ffi.MCG_OK, lib.mcg_last_error(h)
    before = _device_free_bytes()
    for p in bins + bins:
        assert _call(lib, h, "mcg_compute_part_static", p)["status"] == _ffi.MCG_OK, lib.mcg_last_error(h)
    assert _device_free_bytes() == before


def test_static_refuses_a_bin_beyond_the_array(handle):
    lib, h = handle
    p = _chunked_bin()
    p.update(ns=1000, nf=20)  # 20000 samples at one wavelength: ~116 MB
    got = _call(lib, h, "mcg_compute_part_static", p)
    assert got["status"] == _ffi.MCG_ERR_LIMIT
    assert b"static array" in lib.mcg_last_error(h)
