"""The C-ABI library: loads without a GPU, exports every symbol the header
declares, its host-side table builder matches the oracle, and it reports
errors instead of aborting."""
import ctypes as C
import os
import re

import numpy as np

import oracle_ffi as O
from mcmax_b200 import _ffi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names += re.findall(r"^\s*(?:[\w\s\*]+?)\b(mcg_\w+)\s*\(", txt, re.M)
    return sorted(set(names))


def test_every_declared_symbol_is_exported():
    lib = _ffi.load()
    names = _declared()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) <= set(_ffi.SIGNATURES), set(names) - set(_ffi.SIGNATURES)


def test_planck_table_matches_oracle():
    from mcmax_b200 import api
    lam = np.geomspace(0.1, 3000, 37)
    assert np.array_equal(api.bb_table(lam), O.bb_table(lam))


def test_invalid_arguments_do_not_abort():
    lib = _ffi.load()
    assert lib.mcg_create(None, 0) == _ffi.MCG_ERR_ARG
    h = C.c_void_p()
    st = lib.mcg_create(C.byref(h), 10_000)
    assert st in (_ffi.MCG_ERR_ARG, _ffi.MCG_ERR_CUDA)
    assert lib.mcg_bb_table(0, None, None) == _ffi.MCG_ERR_ARG
    assert lib.mcg_set_model(None, None, None) == _ffi.MCG_ERR_ARG
    assert lib.mcg_mcradiation(None, None, None, None) == _ffi.MCG_ERR_ARG
    assert lib.mcg_version() >= 100
