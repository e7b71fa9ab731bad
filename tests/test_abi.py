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
    assert lib.mcg_diffuse(None, 25, 1.0, 10.0, None, None, None, None, None) == _ffi.MCG_ERR_ARG
    assert lib.mcg_disk_structure(None, None, None, None, None, None, None, None) == _ffi.MCG_ERR_ARG
    assert lib.mcg_trace_spectrum(None, None, None, 0, None, None, None) == _ffi.MCG_ERR_ARG
    assert lib.mcg_trace_image(None, None, None, 1.0, None, None, None, None) == _ffi.MCG_ERR_ARG
    assert lib.mcg_version() >= 100


PAIRS = [("mcg_part_in", "PartIn"), ("mcg_part_out", "PartOut"), ("mcg_grid", "Grid"), ("mcg_opacity", "Opacity"),
         ("mcg_run", "Run"), ("mcg_result", "Result"), ("mcg_batch_opts", "BatchOpts"), ("mcg_zone", "Zone"),
         ("mcg_structure", "Structure"), ("mcg_trace_opts", "TraceOpts"), ("mcg_image_opts", "ImageOpts"),
         ("mcg_mlp_train_opts", "MlpTrainOpts"), ("mcg_mlp_train_report", "MlpTrainReport")]


def test_struct_layouts_match_the_header(tmp_path):
    """every struct of the header: size and field offsets as the C compiler
    lays it out, against the ctypes mirror"""
    import subprocess
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "mcmax_gpu.h"', "int main(void) {"]
    for cname, pname in PAIRS:
        st = getattr(_ffi, pname)
        lines.append('printf("%s %%zu\\n", sizeof(%s));' % (cname, cname))
        for f in st._fields_:
            lines.append('printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (cname, f[0], cname, f[0]))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include", str(src), "-o",
                    str(exe)], check=True)
    got = dict(ln.split() for ln in subprocess.run([str(exe)], capture_output=True, text=True,
                                                   check=True).stdout.splitlines())
    for cname, pname in PAIRS:
        st = getattr(_ffi, pname)
        assert int(got[cname]) == C.sizeof(st), cname
        for f in st._fields_:
            assert int(got["%s.%s" % (cname, f[0])]) == getattr(st, f[0]).offset, (cname, f[0])
