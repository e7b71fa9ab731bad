"""Generate the golden fixtures used by the parity tests.

The reference (Fortran MCMax) cannot be compiled or imported here and ships no
test outputs, so the fixtures are outputs of the CPU restatement (oracle/)
for small, fixed inputs, plus the published homogeneous-sphere Mie values of
Bohren & Huffman (1983, appendix A test case: m = 1.55, r = 0.525 micron,
lambda = 0.6328 micron -> Qsca = Qext = 3.10543, Qback = 2.92534).
Run:  python tests/golden/make_golden.py
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle_ffi as O  # noqa: E402
from mcmax_b200 import model as M  # noqa: E402

PART_CASES = [
    # (name, nlam, lam2, kpref, amin, amax, apow, fmax, blend, porosity, ns, nf, nmat)
    ("dhs_blend", 24, 3000.0, 0.03, 0.1, 1.0, 3.5, 0.8, True, 0.25, 3, 5, 1),
    ("dhs_two_materials", 16, 1000.0, 0.3, 0.05, 2.0, 3.5, 0.6, False, 0.0, 2, 4, 2),
    ("mie_only_fmax0", 16, 1000.0, 0.03, 0.1, 5.0, 3.0, 0.0, False, 0.0, 3, 1, 1),
    ("large_grains", 12, 100.0, 0.03, 200.0, 1000.0, 3.5, 0.5, True, 0.3, 2, 3, 1),
]


def part_inputs(case):
    name, nlam, lam2, kpref, amin, amax, apow, fmax, blend, por, ns, nf, nmat = case
    lam, _ = M.wavelength_grid(0.1, lam2, nlam)
    e1, e2 = [], []
    for k in range(nmat):
        n_, k_ = M.synthetic_lnk(lam, kpref * (10.0 ** k))
        e1.append(n_ + 0.2 * k)
        e2.append(k_)
    frac = [1.0 + k for k in range(nmat)]
    rho = [3.0 - 0.5 * k for k in range(nmat)]
    return dict(lam=lam, e1=np.array(e1), e2=np.array(e2), frac=np.array(frac), rho=np.array(rho), amin=amin,
                amax=amax, apow=apow, fmax=fmax, blend=blend, porosity=por, ns=ns, nf=nf)


def main():
    out = {}
    # published Mie known answer
    e, cs, ce, f = O.mie(0.525, 0.6328, 1.55, 0.0)
    out["bh_mie_qsca_qext"] = np.array([cs / (math.pi * 0.525 ** 2), ce / (math.pi * 0.525 ** 2)])
    for case in PART_CASES:
        p = part_inputs(case)
        r = O.compute_part(p["lam"], p["e1"], p["e2"], p["frac"], p["rho"], p["amin"], p["amax"], p["apow"],
                           p["fmax"], p["blend"], p["porosity"], p["ns"], p["nf"])
        for k in ("kabs", "ksca", "kext", "F"):
            out["part_%s_%s" % (case[0], k)] = r[k]
        out["part_%s_counts" % case[0]] = np.array([r["n_dhs"], r["n_dhs_fail"]])
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
