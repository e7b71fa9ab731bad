"""Throughput of the opacity-surrogate network on the tensor cores.

    python -m mcmax_b200.mlp_bench [--rows 2097152] [--batch 8192] [--iters 20]

Forward: rows per second and BF16 TFLOP/s of the four 256-wide products
(2 * (3 * 256 * 256 + 256 * 64) flop per row; the 6 -> 256 input layer runs
on CUDA cores and is not counted).  Training: one Adam step (forward,
backward, update) on `batch` rows, 3x the forward products.  Both against
the measured dense BF16 peak when MEASURED_PEAKS.json is present."""
import argparse
import ctypes as C
import json
import os

from . import api
from . import surrogate as S

TC_FLOP_PER_ROW = 2 * (3 * 256 * 256 + 256 * 64)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rows", type=int, default=1 << 21)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--iters", type=int, default=20)
    a = ap.parse_args()
    ctx = api.Context(0)
    here = os.path.dirname(os.path.abspath(__file__))
    params, _ = S.load(os.path.join(here, "data", "surrogate_nf20.npz"))
    ctx.mlp_set_params(params)
    f = C.c_float(0.0)
    s = C.c_float(0.0)
    ctx._check(ctx.lib.mcg_mlp_time(ctx.h, a.rows, a.iters, a.batch, C.byref(f), C.byref(s)))
    peak = None
    try:
        with open(os.path.join(os.path.dirname(here), "MEASURED_PEAKS.json")) as fh:
            peak = json.load(fh).get("bf16_tflops")
    except OSError:
        pass
    fwd_tflops = TC_FLOP_PER_ROW * a.rows / (f.value * 1e-3) / 1e12
    step_tflops = 3 * TC_FLOP_PER_ROW * a.batch / (s.value * 1e-3) / 1e12
    out = {"rows": a.rows, "forward_ms": f.value, "forward_rows_per_s": a.rows / (f.value * 1e-3),
           "forward_tc_tflops": fwd_tflops, "batch": a.batch, "train_step_ms": s.value,
           "train_tc_tflops": step_tflops, "bf16_peak_tflops": peak,
           "forward_frac_of_peak": fwd_tflops / peak if peak else None}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
