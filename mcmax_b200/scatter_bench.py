"""The scattered-light field of the ray tracer (scatfield.cu) on the
precision disk deck, timed through the C-ABI:

    python -m mcmax_b200.scatter_bench [--nphot 1e6] [--field-packets 1000] [--fields 20] [--angle 45]

Deck: Mdust 1e-3 Msun ZONES disk, nr 200 (+ star cell) x ntheta 120, nlam
200 from 0.1 to 3000 micron, MRN 0.1-1 micron in 20 DHS bins, full Mueller
scattering.  One mixed-precision packet run (--nphot packets, random walk
factRW 10) gives the temperatures; then --fields scattered-light fields
(mcg_scatter_field: TraceMono at one wavelength and inclination) at
wavelengths spread log-uniformly over 0.3-30 micron, each with
--field-packets starlight and Monte Carlo packets, and one spectrum at the
same wavelengths with and without scattered light.  Prints one JSON line:
the host wall time per field (the call ends with a device synchronisation),
the packets per second, the packets ended by the caps, and the spectrum
times."""
import argparse
import json
import math
import time

import numpy as np

from . import api
from . import model as M


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--nphot", type=float, default=1e6)
    ap.add_argument("--field-packets", type=int, default=1000)
    ap.add_argument("--fields", type=int, default=20)
    ap.add_argument("--angle", type=float, default=45.0)
    a = ap.parse_args(argv)
    ctx = api.Context(0)
    m = M.disk_model(ctx, nrad=200, ntheta=120, nlam=200, mdust=1e-3, ngrains=20)
    ctx.set_model(m)
    ctx.mcradiation(int(a.nphot), precision="mixed", randomwalk=True, factRW=10.0, maxinteract=100000)
    T, _, _ = ctx.finalize_t()
    lams = np.geomspace(0.3, 30.0, a.fields)
    ang = math.radians(a.angle)
    n = a.field_packets
    ctx.scatter_field(T, float(lams[0]), ang, nphot=n, nphot_star=n, seed=1)  # first-call set-up
    times, caps = [], [0, 0, 0]
    for k, lam in enumerate(lams):
        t0 = time.perf_counter()
        _, info = ctx.scatter_field(T, float(lam), ang, nphot=n, nphot_star=n, seed=2 + k)
        times.append(time.perf_counter() - t0)
        caps[0] += info["geometry_failures"]
        caps[1] += info["interaction_cap"]
        caps[2] += info["no_start"]
    t0 = time.perf_counter()
    f0, _ = ctx.trace_spectrum(T, lams, ang)
    t_plain = time.perf_counter() - t0
    t0 = time.perf_counter()
    f1, _ = ctx.trace_spectrum(T, lams, ang, scatter=dict(nphot=n, nphot_star=n, seed=99, nexits=5))
    t_scat = time.perf_counter() - t0
    out = {"deck": "precision disk, nr 200 x ntheta 120, nlam 200, 20 grains, full Mueller",
           "fields": int(a.fields), "packets_per_field": 2 * n, "angle_deg": a.angle,
           "field_s_median": float(np.median(times)), "field_s_max": float(np.max(times)),
           "packets_per_s": float(2 * n / np.median(times)),
           "geometry_failures": caps[0], "interaction_cap": caps[1], "no_start": caps[2],
           "spectrum_s": t_plain, "spectrum_scattered_s": t_scat,
           "scattered_share_median": float(np.median(1.0 - f0 / f1))}
    print(json.dumps(out))
    ctx.close()
    return out


if __name__ == "__main__":
    main()
