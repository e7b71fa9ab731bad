"""Packets/s of the MCMax photon-packet loop on B200.

Workload (the "precision" disk deck): star Teff = 10000 K, R* = 2.5 Rsun;
ZONES disk Rin = 0.5 AU, Rout = 100 AU, Sigma ~ r^-1, Mdust = 1e-3 Msun,
H/R = 0.05 at 1 AU (MCMax scale height sh = 0.05*sqrt(2)), flaring 1.125;
grid nr = 200 x ntheta = 120 (+ the star cell), nlam = 200 from 0.1 to 3000
micron; one synthetic .lnk composition, MRN 0.1-1 micron in 20 bins (5 sizes,
20 DHS filling fractions each, fmax = 0.8, blend with porosity 0.25), full
Mueller scattering, Bjorkman-Wood re-emission, modified random walk
(factRW = 10).  Opacities come from the library's own DHS kernels.

One step = one MCRadiation call over the deck's 1e8 packets (`--nphot`), with
the reference's overflow roulette switched on at maxinteract = 1e5 (keyword
'maxinteract', MCRadiation.f:568-571: an energy-compensated kill with
probability 1/maxinteract per interaction).  Without it a few packets
trapped in the optically thick midplane take 1e8+ events each (the CPU
reference pays the same events serially; on the GPU they become the critical
path of the launch).  `value` is the device time of the transport kernel with
all tables resident in HBM; `e2e` times the reference-facing C-ABI
(mcg_set_model from host buffers + mcg_mcradiation + result copies to host).

The same line carries `learned_deck`: the learned-opacities deck (three
compositions in 50 bins from 0.01 to 1000 micron, vertically settled) in its
plain form (FP64 transport on DHS opacities) and in its fast form (mixed
transport on the opacity surrogate's tables), with opacity-stage time,
packets/s, end-to-end time per step and the agreement of per-cell
temperatures and SEDs with the plain form on identical Philox streams.

--impl reference runs the oracle (the CPU restatement of the reference's
loop; the Fortran reference cannot be compiled without a Fortran compiler) on
all host cores.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NPHOT_DEFAULT = 100_000_000
WORKLOAD = dict(mdust=1e-3, nrad=200, ntheta=120, nlam=200, lam1=0.1, lam2=3000.0, ngrains=20, ns=5, nf=20,
                fmax=0.8, blend=True, porosity=0.25, scat_how=2)
RUN = dict(randomwalk=True, factRW=10.0, maxinteract=100_000)
METRIC = "packets/s (MCRadiation packet loop, 1 B200)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nphot", type=int, default=NPHOT_DEFAULT)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed", "exact"])
    ap.add_argument("--compare-fp64", action="store_true", help="also time the FP64 form (one step)")
    ap.add_argument("--cpu-sample-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-post-mc", action="store_true",
                    help="skip the timing of the steps after the packet loop (Diffuse, structure, spectrum, image)")
    ap.add_argument("--learned-nphot", type=int, default=30_000_000,
                    help="packets per run of the learned-opacities comparison (0 skips it)")
    ap.add_argument("--maxinteract", type=int, default=RUN["maxinteract"],
                    help="overflow roulette (keyword maxinteract); smaller values shorten the trapped-packet tail "
                         "for profiling runs")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        load = [s for s in sm if smax and s > 0.5 * smax] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def algorithmic_bytes(counters, nlam):
    """Per-event byte model of the packet loop (the reads and read-modify-
    writes an event needs at minimum): crossing 72 B + 16 B EJv2 on exit,
    absorption 64 B + nlam*24 B re-emission row, scattering 2*180*8 + 48 B,
    random-walk step 56 B, escape 16 B."""
    cross, absorb, scat, rw, esc = (int(counters[k]) for k in (8, 2, 3, 4, 9))
    return cross * (72 + 16) + absorb * (64 + 24 * nlam) + scat * (2 * 180 * 8 + 48) + rw * 56 + esc * 16


def cpu_baseline_sample(model, seconds, cores):
    """Time the CPU restatement (oracle) on a bounded sample of the same
    workload: serial, packets until ~`seconds` of work."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_ffi as O
    tab = O.transport_tables(model, randomwalk=RUN["randomwalk"], factRW=RUN["factRW"], lazy_kd=True)
    n = 20
    total_n, total_t = 0, 0.0
    while total_t < seconds and total_n < 200000:
        t0 = time.perf_counter()
        O.mcradiation(model, n, seed=1000 + total_n, randomwalk=RUN["randomwalk"], factRW=RUN["factRW"],
                      maxinteract=RUN["maxinteract"], tables=tab)
        dt = time.perf_counter() - t0
        total_n += n
        total_t += dt
        n = min(4 * n, max(20, int(n * (seconds - total_t) / max(dt, 1e-3))))
        if n <= 0:
            break
    return total_n / total_t, total_n, total_t


def learned_deck_comparison(ctx, nphot, seed0):
    """The learned-opacities deck (three compositions in 50 bins from 0.01 to
    1000 micron, settled with alpha = 1e-3, nr 200 x ntheta 120, nlam 200)
    in its two forms: plain FP64 transport on DHS opacities and mixed
    transport on surrogate opacities.  Both runs use the same Philox seed;
    a second FP64 run with another seed gives the Monte Carlo noise floor
    of the agreement figures.  Per step: opacity stage (ComputePart of the
    150 bins), mcg_set_model from host arrays, the packet loop, results to
    the host."""
    import numpy as np
    from mcmax_b200 import model as M
    from mcmax_b200 import surrogate as S
    params, sinfo = S.load(os.path.join(ROOT, "mcmax_b200", "data", "surrogate_nf20.npz"))
    out = {"workload": "learned-opacities deck: 3 compositions x 50 bins 0.01-1000 micron (ns 5, nf 20), "
                       "settling alpha 1e-3, Mdust 1e-3 Msun, nr 200 x ntheta 120, nlam 200, random walk, "
                       "maxinteract %g, %d packets per run" % (RUN["maxinteract"], nphot)}
    runs = {}
    for tag, opac, prec, seed in (("fp64_dhs", "dhs", "fp64", seed0), ("mixed_surrogate", "surrogate", "mixed", seed0),
                                  ("fp64_dhs_seed2", "dhs", "fp64", seed0 + 1)):
        t0 = time.perf_counter()
        m, t_opac, served = M.learned_disk_model(ctx, opacity=opac, params=params if opac == "surrogate" else None)
        ctx.set_model(m)
        t_setup = time.perf_counter() - t0
        t1 = time.perf_counter()
        _, o = ctx.mcradiation(nphot, seed=seed, precision=prec, fetch=True, **RUN)
        T, _, _ = ctx.finalize_t()
        t_run = time.perf_counter() - t1
        runs[tag] = dict(T=T, spec=o["spec"], Ni=o["Ni"])
        out[tag] = {"opacity_stage_s": t_opac, "setup_s": t_setup, "transport_device_ms": o["device_ms"],
                    "packets_per_s": nphot / (o["device_ms"] / 1e3), "run_s": t_run,
                    "e2e_step_s": t_setup + t_run, "bins_served_by_network": served,
                    "progress_ms": o["progress_ms"]}
    ref = runs["fp64_dhs"]
    sel = (ref["Ni"] >= 1000) & (ref["T"] > 0)
    for tag in ("mixed_surrogate", "fp64_dhs_seed2"):
        r = runs[tag]
        rel = np.abs(r["T"][sel] / ref["T"][sel] - 1)
        sr, sp = ref["spec"][:, 1:].sum(1), r["spec"][:, 1:].sum(1)
        ok = sr > 0
        sed = np.abs(sp[ok] / sr[ok] - 1)
        out[tag]["agreement_with_fp64_dhs"] = {
            "cells_Ni_ge_1e3": int(sel.sum()), "T_within_1pct": float(np.mean(rel < 0.01)),
            "T_median_rel": float(np.median(rel)), "T_p95_rel": float(np.percentile(rel, 95)),
            "sed_median_rel": float(np.median(sed))}
    out["speedup_e2e_step"] = out["fp64_dhs"]["e2e_step_s"] / out["mixed_surrogate"]["e2e_step_s"]
    out["speedup_transport"] = out["mixed_surrogate"]["packets_per_s"] / out["fp64_dhs"]["packets_per_s"]
    out["surrogate"] = {"train_samples": int(sinfo["n"]), "epochs": int(sinfo["epochs"]),
                        "bins_median_dex_kabs": float(sinfo["bins_median_dex_kabs"]),
                        "bins_median_dex_ksca": float(sinfo["bins_median_dex_ksca"])}
    return out


def post_mc_steps(ctx, model, res):
    """The steps after the packet loop on the same deck and the packet
    run's result, each C-ABI call timed on the host (every call ends with a
    device synchronisation): the temperatures (mcg_finalize_t), Diffuse
    (mcg_diffuse), one vertical-structure pass on the zone taken as not
    fixed (mcg_disk_structure), the ray-traced spectrum at 45 degrees on the
    grid's wavelengths (mcg_trace_spectrum) and a 500 x 500 image with 1000
    points per image cell at the middle of the wavelength range
    (mcg_trace_image).  Not part of the headline metric."""
    import math
    import numpy as np
    from mcmax_b200 import model as M
    from mcmax_b200 import outputs
    from mcmax_b200 import structure as S

    def timed(fn):
        t0 = time.perf_counter()
        r = fn()
        return r, time.perf_counter() - t0

    out = {}
    (T, dT, _), t = timed(ctx.finalize_t)
    out["finalize_t_s"] = t
    (Td, _, counts), t = timed(lambda: ctx.diffuse(res["Ni"], dT, T))
    out["diffuse"] = {"s": t, "selected_cells": int(counts[0]), "unknowns": int(counts[1])}
    st = S.initial_state(model)
    zones = [(0.5, 100.0, 0.05 * math.sqrt(2.0), 1.0, 1.125, 1.0, 0)]
    _, t = timed(lambda: ctx.disk_structure(model.R, model.Theta, model.V, 2.5 * M.MSUN, zones, np.maximum(Td, 2.7),
                                            st["dens"], st["dens0"], st["gasdens"], st["w"], st["w0"]))
    out["disk_structure"] = {"s": t, "columns": int((model.nr - 1) * (model.ncomp + 1))}
    lam_obs = outputs.spectrum_wavelengths(model.lam, model.lam[0], model.lam[-1])
    (flux, info), t = timed(lambda: ctx.trace_spectrum(Td, lam_obs, math.radians(45.0)))
    out["trace_spectrum"] = {"s": t, "wavelengths": int(lam_obs.size), "image_radii": info[0],
                             "rays_per_s": info[0] * 45 * lam_obs.size / t, "bad_rays": info[1]}
    lam0 = (model.lam[0] + model.lam[-1]) / 2.0
    img, t = timed(lambda: ctx.trace_image(Td, lam0, math.radians(45.0), npixel=500, nint=1000))
    pts = (img["info"][0] - 1) * 45 * 1000
    out["trace_image"] = {"s": t, "points": int(pts), "points_per_s": pts / t,
                          "sum_over_flux": float(img["image"].sum() / img["flux"])}
    return out


def build_model(ctx):
    from mcmax_b200 import model as M
    return M.disk_model(ctx, **WORKLOAD)


def run_reference(args, rank, world):
    """CPU restatement on all host cores: independent packet batches per
    process (multiprocessing, spawn), reported like our arm."""
    import multiprocessing as mp
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    model = _cpu_model()
    per = max(1, int(os.environ.get("MCMAX_REF_PACKETS", "200")))
    ctxmp = mp.get_context("spawn")
    step_times = []
    with ctxmp.Pool(cores, initializer=_ref_init) as pool:
        for it in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            pool.map(_ref_work, [(s + 1000 * it, per) for s in range(cores)])
            dt = time.perf_counter() - t0
            if it >= args.warmup:
                step_times.append(dt)
    total = per * cores
    value = total / statistics.mean(step_times)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "packets/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(step_times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "precision disk deck (CPU restatement of the reference loop, packets per step %d)" % total,
                       "nr": 200, "ntheta": 120, "nlam": 200, "packets_per_step": total},
            "cpu_baseline": {"value": value, "unit": "packets/s", "cores": cores, "kind": "port",
                             "sample": "%d packets per step on %d processes" % (total, cores)},
            "e2e": {"value": value, "unit": "packets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


_REF = {}


def _cpu_model():
    """The same deck with opacities from the oracle's ComputePart."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import models
    return models.small_disk(nrad=WORKLOAD["nrad"], ntheta=WORKLOAD["ntheta"], nlam=WORKLOAD["nlam"],
                             ngrains=WORKLOAD["ngrains"], ns=WORKLOAD["ns"], nf=WORKLOAD["nf"],
                             mdust=WORKLOAD["mdust"], scat_how=2)


def _ref_init():
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_ffi as O
    m = _cpu_model()
    _REF["m"] = m
    _REF["tab"] = O.transport_tables(m, randomwalk=True, factRW=RUN["factRW"], lazy_kd=True)


def _ref_work(a):
    import oracle_ffi as O
    seed, n = a
    O.mcradiation(_REF["m"], n, seed=seed, randomwalk=True, factRW=RUN["factRW"], maxinteract=RUN["maxinteract"],
                  tables=_REF["tab"])
    return n


def main():
    args = parse()
    RUN["maxinteract"] = args.maxinteract
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    if args.impl == "reference":
        run_reference(args, rank, world)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    import numpy as np
    from mcmax_b200 import api

    ctx = api.Context(local)
    model = build_model(ctx)
    ctx.set_model(model)
    # warm-up steps (also builds the random-walk tables once)
    for w in range(args.warmup):
        ctx.mcradiation(args.nphot, seed=10_000 * (rank + 1) + w, precision=args.precision, fetch=False, **RUN)
    sync = _barrier(dist)
    clocks = ClockSampler(local)
    clocks.start()
    dev_ms = []
    counters = np.zeros(16, np.int64)
    t0 = time.perf_counter()
    for s in range(args.steps):
        _, out = ctx.mcradiation(args.nphot, seed=rank * 1_000_003 + s + 1, precision=args.precision, fetch=False,
                                 **RUN)
        dev_ms.append(out["device_ms"])
        counters += out["counters"]
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    t_dev = sum(dev_ms) / 1e3
    t_max = _max_over_ranks(dist, t_dev)
    packets = args.nphot * args.steps * world
    value = packets / t_max
    # end to end through the C-ABI with host buffers
    import ctypes
    h2d = sum(np.asarray(getattr(model, k)).nbytes for k in ("R", "Theta", "SinTheta", "dens", "V", "comp_w", "lam",
                                                               "nu", "Kabs", "Ksca", "F", "BB", "Fstar"))
    nc = model.ncell
    d2h = nc * (8 * 4 + 4) + model.nlam * 31 * (8 * 2 + 4)
    e2e_steps = 1
    _barrier(dist)
    t1 = time.perf_counter()
    for s in range(e2e_steps):
        ctx.set_model(model)
        _, e2e_res = ctx.mcradiation(args.nphot, seed=rank * 7_000_001 + s + 1, precision=args.precision,
                                     fetch=True, **RUN)
    e2e_t = _max_over_ranks(dist, time.perf_counter() - t1)
    post_mc = None
    if rank == 0 and world == 1 and not args.no_post_mc:
        try:
            post_mc = post_mc_steps(ctx, model, e2e_res)
        except Exception as e:  # the extra timings must not sink the GPU line
            post_mc = {"failed": str(e)}
    e2e_value = args.nphot * e2e_steps * world / e2e_t
    fp64_line = None
    if args.compare_fp64 and args.precision != "fp64":
        _, o64 = ctx.mcradiation(args.nphot, seed=rank * 5_000_011 + 1, precision="fp64", fetch=False, **RUN)
        t64 = _max_over_ranks(dist, o64["device_ms"] / 1e3)
        fp64_line = {"value": args.nphot * world / t64, "unit": "packets/s", "steps": 1,
                     "ms_per_step": 1e3 * t64}
    learned = None
    if rank == 0 and world == 1 and args.learned_nphot > 0:
        learned = learned_deck_comparison(ctx, args.learned_nphot, 7_000_003)
    # roofline of the transport kernel against the measured HBM copy bandwidth
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    algo = algorithmic_bytes(counters, model.nlam) / args.steps
    per_launch_s = t_dev / args.steps
    achieved = algo / per_launch_s / 1e9
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cm = _cpu_model()
            v, n, t = cpu_baseline_sample(cm, args.cpu_sample_seconds, 1)
            cpu = {"value": v, "unit": "packets/s", "cores": 1, "kind": "port",
                   "sample": "%d packets of the same deck, serial CPU restatement, %.1f s" % (n, t)}
        except Exception as e:  # the baseline must not sink the GPU line
            cpu = {"value": None, "unit": "packets/s", "cores": 1, "kind": "port", "sample": "failed: %s" % e}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "packets/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic",
            "config": {"workload": "precision disk deck: Mdust 1e-3 Msun, nr 200 x ntheta 120, nlam 200, "
                                   "random walk (factRW 10), full Mueller scattering, maxinteract %g, %s transport"
                                   % (args.maxinteract, args.precision),
                       "packets_per_step": args.nphot, "precision": args.precision,
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": "model tables exceed L2 (126 MB): per-cell opacity rows, emission CDF, "
                             "random-walk tables"},
            "e2e": {"value": e2e_value, "unit": "packets/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": 2 * int(args.steps),  # transport kernel + per-run combine kernel per step
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "note": "algorithmic bytes from the event counters (crossings, absorptions, scatterings, "
                                 "random-walk steps) per launch / transport-kernel time; peak = measured HBM copy"},
            "progress_ms_last_step": out["progress_ms"],
            "events_per_step": {"crossings": int(counters[8] // args.steps), "absorptions": int(counters[2] // args.steps),
                                "scatterings": int(counters[3] // args.steps), "rw_steps": int(counters[4] // args.steps)},
            "wall_s": wall, "clocks": clk, "cpu_baseline": cpu,
        }
        if fp64_line:
            line["fp64_form"] = fp64_line
        if learned:
            line["learned_deck"] = learned
        if post_mc:
            line["post_mc"] = post_mc
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def _barrier(dist):
    if dist:
        import torch
        if dist.get_backend() == "nccl":
            torch.cuda.synchronize()
        dist.barrier()
    return True


def _max_over_ranks(dist, v):
    """the largest value over the ranks (timings: the slowest rank)"""
    if not dist:
        return v
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


if __name__ == "__main__":
    main()
