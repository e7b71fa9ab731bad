"""Packets/s of the MCMax photon-packet loop on B200.

Headline workload -- the learned-opacities deck: star Teff = 10000 K,
R* = 2.5 Rsun; ZONES disk Rin = 0.5 AU, Rout = 100 AU, Sigma ~ r^-1,
Mdust = 1e-3 Msun, H/R = 0.05 at 1 AU (MCMax scale height sh = 0.05*sqrt(2)),
flaring 1.125, vertically settled with alpha = 1e-3 (FixedMPSettling), so
every cell has its own grain mixture; three synthetic .lnk compositions
(k prefactors 0.003 / 0.03 / 0.3) in 50 log bins each from 0.01 to 1000
micron (150 grain components); grid nr = 200 x ntheta = 120 (+ the star
cell), nlam = 200 from 0.1 to 3000 micron; full Mueller scattering,
Bjorkman-Wood re-emission, modified random walk (factRW = 10), 1e8 packets
per step, the overflow roulette at maxinteract = 1e5 (keyword 'maxinteract',
MCRadiation.f:568-571).  All inputs are synthetic and seeded.

Forms.  The fast form -- mixed-precision transport on opacities from the
opacity surrogate network -- is the headline `value`: packets per second of
the transport kernel's device time over the K timed steps, tables resident
in HBM.  `e2e` times the same K steps end to end through the C-ABI from host
buffers: the surrogate opacity stage, the model set-up (mcg_set_model from
host arrays), the packet loop, and the per-cell results and temperatures
back on the host.  The plain form -- FP64 transport on the DHS kernels'
opacities -- runs beside it on the same Philox streams (`fp64_form`), and a
second FP64 run with another seed gives the Monte Carlo noise floor of the
agreement figures (`accuracy`: per-cell temperatures of cells with >= 1e3
absorption events within 1 %, SED bins with S/N > 50 within 2 %).  The
precision deck (one composition, MRN 0.1-1 micron in 20 bins, no settling)
is reported as `precision_deck` in both forms.

--impl reference runs the oracle (the CPU restatement of the reference's
loop; the Fortran reference cannot be compiled without a Fortran compiler) on
every host core, on the same deck with the DHS opacity tables.
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
RUN = dict(randomwalk=True, factRW=10.0, maxinteract=100_000)
METRIC = "packets/s on 1 B200: mixed-prec+surrogate vs plain FP64 GPU at equal T/SED error"
WORKLOAD = ("learned-opacities deck: 3 compositions x 50 bins 0.01-1000 micron (ns 5, nf 20), settling alpha 1e-3, "
            "Mdust 1e-3 Msun, nr 200 x ntheta 120, nlam 200, random walk factRW 10, full Mueller scattering, "
            "maxinteract 1e5")
PRECISION_DECK = dict(mdust=1e-3, nrad=200, ntheta=120, nlam=200, lam1=0.1, lam2=3000.0, ngrains=20, ns=5, nf=20,
                      fmax=0.8, blend=True, porosity=0.25, scat_how=2)
SURROGATE = os.path.join(ROOT, "mcmax_b200", "data", "surrogate_nf20.npz")
TRAFFIC_PROFILE = os.path.join(ROOT, "profiles", "transport_event_learned_deck_2e6.md")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nphot", type=int, default=NPHOT_DEFAULT)
    ap.add_argument("--maxinteract", type=int, default=RUN["maxinteract"],
                    help="overflow roulette (keyword maxinteract); smaller values shorten the trapped-packet tail "
                         "for profiling runs")
    ap.add_argument("--no-compare", action="store_true", help="skip the FP64 + DHS form and the accuracy figures")
    ap.add_argument("--no-precision-deck", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-post-mc", action="store_true",
                    help="skip the timing of the steps after the packet loop (Diffuse, structure, spectrum, image)")
    ap.add_argument("--cpu-sample-seconds", type=float, default=15.0)
    ap.add_argument("--ref-packets", type=int, default=0,
                    help="reference arm: packets per step (0: sized to about 8 s per step on the host cores)")
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


def algorithmic_bytes(counters, nlam):
    """Per-event byte model of the packet loop (the reads and read-modify-
    writes an event needs at minimum): crossing 72 B + 16 B EJv2 on exit,
    absorption 64 B + nlam*24 B re-emission row, scattering 2*180*8 + 48 B,
    random-walk step 56 B, escape 16 B."""
    cross, absorb, scat, rw, esc = (int(counters[k]) for k in (8, 2, 3, 4, 9))
    return cross * (72 + 16) + absorb * (64 + 24 * nlam) + scat * (2 * 180 * 8 + 48) + rw * 56 + esc * 16


def traffic_per_packet():
    """DRAM bytes per packet of the transport kernel on this deck, from the
    ncu capture summarised in the profiles folder (dram__bytes_read.sum +
    dram__bytes_write.sum of one launch / its packets), or None."""
    try:
        with open(TRAFFIC_PROFILE) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_packet:"):
                    return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


def learned_step(ctx, params, nphot, seed, precision, opacity, fetch=True):
    """One end-to-end model run through the public API: the opacity stage
    (the surrogate network or the DHS kernels), the model set-up from host
    arrays, the packet loop, the post-run temperatures on the host."""
    from mcmax_b200 import model as M
    t0 = time.perf_counter()
    m, t_opac, served = M.learned_disk_model(ctx, opacity=opacity, params=params)
    ctx.set_model(m)
    n, o = ctx.mcradiation(nphot, seed=seed, precision=precision, fetch=fetch, **RUN)
    if fetch:
        o["T"], _, _ = ctx.finalize_t()
    wall = time.perf_counter() - t0
    return m, o, {"wall_s": wall, "opacity_stage_s": t_opac, "bins_served_by_network": served,
                  "device_ms": o["device_ms"]}


def io_bytes(m):
    """Host -> device bytes of one model set-up (the arrays mcg_set_model
    uploads and the opacity stage's inputs) and device -> host bytes of one
    run's results (per-cell EJv, EJv2, Eabs, T, Ni, Nabs, the spectra and
    the post-run temperatures)."""
    import numpy as np
    h2d = sum(np.asarray(getattr(m, k)).nbytes for k in ("R", "Theta", "SinTheta", "dens", "V", "comp_w", "lam", "nu",
                                                            "Kabs", "Ksca", "F", "BB", "Fstar"))
    h2d += m.ncomp * m.nlam * 8 * 3  # lam, n, k of every grain bin
    d2h = m.ncell * (8 * 4 + 4 * 2) + m.nlam * 31 * (8 * 2 + 4) + m.ncell * 8 * 3
    return int(h2d), int(d2h)


def agreement(ref, other):
    """Agreement of a run with a reference run: per-cell temperatures of the
    cells with >= 1e3 absorption events in the reference run (within 1 %,
    median and 95th percentile of the relative difference), and the SED
    (MCRadiation.f:581-646) in the (wavelength, inclination) bins and the
    inclination-summed bins whose packet counts give S/N > 50 on both
    sides (within 2 %, median)."""
    import numpy as np
    nc_star = ref["_nt"] - 1
    sel = (np.asarray(ref["Nabs"]) >= 1000) & (np.arange(ref["T"].size) >= nc_star) & (ref["T"] > 0)
    rel = np.abs(other["T"][sel] / ref["T"][sel] - 1)
    out = {"cells_nabs_ge_1e3": int(sel.sum()), "T_within_1pct": float(np.mean(rel < 0.01)),
           "T_median_rel": float(np.median(rel)), "T_p95_rel": float(np.percentile(rel, 95))}
    a, b = ref["spec"][:, 1:], other["spec"][:, 1:]
    na, nb = ref["ispec"][:, 1:], other["ispec"][:, 1:]
    for tag, x, y, cx, cy in (("sed_bins", a, b, na, nb), ("sed_lam", a.sum(1), b.sum(1), na.sum(1), nb.sum(1))):
        ok = (cx > 2500) & (cy > 2500) & (x > 0)
        r = np.abs(y[ok] / x[ok] - 1)
        out[tag + "_sn50"] = int(ok.sum())
        out[tag + "_within_2pct"] = float(np.mean(r < 0.02)) if ok.any() else None
        out[tag + "_median_rel"] = float(np.median(r)) if ok.any() else None
    return out


def post_mc_steps(ctx, model, res):
    """The steps after the packet loop on the headline deck and the last
    timed run's result, each C-ABI call timed on the host (every call ends
    with a device synchronisation): the temperatures (mcg_finalize_t),
    Diffuse (mcg_diffuse), one vertical-structure pass on the zone taken as
    not fixed (mcg_disk_structure), the ray-traced spectrum at 45 degrees on
    the grid's wavelengths (mcg_trace_spectrum), without and with scattered
    light, and a 500 x 500 image with
    1000 points per image cell at the middle of the wavelength range
    (mcg_trace_image).  Not part of the headline metric."""
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
    # the same spectrum with scattered light at an observation's defaults:
    # per wavelength one TraceMono field of 1000 starlight and 1000 Monte
    # Carlo packets, five exit rays per cell
    sc = dict(nphot=1000, nphot_star=1000, seed=7, nexits=5)
    (fsc, info), t = timed(lambda: ctx.trace_spectrum(Td, lam_obs, math.radians(45.0), scatter=sc))
    ok = flux > 0
    out["trace_spectrum_scattered"] = {"s": t, "fields": int(lam_obs.size), "packets_per_field": 2000,
                                       "median_scattered_share": float(np.median(1.0 - flux[ok] / fsc[ok]))}
    lam0 = (model.lam[0] + model.lam[-1]) / 2.0
    img, t = timed(lambda: ctx.trace_image(Td, lam0, math.radians(45.0), npixel=500, nint=1000))
    pts = (img["info"][0] - 1) * 45 * 1000
    out["trace_image"] = {"s": t, "points": int(pts), "points_per_s": pts / t,
                          "sum_over_flux": float(img["image"].sum() / img["flux"])}
    return out


def oracle_tables(m):
    """The oracle's tables of a model (one set, shared read-only by every
    thread that runs the oracle's packet loop on it)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_ffi as O
    return O, O.transport_tables(m, randomwalk=RUN["randomwalk"], factRW=RUN["factRW"], lazy_kd=True)


def cpu_baseline_sample(m, seconds):
    """The oracle (the serial CPU restatement of the reference loop) on a
    bounded sample of the same deck and tables: packets until ~`seconds` of
    work, one core."""
    O, tab = oracle_tables(m)
    n = 20
    total_n, total_t = 0, 0.0
    while total_t < seconds and total_n < 200000:
        t0 = time.perf_counter()
        O.mcradiation(m, n, seed=1000 + total_n, randomwalk=RUN["randomwalk"], factRW=RUN["factRW"],
                      maxinteract=RUN["maxinteract"], tables=tab)
        dt = time.perf_counter() - t0
        total_n += n
        total_t += dt
        n = min(4 * n, max(20, int(n * (seconds - total_t) / max(dt, 1e-3))))
        if n <= 0:
            break
    return total_n / total_t, total_n, total_t


def run_reference(args, rank, world):
    """The oracle's packet loop on every host core: independent chunks of
    packets (the oracle releases the interpreter lock inside its C calls)
    from one pool of threads sharing the deck's tables, K steps of work
    queued back to back after W warm-up steps.  The deck's DHS opacity tables
    come from the library's ComputePart kernels (equal bit for bit to the
    oracle's ComputePart, tests/test_gpu_part.py); only the packet loop is
    timed."""
    from concurrent.futures import ThreadPoolExecutor, wait
    if rank != 0:
        return
    from mcmax_b200 import api
    from mcmax_b200 import model as M
    ctx = api.Context(int(os.environ.get("LOCAL_RANK", "0")))
    m, _, _ = M.learned_disk_model(ctx, opacity="dhs")
    ctx.close()
    O, tab = oracle_tables(m)
    cores = os.cpu_count() or 1
    chunk = 100  # the calibration's; the timed steps use larger chunks

    def work(seed):
        O.mcradiation(m, chunk, seed=seed, randomwalk=RUN["randomwalk"], factRW=RUN["factRW"],
                      maxinteract=RUN["maxinteract"], tables=tab)

    seed = [50_000]

    def batch(nchunks):
        s0 = seed[0]
        seed[0] += nchunks
        return [s0 + k for k in range(nchunks)]

    with ThreadPoolExecutor(cores) as ex:
        # calibration: two chunks per core
        t0 = time.perf_counter()
        wait([ex.submit(work, s) for s in batch(2 * cores)])
        rate = 2 * cores * chunk / (time.perf_counter() - t0)
        per_step = args.ref_packets or max(cores * chunk, int(rate * 8.0) // chunk * chunk)
        # chunks large enough that the oracle's lazily evaluated diffusion
        # coefficients are reused within a call, four per thread and step
        chunk = max(100, per_step // (4 * cores))
        per_step = per_step // chunk * chunk
        nchunks = per_step // chunk
        for _ in range(args.warmup):
            wait([ex.submit(work, s) for s in batch(nchunks)])
        t0 = time.perf_counter()
        wait([ex.submit(work, s) for s in batch(nchunks * args.steps)])
        wall = time.perf_counter() - t0
    value = per_step * args.steps / wall
    sample = ("%d packets per step in chunks of %d on %d threads, %d steps queued back to back after %d warm-up steps"
              % (per_step, chunk, cores, args.steps, args.warmup))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "packets/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD + " (CPU restatement of the reference loop, DHS opacities)",
                       "packets_per_step": per_step, "parallelism": "host threads"},
            "cpu_baseline": {"value": value, "unit": "packets/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "packets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
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
    from mcmax_b200 import model as M
    from mcmax_b200 import surrogate as S

    ctx = api.Context(local)
    params, sinfo = S.load(SURROGATE)
    for w in range(args.warmup):
        learned_step(ctx, params, args.nphot, 10_000 * (rank + 1) + w, "mixed", "surrogate", fetch=False)
    _barrier(dist)
    clocks = ClockSampler(local)
    clocks.start()
    dev_ms, walls, infos = [], [], []
    counters = np.zeros(16, np.int64)
    seeds = [rank * 1_000_003 + s + 1 for s in range(args.steps)]
    for s in range(args.steps):
        m, o, info = learned_step(ctx, params, args.nphot, seeds[s], "mixed", "surrogate")
        dev_ms.append(info["device_ms"])
        walls.append(info["wall_s"])
        infos.append(info)
        counters += o["counters"]
    clk = clocks.stop()
    _barrier(dist)
    t_dev = _max_over_ranks(dist, sum(dev_ms) / 1e3)
    t_e2e = _max_over_ranks(dist, sum(walls))
    packets = args.nphot * args.steps * world
    value = packets / t_dev
    e2e_value = packets / t_e2e
    h2d, d2h = io_bytes(m)
    last = dict(o, _nt=m.nt)
    mixed_model = m
    extra = {}
    if rank == 0 and world == 1 and not args.no_post_mc:
        try:
            extra["post_mc"] = post_mc_steps(ctx, mixed_model, last)
        except Exception as e:  # the extra timings must not sink the GPU line
            extra["post_mc"] = {"failed": str(e)}
    dhs_model = None
    if rank == 0 and world == 1 and not args.no_compare:
        # the plain form on the same Philox streams as the last timed step,
        # and once more with another seed (the noise floor)
        dhs_model, od, infod = learned_step(ctx, None, args.nphot, seeds[-1], "fp64", "dhs")
        _, od2 = ctx.mcradiation(args.nphot, seed=seeds[-1] + 7_777, precision="fp64", fetch=True, **RUN)
        od2["T"], _, _ = ctx.finalize_t()
        od = dict(od, _nt=dhs_model.nt)
        fp64_ms = (od["device_ms"] + od2["device_ms"]) / 2.0
        extra["fp64_form"] = {
            "value": args.nphot / (fp64_ms / 1e3), "unit": "packets/s", "steps": 2, "ms_per_step": fp64_ms,
            "dtype": "f64", "opacities": "DHS kernels (ComputePart.f) for all 150 bins",
            "opacity_stage_s": infod["opacity_stage_s"], "e2e_step_s": infod["wall_s"],
            "e2e_packets_per_s": args.nphot / infod["wall_s"], "progress_ms": od["progress_ms"]}
        extra["speedup_vs_fp64_form"] = {"transport": value / extra["fp64_form"]["value"],
                                         "e2e": infod["wall_s"] / statistics.mean(walls)}
        extra["accuracy"] = {
            "criterion": "per-cell T of cells with >= 1e3 absorption events within 1 % of the FP64 + DHS run on the "
                         "same Philox streams; SED bins with S/N > 50 within 2 %",
            "mixed_surrogate_vs_fp64_dhs": agreement(od, last),
            "noise_floor_fp64_dhs_other_seed": agreement(od, od2),
            "surrogate": {"train_samples": int(sinfo["n"]), "epochs": int(sinfo["epochs"]),
                          "bins_median_dex_kabs": float(sinfo["bins_median_dex_kabs"]),
                          "bins_median_dex_ksca": float(sinfo["bins_median_dex_ksca"])}}
    if rank == 0 and world == 1 and not args.no_precision_deck:
        pm = M.disk_model(ctx, **PRECISION_DECK)
        ctx.set_model(pm)
        ctx.mcradiation(1_000_000, seed=3, precision="mixed", fetch=False, **RUN)
        pd = {}
        for prec in ("mixed", "fp64"):
            _, op = ctx.mcradiation(args.nphot, seed=5, precision=prec, fetch=False, **RUN)
            pd[prec] = {"value": args.nphot / (op["device_ms"] / 1e3), "unit": "packets/s", "steps": 1,
                        "ms_per_step": op["device_ms"], "progress_ms": op["progress_ms"]}
        pd["workload"] = ("precision disk deck: one composition, MRN 0.1-1 micron in 20 bins (ns 5, nf 20, fmax 0.8, "
                          "porosity 0.25), Mdust 1e-3 Msun, nr 200 x ntheta 120, nlam 200, random walk factRW 10, "
                          "maxinteract 1e5, %d packets" % args.nphot)
        extra["precision_deck"] = pd
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            if dhs_model is None:
                dhs_model, _, _ = M.learned_disk_model(ctx, opacity="dhs")
            v, n, t = cpu_baseline_sample(dhs_model, args.cpu_sample_seconds)
            cpu = {"value": v, "unit": "packets/s", "cores": 1, "kind": "port",
                   "sample": "%d packets of the same deck (DHS opacities), serial CPU restatement, %.1f s" % (n, t)}
        except Exception as e:  # the baseline must not sink the GPU line
            cpu = {"value": None, "unit": "packets/s", "cores": 1, "kind": "port", "sample": "failed: %s" % e}
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    peak = peaks.get("hbm_gbs")
    peak_src = "measured"
    if not peak:
        peak, peak_src = 6650.0, "fallback"
    per_launch_s = t_dev / args.steps
    algo = algorithmic_bytes(counters, mixed_model.nlam) / args.steps
    achieved = algo / per_launch_s / 1e9
    tpp = traffic_per_packet()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "packets/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_dev / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": WORKLOAD + ", mixed-precision transport on surrogate opacities",
                       "packets_per_step": args.nphot, "precision": "mixed", "opacities": "surrogate network",
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": "inputs larger than L2 (126 MB): per-cell opacity rows, Planck-mean and re-emission "
                             "tables, Mueller tables; no flush between steps"},
            "e2e": {"value": e2e_value, "unit": "packets/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "step": "surrogate opacity stage + mcg_set_model from host arrays + mcg_mcradiation + results "
                            "and temperatures to the host",
                    "opacity_stage_s": statistics.mean(i["opacity_stage_s"] for i in infos)},
            # 23 kernels per end-to-end step (the launch list of one step in
            # the profiles folder: the surrogate, the model tables, the
            # transport kernel, the run combination, the temperatures)
            "gpu_launches": 23 * args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": tpp * args.nphot if tpp else None,
                         "note": "algorithmic bytes from the event counters (crossings, absorptions, scatterings, "
                                 "random-walk steps, escapes) per launch / transport-kernel time; peak = %s HBM copy "
                                 "bandwidth; traffic = DRAM bytes per packet of an ncu capture of this kernel on this "
                                 "deck (2e6 packets) x packets per launch" % peak_src},
            "progress_ms_last_step": o["progress_ms"],
            "events_per_step": {"crossings": int(counters[8] // args.steps),
                                "absorptions": int(counters[2] // args.steps),
                                "scatterings": int(counters[3] // args.steps),
                                "rw_steps": int(counters[4] // args.steps),
                                "lanes_per_crossing_step": float(counters[15] / max(counters[14], 1)),
                                "lanes_per_phase": float(counters[13] / max(counters[12], 1))},
            "clocks": clk, "cpu_baseline": cpu,
        }
        line.update(extra)
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
