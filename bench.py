#!/usr/bin/env python
"""Benchmark of the ipole ray pipeline on B200.

Workload (the headline configuration): a seeded synthetic iharm FMKS dump of
288x128x128 zones (seed 1), imaged at 400x400 pixels, full polarization,
230 GHz, thetacam 163 deg, R_high 160 / R_low 1, MBH 6.5e9 Msun, D 16.8 Mpc,
160 muas field of view, M_unit chosen so that the total flux is ~0.6 Jy.
One *step* is one complete 400^2 image (every pixel traced, no refinement).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` = images/s with the pixel list and outputs resident in device memory
(ipg_trace_pixels_device), `e2e` = images/s through the host image driver
(ipg_render_image: host pixel lists, host output arrays, copies in the timed
region).  `mixed_records` times the same image in the mixed form: compact
step records (ipg_set_record_precision) and the polarized step in FP32
(ipg_set_step_precision), with its error against the FP64 image;
`--records mixed --step fp32` select them for a --quick run.  Under torchrun each rank
renders its own image (weak scaling, no collective on the data path); time
is the max over ranks.  The reference arm
runs the reference ipole built from its sources (oracle/_ref/ipole, the
makefile's -O3 flags, OpenMP on every host core) on a bounded 64^2 sample of
the same workload and scales it to a 400^2 image.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "IQUV 400² images/s & ray-steps/s, 1 B200: plain FP64 vs mixed+batched+adjoint"
DUMP = dict(n1=288, n2=128, n3=128, seed=1)
SMALL_DUMP = dict(n1=128, n2=64, n3=64, seed=1)
NX = NY = 400
M_UNIT = 7.96e27  # total flux 0.6 Jy at R_high 160, thetacam 163 (tests/golden/tune_munit.py)
BASE_ARGS = ["--freqcgs=230.e9", "--thetacam=163", "--phicam=0", "--rotcam=0", "--MBH=6.5e9", "--dsource=16.8e6",
             "--fov=160", "--trat_large=160", "--trat_small=1"]
CPU_SAMPLE = 64  # reference / oracle sample image size (pixels per side)
# The reference algorithm's FP64 work, counted exactly by running the oracle's
# restatement of it over a counting number type on the 128x128 image of the
# 128x64x64 dump (oracle/opcount/count_ops.py -> counts_c1_128.json; each
# transcendental call weighted 20 flops): per ray-step, the geodesic step
# (push_photon, stepsize, stop test) and the two push_polar calls of
# integrate_emission; per radiating step, the coefficients (point queries,
# get_jkinv, jar_calc, plasma tetrad) and the transfer arithmetic (evolve_N).
# These are the algorithmic flops of the roofline: the geodesic kernel does
# the geodesic and the connections, the coefficient and transfer kernels the
# rest.
REF_FLOPS = {"geodesic_per_step": 24172.6, "push_per_step": 30454.0, "coeffs_per_radiating_step": 8942.3,
             "transfer_per_radiating_step": 4751.9}
# What the kernels execute per ray-step, from the ncu capture of a 200x200
# image of the 128x64x64 dump: FP64 flops (2 per DFMA, 1 per DADD/DMUL) and
# DRAM bytes read + written (k_coeffs works per step record); the walk's
# bytes are those of its bulk-copy form (the image's walk outside the
# longest class) on an unsplit 256x256 wave of the same dump, 618 per step
# against 539 for its 16-byte-copy form.
EXEC_FLOPS_PER_STEP = {"geodesic": 1831, "coeffs": 1535, "transfer": 913}
DRAM_BYTES_PER_STEP = {"geodesic": 377, "coeffs": 412, "transfer": 619}


def data_dir():
    d = os.environ.get("IPG_BENCH_DATA", os.path.join(tempfile.gettempdir(), "ipole_b200_bench"))
    os.makedirs(d, exist_ok=True)
    return d


def ensure_dump(spec, tag=""):
    from ipole_b200 import synthdump
    path = os.path.join(data_dir(), f"dump_{spec['n1']}x{spec['n2']}x{spec['n3']}_s{spec['seed']}{tag}.ipgc")
    if not os.path.exists(path):
        tmp = path + f".tmp{os.getpid()}"
        synthdump.write_iharm_dump(tmp, spec["n1"], spec["n2"], spec["n3"], seed=spec["seed"])
        os.replace(tmp, path)
    return path


def workload_args(dump, nx, ny, m_unit):
    return [f"--dump={dump}", *BASE_ARGS, f"--M_unit={m_unit:g}", f"--nx={nx}", f"--ny={ny}"]


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
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
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    """One process per GPU under torchrun (RANK / LOCAL_RANK / WORLD_SIZE from
    the environment).  NCCL on GPUs; IPG_DIST_BACKEND=gloo runs the same host
    logic on CPU processes (tests)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = os.environ.get("IPG_DIST_BACKEND", "nccl")
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=60))
    return rank, world, local


def _dist_device():
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_dist_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_dist_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def images_per_s(world, steps, ms_max):
    """Whole-job throughput: every rank renders one image per step (weak
    scaling); the job takes as long as its slowest rank."""
    return world * steps / (ms_max / 1e3)


def cpu_reference_sample(dump, m_unit, n=CPU_SAMPLE, threads=None):
    """Time the reference binary (or, without it, the C restatement) on an
    n x n image of the workload; returns dict with seconds per 400^2 image."""
    threads = threads or os.cpu_count()
    from oracle import oracle as orc
    if orc.have_reference_binary():
        out = os.path.join(data_dir(), f"ref_sample_{os.getpid()}.ipgc")
        rc, err = orc.run_reference([*workload_args(dump, n, n, m_unit), f"--outfile={out}"], binary=orc.REF_BIN,
                                    threads=threads)
        if rc != 0:
            raise RuntimeError("reference run failed: " + err[-500:])
        m = re.search(r"Total wallclock time: ([0-9.eE+-]+) s \(([0-9.eE+-]+) s\)", err)
        render_s = float(m.group(1)) - float(m.group(2))
        ftot = float(re.search(r"Ftot: ([0-9.eE+-]+) Jy", err).group(1))
        kind = "reference"
    else:
        import ipole_b200 as ip
        p = ip.Params.from_args(workload_args(dump, n, n, m_unit))
        mdl = ip.Model.load(p)
        o = orc.Oracle(mdl.grid, [mdl.field(q) for q in range(10)])
        cam = o.camera(p.rcam, p.thetacam, p.phicam, p.rotcam, p.fovx_dsource, p.dsource, n, n, p.freqcgs)
        ij = [(i, j) for i in range(n) for j in range(n)]
        t0 = time.perf_counter()
        o.trace(cam, ij, threads=threads)
        render_s = time.perf_counter() - t0
        ftot = None
        kind = "port"
    per_image = render_s * (NX * NY) / (n * n)
    return {"seconds_per_image": per_image, "render_s": render_s, "kind": kind, "cores": threads,
            "sample": f"{n}x{n} image of the same workload ({n * n} rays), scaled by pixel count to 400x400",
            "Ftot_sample": ftot}


def run_reference_arm(args):
    rank, world, _ = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), 0
    if rank != 0:
        return 0
    dump = ensure_dump(DUMP)
    times = []
    for s in range(args.warmup + args.steps):
        r = cpu_reference_sample(dump, args.m_unit)
        if s >= args.warmup:
            times.append(r)
    per = statistics.mean(t["seconds_per_image"] for t in times)
    v = 1.0 / per
    line = {"metric": METRIC, "value": v, "unit": "images/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "iharm FMKS 288x128x128 seed 1, 400x400 IQUV, 230 GHz, thetacam 163, "
                                   f"R_high 160, plain FP64 ({CPU_SAMPLE}² sample scaled to 400²)",
                       "M_unit": args.m_unit},
            "cpu_baseline": {"value": v, "unit": "images/s", "cores": times[0]["cores"], "kind": times[0]["kind"],
                             "sample": times[0]["sample"]},
            "e2e": {"value": v, "unit": "images/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_ours(args):
    import numpy as np
    import torch

    import ipole_b200 as ip
    rank, world, local = dist_setup()
    torch.cuda.set_device(local)
    spec = SMALL_DUMP if args.small else DUMP
    nx = ny = args.size
    dump = ensure_dump(spec, tag=f"_r{rank}" if world > 1 else "")
    extra = [f"--eps={args.eps}"] if args.eps else []
    p = ip.Params.from_args(workload_args(dump, nx, ny, args.m_unit) + extra)
    model = ip.Model.load(p)
    ctx = ip.Context(local, pool_bytes=int(args.pool_gb * (1 << 30)))
    if args.records == "mixed":
        ctx.set_record_precision(ip.IPG_RECORDS_MIXED)
    if args.step == "fp32":
        ctx.set_step_precision(ip.IPG_STEP_FP32)
    ctx.upload(model)
    cam = ip.camera_for(p, model.grid)
    ij = np.array([(i, j) for i in range(nx) for j in range(ny)], dtype=np.int32)
    n = len(ij)
    d_ij = torch.from_numpy(ij).cuda()
    d_out = torch.empty(n * ip.PIXEL_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.ExternalStream(ctx.stream())

    for _ in range(args.warmup):
        ctx.trace_device(cam, d_ij.data_ptr(), n, d_out.data_ptr())
    torch.cuda.synchronize()
    barrier(world)
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    steps = rad = launches = 0
    kms = {"geodesic": 0.0, "coeffs": 0.0, "transfer": 0.0}
    span = {"geodesic": 0.0, "coeffs": 0.0, "transfer": 0.0}
    pred_ms = wall_ms = 0.0
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        ctx.trace_device(cam, d_ij.data_ptr(), n, d_out.data_ptr())
        s = ctx.stats()
        steps += s["ray_steps"]
        rad += s["radiating_steps"]
        launches += s["launches"]
        for k in kms:
            kms[k] += s[f"{k}_ms"]
            span[k] += s[f"{k}_span_ms"]
        pred_ms += s["predict_ms"]
        wall_ms += s["wall_ms"]
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, world)
    total_steps = sum_over_ranks(float(steps), world)
    value = images_per_s(world, args.steps, ms_max)
    out = np.frombuffer(d_out.cpu().numpy().tobytes(), dtype=ip.PIXEL_DTYPE)
    f3 = p.freqcgs ** 3
    ftot = float(out["I"].sum() * f3 * cam._scale)

    if args.quick:
        if rank == 0:
            print(json.dumps({"quick": True, "value": value, "ms_per_step": ms_max / args.steps,
                              **{f"{k}_ms": v / args.steps for k, v in kms.items()},
                              "predict_ms": pred_ms / args.steps, "device_wall_ms": wall_ms / args.steps,
                              "ray_steps_per_image": steps / args.steps, "Ftot_Jy": ftot, "clocks": clk,
                              "lib": os.environ.get("IPOLE_B200_LIB", "default")}))
        ctx.close()
        return 0
    # e2e: the image API (ipg_render_image): host parameters in, host image
    # out; the per-call uploads (camera and grid constants) and the image
    # read-back are inside the timed region
    ctx.render(p, model)
    torch.cuda.synchronize()
    barrier(world)
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        ctx.render(p, model)
    e3.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    e2e_ms = max_over_ranks(e2.elapsed_time(e3), world)
    import ctypes
    img_bytes = n * (8 + 8 + 5 * 8 + 3 * 4)  # image, taus, imageS, interp/oddflag/nstep
    e2e = {"value": images_per_s(world, args.steps, e2e_ms), "unit": "images/s",
           "h2d_bytes_per_step": int(ctypes.sizeof(ip.Camera) + ctypes.sizeof(ip.Grid)),
           "d2h_bytes_per_step": int(img_bytes),
           "api": "ipg_render_image: host parameters in, host image out (pixel lists built on the device)"}

    # the compact-record form (ipg_set_record_precision): the same image with
    # the transport matrices and tetrad rows stored in FP32 between the
    # kernels, timed like the headline, and its error against that image
    ctx.set_record_precision(ip.IPG_RECORDS_MIXED)
    ctx.set_step_precision(ip.IPG_STEP_FP32)
    ctx.set_fit_precision(ip.IPG_FITS_FP32)
    ctx.trace_device(cam, d_ij.data_ptr(), n, d_out.data_ptr())
    torch.cuda.synchronize()
    barrier(world)
    m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    m0.record(stream)
    for _ in range(args.steps):
        ctx.trace_device(cam, d_ij.data_ptr(), n, d_out.data_ptr())
    m1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    mixed_ms = max_over_ranks(m0.elapsed_time(m1), world)
    mo = np.frombuffer(d_out.cpu().numpy().tobytes(), dtype=ip.PIXEL_DTYPE)
    ctx.set_record_precision(ip.IPG_RECORDS_FP64)
    ctx.set_step_precision(ip.IPG_STEP_FP64)
    ctx.set_fit_precision(ip.IPG_FITS_FP64)
    I0, Q0, U0, V0 = (float(out[k].sum()) for k in "IQUV")
    I1, Q1, U1, V1 = (float(mo[k].sum()) for k in "IQUV")
    bright = out["I"] > 1e-6 * out["I"].max()
    mixed = {"value": images_per_s(world, args.steps, mixed_ms), "unit": "images/s",
             "ms_per_step": mixed_ms / args.steps,
             "form": "compact step records (transport matrices and tetrad rows in FP32), the polarized "
                     "step (Faraday rotation, absorption/emission) in FP32 and the thermal fits' shapes in FP32 "
                     "(prefactors and exponents FP64); geodesics, metric, tetrads and the accumulation of N in "
                     "FP64",
             "vs_fp64": {"Ftot_rel": abs(I1 / I0 - 1), "Q_rel_to_I": abs(Q1 - Q0) / abs(I0),
                         "U_rel_to_I": abs(U1 - U0) / abs(I0), "V_rel_to_I": abs(V1 - V0) / abs(I0),
                         "EVPA_deg": abs(float(np.degrees(0.5 * (np.arctan2(U1, Q1) - np.arctan2(U0, Q0))))),
                         "pix_I_max_rel": float(np.max(np.abs(mo["I"][bright] / out["I"][bright] - 1)))}}

    batched = bench_batched(ip, ctx, model, dump, args, world, stream, ms_max / args.steps)
    adjoint = bench_adjoint(ip, ctx, model, p, args, world, stream)
    ctx.upload(model)

    peak = ip.fp64_peak_tflops(local, 300.0)
    peak32 = ip.fp32_peak_tflops(local, 300.0)
    # algorithmic flops (the reference algorithm's counted work) of each
    # kernel over the timed images, against each kernel's wall span (first
    # class start to last class end, per wave) and the whole pipeline against
    # the image time
    alg = {"geodesic": (REF_FLOPS["geodesic_per_step"] + REF_FLOPS["push_per_step"]) * steps,
           "coeffs": REF_FLOPS["coeffs_per_radiating_step"] * rad,
           "transfer": REF_FLOPS["transfer_per_radiating_step"] * rad}
    dom = max(span, key=span.get)
    kern = {k: {"span_ms_per_image": span[k] / args.steps, "summed_class_ms_per_image": kms[k] / args.steps,
                "alg_tflops": alg[k] / (span[k] / 1e3) / 1e12 if span[k] > 0 else None,
                "exec_tflops": EXEC_FLOPS_PER_STEP[k] * steps / (span[k] / 1e3) / 1e12 if span[k] > 0 else None}
            for k in kms}
    for k in kern:
        a, x = kern[k]["alg_tflops"], kern[k]["exec_tflops"]
        kern[k]["alg_frac"] = a / peak if a else None
        kern[k]["exec_frac"] = x / peak if x else None
    achieved = kern[dom]["alg_tflops"]
    alg_total = sum(alg.values())
    exec_total = sum(EXEC_FLOPS_PER_STEP.values()) * steps
    traffic = DRAM_BYTES_PER_STEP[dom] * (steps / args.steps)
    # the walk of FP64 records fetches them by bulk copies into shared memory
    # (16-byte copies in the longest length class) unless IPG_XFER_STAGE
    # selects 16-byte copies (1) or global loads (0) for every class
    walk = {"0": "k_transfer", "1": "k_transfer_staged"}.get(os.environ.get("IPG_XFER_STAGE", ""),
                                                           "k_transfer_bulk (k_transfer_staged for the longest class)")
    kname = walk if dom == "transfer" else f"k_{dom}"
    roofline = {"bound": "fp64", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                "traffic_note": "DRAM bytes per image (all class launches of the kernel): ncu bytes per ray-step "
                                "of a small case of the 128x64x64 dump (the walk: its bulk-copy form on an "
                                "unsplit 256x256 wave) times this image's ray-steps",
                "frac_pipeline": alg_total / (ms / 1e3) / 1e12 / peak,
                "frac_pipeline_executed": exec_total / (ms / 1e3) / 1e12 / peak,
                "alg_flops_per_ray_step": alg_total / max(steps, 1),
                "exec_flops_per_ray_step": exec_total / max(steps, 1),
                "alg_note": "algorithmic = the reference algorithm's FP64 operations counted with a counting "
                            "number type (transcendentals 20 flops); the kernels execute ~15x fewer (analytic "
                            "connection and metric instead of finite differences of gcov with LU inversions), "
                            "so the algorithmic fractions can exceed 1; *_executed uses ncu's executed FP64 flops",
                "kernels": kern, "hbm_GBps_of_dominant": traffic * args.steps / (span[dom] / 1e3) / 1e9,
                "peak_source": "measured in this run: FP64 FMA loop (ipg_measure_fp64_peak); MEASURED_PEAKS.json "
                               "has no FP64 figure",
                "fp32_peak_tflops": peak32, "predict_ms_per_image": pred_ms / args.steps}
    line = {"metric": METRIC, "value": value, "unit": "images/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": ("iharm FMKS 288x128x128 seed 1" if not args.small else
                                    "iharm FMKS 128x64x64 seed 1") + f", {nx}x{ny} IQUV, 230 GHz, thetacam 163, "
                                                                     "R_high 160, plain FP64",
                       "M_unit": args.m_unit, "parallelism": f"replicas x{world} (one image per GPU)",
                       "l2": "inputs larger than L2: 392 MB field array + trajectory pool writes per step"},
            "ray_steps_per_s": total_steps / (ms_max / 1e3), "ray_steps_per_image": steps / args.steps,
            "radiating_fraction": rad / max(steps, 1), "Ftot_Jy": ftot, "e2e": e2e, "roofline": roofline,
            "clocks": clk, "gpu_launches": launches, "mixed_records": mixed, "batched": batched,
            "adjoint": adjoint}
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            cb = cpu_reference_sample(dump, args.m_unit)
            line["cpu_baseline"] = {"value": 1.0 / cb["seconds_per_image"], "unit": "images/s", "cores": cb["cores"],
                                    "kind": cb["kind"], "sample": cb["sample"],
                                    "ray_steps_per_s": (steps / args.steps) / cb["seconds_per_image"]}
        except Exception as ex:  # reported, not fatal
            line["cpu_baseline"] = {"value": None, "unit": "images/s", "error": str(ex)[:300]}
    if rank == 0:
        print(json.dumps(line))
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


# Batches of instances (ipg_render_batch).  The headline batch is the bench
# image's camera with the electron models of the batched workload: R_high
# {1, 10, 40, 160} x M_unit {0.5, 2} x the bench's, 8 images of 400x400.  The
# batched workload itself: {86, 230, 345} GHz x inclinations {17, 60, 120,
# 163} x the same 8 electron models, 96 images; each of the 12 cameras has
# its own resolution, 64, 160 or 320 pixels a side in turn, refined from a
# quarter of it (refine_abs 2e-2, refine_rel 1e-2).
BATCH_RHIGH = (1, 10, 40, 160)
BATCH_MU = (0.5, 2.0)
BATCH_FREQS = (86e9, 230e9, 345e9)
BATCH_INCL = (17, 60, 120, 163)
BATCH_RES = (64, 160, 320)


def batch_params(ip, dump, m_unit, nx, incl=163, freq=230e9, refine=False):
    out = []
    for rh in BATCH_RHIGH:
        for f in BATCH_MU:
            a = [f"--dump={dump}", f"--freqcgs={freq:.6g}", f"--thetacam={incl}", "--phicam=0", "--rotcam=0",
                 "--MBH=6.5e9", "--dsource=16.8e6", "--fov=160", "--trat_small=1", f"--trat_large={rh}",
                 f"--M_unit={m_unit * f:g}", f"--nx={nx}", f"--ny={nx}"]
            if refine:
                a += [f"--nx_min={nx // 4}", f"--ny_min={nx // 4}", "--refine_abs=2e-2", "--refine_rel=1e-2"]
            out.append(ip.Params.from_args(a))
    return out


def bench_batched(ip, ctx, model, dump, args, world, stream, single_ms):
    """images/s of the batched forms: FP64, with the FP32 polarized step, and
    the mixed tier (FP32 step and FP32 fit shapes), beside the single-image
    FP64 rate of this run"""
    import torch
    nx = args.size
    ctx.upload_batch(model)
    res = {}
    ps = batch_params(ip, dump, args.m_unit, nx)
    for name, step32, fits32 in (("fp64", False, False), ("fp32_step", True, False), ("mixed", True, True)):
        ctx.set_step_precision(ip.IPG_STEP_FP32 if step32 else ip.IPG_STEP_FP64)
        ctx.set_fit_precision(ip.IPG_FITS_FP32 if fits32 else ip.IPG_FITS_FP64)
        ctx.set_record_precision(ip.IPG_RECORDS_MIXED if fits32 else ip.IPG_RECORDS_FP64)
        # untimed: the first two calls of a batch shape try both transfer
        # block sizes (the context's tuner), the timed ones use the faster
        for _ in range(2):
            ctx.render_batch(ps, model)
        torch.cuda.synchronize()
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = max(1, args.steps // 2)
        e0.record(stream)
        for _ in range(reps):
            imgs = ctx.render_batch(ps, model)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), world) / reps
        st = ctx.stats()
        res[name] = {"value": images_per_s(world, len(ps), ms), "unit": "images/s", "ms_per_batch": ms,
                     "instances": len(ps), "vs_single_fp64": (len(ps) / ms) / (1.0 / single_ms),
                     "geodesic_ms": st["geodesic_ms"], "coeffs_ms": st["coeffs_ms"],
                     "transfer_ms": st["transfer_ms"], "waves": st["waves"],
                     "long_class_items": st["long_class_items"]}
        if step32:
            ref = fp64_imgs
            errs = []
            for a, b in zip(imgs, ref):
                I0, I1 = b.pol[..., 0].sum(), a.pol[..., 0].sum()
                errs.append(abs(I1 / I0 - 1))
            res[name]["vs_fp64_Ftot_rel_max"] = float(max(errs))
        else:
            fp64_imgs = imgs
    ctx.set_step_precision(ip.IPG_STEP_FP64)
    ctx.set_fit_precision(ip.IPG_FITS_FP64)
    ctx.set_record_precision(ip.IPG_RECORDS_FP64)
    res["workload"] = (f"{len(ps)} instances of the bench image's camera ({nx}x{nx}, 230 GHz, thetacam 163): "
                       f"R_high {list(BATCH_RHIGH)} x M_unit {list(BATCH_MU)} x {args.m_unit:g}")
    if args.size == NX and not args.small:
        # the batched workload: 96 instances of mixed resolution, refined
        ps96 = []
        for fi, fq in enumerate(BATCH_FREQS):
            for ii, inc in enumerate(BATCH_INCL):
                ps96 += batch_params(ip, dump, args.m_unit, BATCH_RES[(fi + ii) % 3], inc, fq, refine=True)
        # FP64, then the mixed tier (FP32 step, FP32 fit shapes, compact
        # records); each timed on its second call (the first tunes the
        # transfer's block size for the batch's shape)
        for tag, mixed in (("workload_96", False), ("workload_96_mixed", True)):
            ctx.set_step_precision(ip.IPG_STEP_FP32 if mixed else ip.IPG_STEP_FP64)
            ctx.set_fit_precision(ip.IPG_FITS_FP32 if mixed else ip.IPG_FITS_FP64)
            ctx.set_record_precision(ip.IPG_RECORDS_MIXED if mixed else ip.IPG_RECORDS_FP64)
            ctx.render_batch(ps96, model)
            torch.cuda.synchronize()
            t = time.time()
            imgs = ctx.render_batch(ps96, model)
            torch.cuda.synchronize()
            sec = time.time() - t
            st = ctx.stats()
            pix = sum(int(i.traced) for i in imgs)
            res[tag] = {"value": len(ps96) / sec, "unit": "images/s", "seconds": sec,
                        "instances": len(ps96), "traced_pixels": pix, "ray_steps": st["ray_steps"],
                        "pixels_per_s": pix / sec,
                        "workload": "96 instances: {86,230,345} GHz x thetacam {17,60,120,163} x R_high "
                                    "{1,10,40,160} x M_unit {0.5,2} x base; 64/160/320 pixels a side per "
                                    "camera, refined from a quarter (refine_abs 2e-2, refine_rel 1e-2); "
                                    "host-timed call after one untimed call"
                                    + ("; mixed tier" if mixed else "; FP64")}
        ctx.set_step_precision(ip.IPG_STEP_FP64)
        ctx.set_fit_precision(ip.IPG_FITS_FP64)
        ctx.set_record_precision(ip.IPG_RECORDS_FP64)
    return res


def bench_adjoint(ip, ctx, model, p, args, world, stream):
    """one adjoint image (ipg_adjoint_params: its own forward trace, then the
    reverse walk) against one forward image of the same parameters"""
    import numpy as np
    import torch
    ctx.upload(model)
    img = ctx.render(p, model)
    scale = float(np.abs(img.pol[..., 0]).max())
    dL = img.pol[..., :4] / (scale * scale)  # the gradient of 0.5 sum (pol / scale)^2
    res = {}
    for K in (16, 64):
        ctx.adjoint_image(p, model, dL, ckpt=K)
        torch.cuda.synchronize()
        t0 = time.time()
        r = ctx.adjoint_image(p, model, dL, ckpt=K)
        torch.cuda.synchronize()
        res[f"K{K}_ms"] = (time.time() - t0) * 1e3
        st = ctx.stats()
        res[f"K{K}_device_ms"] = {k: st[f"{k}_ms"] for k in ("geodesic", "coeffs", "transfer", "adjoint", "adj_scatter",
                                                             "wall")}
        res[f"K{K}_waves"] = st["waves"]
        res[f"K{K}_nonfinite_cells"] = int(sum((~np.isfinite(r[k])).sum() for k in ("ne", "thetae", "b")))
    t0 = time.time()
    ctx.render(p, model)
    torch.cuda.synchronize()
    fwd_ms = (time.time() - t0) * 1e3
    res.update({"forward_image_ms": fwd_ms, "cost_vs_forward_K16": res["K16_ms"] / fwd_ms,
                "cost_vs_forward_K64": res["K64_ms"] / fwd_ms, "dL_dM_unit": r["M_unit"],
                "note": "host-timed calls through ipg_adjoint_params and ipg_render_image (both include their "
                        "host-side set-up and copies); the adjoint call includes its own forward trace"})
    return res


def run_leg(args):
    """One call of the batched or the adjoint leg at --size (a profiling case;
    no timing is printed)."""
    import numpy as np

    import ipole_b200 as ip
    dump = ensure_dump(SMALL_DUMP if args.small else DUMP)
    n = args.size
    p = ip.Params.from_args(workload_args(dump, n, n, args.m_unit))
    model = ip.Model.load(p)
    with ip.Context(0, pool_bytes=int(args.pool_gb * (1 << 30))) as ctx:
        if args.leg == "batched":
            ps = batch_params(ip, dump, args.m_unit, n)
            ctx.upload_batch(model)
            ctx.render_batch(ps, model)
        else:
            ctx.upload(model)
            img = ctx.render(p, model)
            scale = float(np.abs(img.pol[..., 0]).max())
            ctx.adjoint_image(p, model, img.pol[..., :4] / (scale * scale), ckpt=16)
        st = ctx.stats()
        print(json.dumps({"leg": args.leg, "size": n, "ray_steps": st["ray_steps"], "waves": st["waves"]}))
    return 0


def run_one_ray(args):
    """One ray alone on the GPU: the geodesic and transfer kernels' device time
    divided by its steps is the step latency of a lone lane, which bounds the
    sequential kernels for the longest rays of an image."""
    import numpy as np

    import ipole_b200 as ip
    os.environ["IPG_NO_SPLIT"] = "1"  # one wave, no length classes
    spec = SMALL_DUMP if args.small else DUMP
    dump = ensure_dump(spec)
    extra = [f"--eps={args.eps}"] if args.eps else []
    p = ip.Params.from_args(workload_args(dump, args.size, args.size, args.m_unit) + extra)
    model = ip.Model.load(p)
    i, j = (int(v) for v in args.ray.split(","))
    with ip.Context(0, pool_bytes=int((args.pool_gb or 2.0) * (1 << 30))) as ctx:
        ctx.upload(model)
        cam = ip.camera_for(p, model.grid)
        out = ctx.trace(cam, np.array([[i, j]], dtype=np.int32))
        s = ctx.stats()
    n = int(out["nstep"][0])
    print(json.dumps({"ray": [i, j], "nstep": n, "geodesic_ms": s["geodesic_ms"], "transfer_ms": s["transfer_ms"],
                      "geodesic_us_per_step": s["geodesic_ms"] * 1e3 / max(n, 1),
                      "transfer_us_per_step": s["transfer_ms"] * 1e3 / max(n, 1)}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--m-unit", dest="m_unit", type=float, default=M_UNIT)
    ap.add_argument("--size", type=int, default=NX, help="image side in pixels (400 for the headline)")
    ap.add_argument("--small", action="store_true", help="128x64x64 dump (profiling case)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--quick", action="store_true", help="device-resident timing only (no e2e / CPU / peak legs)")
    ap.add_argument("--eps", type=float, default=0.0,
                    help="geodesic step parameter for profiling cases (0: the workload's 0.01)")
    ap.add_argument("--ray", default="", help="I,J: trace this one pixel alone and report the step latency "
                                              "of the sequential kernels (diagnostic)")
    ap.add_argument("--pool-gb", dest="pool_gb", type=float, default=0.0,
                    help="trajectory pool size in GiB (0: 60%% of free device memory)")
    ap.add_argument("--records", default="fp64", choices=["fp64", "mixed"],
                    help="step-record storage between the kernels (ipg_set_record_precision); with --quick only")
    ap.add_argument("--step", default="fp64", choices=["fp64", "fp32"],
                    help="arithmetic of the polarized step (ipg_set_step_precision); with --quick only")
    ap.add_argument("--leg", default="", choices=["", "batched", "adjoint"],
                    help="run one call of that leg at --size and nothing else (profiling case): the batch of 8 "
                         "instances of the bench camera, or one adjoint image")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.ray:
        return run_one_ray(args)
    if args.leg:
        return run_leg(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
