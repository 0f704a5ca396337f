#!/usr/bin/env python3
"""Benchmark: MAP-EM iterations/s of positron-range correction at 128x128x159 68Ga.

Workload (the clinical configuration): a seeded torso phantom on a 128x128x159 grid of
0.776x0.776x0.795 mm voxels, isotope 68Ga, 128 far rays, support density 0.05, RDP beta 0.03 /
gamma 20, Biggs-Andrews acceleration on.  The measured data are the truth blurred by the
projector and Poisson-sampled at 5e7 counts.  One step = one complete 6-iteration MAP-EM
correction (initialisation included) of that volume.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Arms:
  ours       the CUDA engine through its C ABI (libprc_b200.so).  `value` is device-resident
             (data already in HBM); `e2e` times prc_em_run_host from pinned host buffers, with
             the host->device copy of the data and the device->host copy of the result inside.
  reference  the CPU restatement of the reference's algorithm (oracle/, rays re-marched every
             projection as prc.cu does), on all host cores, over a bounded sample of sources.
Both arms' `cpu_baseline` also times the reference's own CPU computation, the FP64 water-kernel
quadrature of its tests/reference.py (restated in oracle/kernel_oracle.py), single-threaded.

Multi-GPU (torchrun): every rank corrects its own frame (replicas, no collective on the data
path); value = iterations of all ranks / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import collections
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "EM iters/sec at 128x128x159 68Ga, learned vs plain projector, NRMSE<=1% vs FP64"
# The tracer's judge of the learned surrogate keeps a predicted far ray when its error norm is at
# most this multiple of the source's RMS ray norm (prc_create_surrogate's fallback_nrmse).
JUDGE_THRESHOLD = 0.45
ISOTOPE, RAYS, BETA, GAMMA, ITERS, SUPPORT_RHO, COUNTS = "68Ga", 128, 0.03, 20.0, 6, 0.05, 5e7
L2_BYTES = 126 * 2**20
REFERENCE_ARM_SECONDS = 150.0  # host seconds of projection the reference arm's timed steps share


def parse():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--grid", type=int, nargs=3, metavar=("NZ", "NY", "NX"), default=(159, 128, 128),
                    help="override the torso grid (profiling of smaller cases)")
    ap.add_argument("--iterations", type=int, default=ITERS)
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-forms", action="store_true", help="skip the per-form comparison")
    ap.add_argument("--no-oracle-check", action="store_true",
                    help="skip the FP64-oracle NRMSE of every form on a crop of the workload")
    ap.add_argument("--ops", type=int, default=0,
                    help="only run this many forward+adjoint pairs of the headline form (profiling)")
    ap.add_argument("--form", choices=("fp32", "fp24", "bf16", "traced"), default="fp32",
                    help="projector form of the headline number (default: plain fp32 stored field)")
    ap.add_argument("--workload", choices=("torso", "batch", "surrogate", "tiles", "frames"), default="torso",
                    help="batch: 32 dynamic-PET frames of mixed grids and isotopes, 10 iterations each; "
                         "surrogate: the learned surrogate's evaluation on the small phantom at 128x128x159; "
                         "tiles: projection and MAP-EM times of every source tile shape in both precisions; "
                         "frames: projections and MAP-EM of --frames frames sharing the torso's density map")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the comparison with the reference executable and the time-to-image leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-frames sub-record")
    ap.add_argument("--oracle-full", action="store_true",
                    help="also run the FP64 oracle on the whole volume (minutes on the host cores)")
    ap.add_argument("--tile", choices=("auto", "8x2x2", "16x2x1", "32x1x1", "4x4x2", "16x1x2"), default="auto",
                    help="source tile of the headline form's stored field (default: the autotuner's choice)")
    ap.add_argument("--frames", type=int, default=32)
    ap.add_argument("--surrogate", action="store_true", help="batch: learned surrogate where it applies")
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, flag in zip(names, f[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def aggregate(total_ms: float, steps: int, iterations: int, world: int, device=None) -> tuple[float, float]:
    """Whole-job throughput of the replicas: every rank corrected its own frame; the time is the
    maximum over ranks (an all-reduce MAX, the only collective), the units are all ranks'
    iterations.  Returns (max-over-ranks milliseconds, iterations per second)."""
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.tensor([total_ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    return total_ms, world * steps * iterations / (total_ms / 1e3)


def algorithmic_bytes(n_vox: int, n_active: int, deposits: int, weight_bytes: int = 4) -> dict:
    """Fixed byte accounting of the path (per projection and per MAP-EM iteration).

    A projection moves 12 B per source (active index, W_s, f_s or out_s) and per deposit one
    stored weight (4 B fp32, 2 B bf16) plus a 4 B target value.  An iteration adds the 74 B per
    voxel of the elementwise chain (extrapolate 12, clear 4, ratio 13, RDP update 13, sum 4,
    finish 16, two dots 12) to its two projections.  The compulsory figure is what an iteration
    moves when every volume and per-source array is touched once and no deposit costs traffic.
    """
    projection = 12 * n_active + (weight_bytes + 4) * deposits
    return {"projection": projection,
            "iteration": 74 * n_vox + 2 * projection,
            "compulsory": 74 * n_vox + 2 * 12 * n_active}


def workload_config(grid, iterations: int, world: int) -> dict:
    """The `config` both arms print: the workload, identical in the reference arm's line."""
    nz, ny, nx = grid
    return {"workload": f"torso {nx}x{ny}x{nz} at 0.776x0.776x0.795 mm, {ISOTOPE}, rays {RAYS}, beta {BETA}, "
                        f"gamma {GAMMA:g}, accel on, support rho {SUPPORT_RHO}, {iterations} MAP-EM iterations "
                        "per step",
            "iterations_per_step": iterations,
            "l2": "flushed (256 MB write) before every timed GPU step; every step also streams a multi-GB "
                  "coefficient field, far above the 126 MB L2",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}


def make_workload(grid):
    from prc_mlem_b200 import phantoms
    rho, truth, spacing = phantoms.torso_phantom(seed=2, shape=tuple(grid))
    return rho, truth, spacing


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.is_file():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


FORMS = {"fp32": (2, 0), "fp24": (2, 3), "bf16": (2, 1), "traced": (1, 0)}  # (PRC_CACHE_*, PRC_PRECISION_*)
WEIGHT_BYTES = {"fp32": 4, "fp24": 3, "bf16": 2, "traced": 4}


def ncu_traffic(kernel_key: str, stored_bytes: float):
    """Per-launch DRAM bytes of the headline kernel, from the committed ncu summary.

    The capture runs on a smaller torso (the full workload holds too much memory for a
    multi-pass capture); its DRAM bytes per stored field byte are scaled to this run's field."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    if not p.is_file():
        return None
    try:
        entry = json.loads(p.read_text()).get(kernel_key)
    except (ValueError, OSError):
        return None
    if not entry:
        return None
    return int(entry["dram_bytes"] / entry["stored_bytes"] * stored_bytes)


# ------------------------------------------------------------------------------- our arm
def run_ours(args):
    import torch
    import prc_mlem_b200 as pm
    from prc_mlem_b200 import phantoms

    world, rank, local = dist_env()
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()

    rho, truth, spacing = make_workload(args.grid)
    cache, prec = FORMS[args.form]
    tune_s = None
    if args.tile == "auto" and not args.ops:  # the autotuner's choice for this configuration
        t0 = time.perf_counter()
        pm.tune_tile(ISOTOPE, rho, spacing, rays=RAYS, support_rho=SUPPORT_RHO, cache=cache, precision=prec)
        if prec == pm.PRC_PRECISION_FP32:  # the bf16 forms of the comparison use their own choice
            pm.tune_tile(ISOTOPE, rho, spacing, rays=RAYS, support_rho=SUPPORT_RHO, cache=cache,
                         precision=pm.PRC_PRECISION_BF16)
        tune_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    tile = {"auto": pm.PRC_TILE_AUTO, "8x2x2": pm.PRC_TILE_8x2x2, "16x2x1": pm.PRC_TILE_16x2x1,
            "32x1x1": pm.PRC_TILE_32x1x1, "4x4x2": pm.PRC_TILE_4x4x2, "16x1x2": pm.PRC_TILE_16x1x2}[args.tile]
    P = pm.Projector(ISOTOPE, rho, spacing, rays=RAYS, support_rho=SUPPORT_RHO, cache=cache, precision=prec, tile=tile)
    P.synchronize()
    setup_s = time.perf_counter() - t0
    stream = torch.cuda.ExternalStream(P.stream)
    # (profiling runs with --ops make their data with the engine: no second process under ncu)
    g_host, data_how, data_sha = measured_data(rho, truth, spacing, P, use_reference=world == 1 and not args.ops)
    d_g = torch.from_numpy(g_host).cuda()
    d_out = torch.empty_like(d_g)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def l2_flush():
        with torch.cuda.stream(stream):
            flush.fill_(1.0)

    if args.ops:  # profiling mode: a few operator pairs only
        for _ in range(args.ops):
            P.forward(d_g, d_out)
            P.adjoint(d_g, d_out)
        P.synchronize()
        print(json.dumps({"ops": args.ops, "n_active": P.n_active, "cache": P.cache_mode}))
        return

    for _ in range(args.warmup):
        P.correct(d_g, d_out, args.iterations, BETA, GAMMA, True)
    barrier()

    clocks = ClockSampler(dev)
    clocks.start()
    times = []
    barrier()
    P.timing(True)  # CUDA events around every projection launch of the timed steps
    launches0 = P.launches
    for _ in range(args.steps):
        l2_flush()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        P.correct(d_g, d_out, args.iterations, BETA, GAMMA, True)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    barrier()
    launches_timed = P.launches - launches0  # this handle's kernels inside the timed region
    P.timing(False)
    in_region = P.timing_read()
    clock_info = clocks.stop()
    total_ms, value = aggregate(sum(times), args.steps, args.iterations, world, device="cuda")
    iters_total = world * args.steps * args.iterations

    # end to end through the public API from pinned host buffers
    g_pin = torch.from_numpy(g_host).pin_memory()
    out_pin = torch.empty_like(g_pin).pin_memory()
    e2e_ms = []
    for i in range(args.warmup + args.steps):
        l2_flush()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rc = pm.lib().prc_em_run_host(P._h, g_pin.data_ptr(), out_pin.data_ptr(), args.iterations, BETA, GAMMA, 1)
        e1.record(stream)
        e1.synchronize()
        if rc != 0:
            raise RuntimeError(pm.lib().prc_last_error().decode())
        if i >= args.warmup:
            e2e_ms.append(e0.elapsed_time(e1))
    e2e_total, e2e_value = aggregate(sum(e2e_ms), args.steps, args.iterations, world, device="cuda")
    corrected = out_pin.numpy().copy()

    # dominant kernel: its mean launch time inside the timed steps (events around each launch),
    # and single launches timed alone for comparison
    n_active = P.n_active
    deposits = P.count_deposits()
    region_ms = {"forward": in_region["forward_ms"] / max(in_region["forward_launches"], 1),
                 "adjoint": in_region["adjoint_ms"] / max(in_region["adjoint_launches"], 1)}
    launch_ms = {}
    for name, fn in (("forward", P.forward), ("adjoint", P.adjoint)):
        ts = []
        for i in range(8):
            l2_flush()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn(d_g, d_out)
            e1.record(stream)
            e1.synchronize()
            if i >= 2:
                ts.append(e0.elapsed_time(e1))
        launch_ms[name] = statistics.mean(ts)
    top = max(region_ms, key=region_ms.get)
    nz, ny, nx = args.grid
    n_vox = nx * ny * nz
    acct = algorithmic_bytes(n_vox, n_active, deposits, weight_bytes=WEIGHT_BYTES[args.form])
    alg_bytes = acct["projection"]
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (region_ms[top] / 1e3) / 1e9
    iter_s = total_ms / (args.steps * args.iterations) / 1e3
    iteration = {"algorithmic_bytes": acct["iteration"],
                 "achieved": round(acct["iteration"] / iter_s / 1e9, 1),
                 "frac": round(acct["iteration"] / iter_s / 1e9 / peak, 4),
                 "compulsory_bytes": acct["compulsory"],
                 "compulsory_gbs": round(acct["compulsory"] / iter_s / 1e9, 1)}
    projection_share = (in_region["forward_ms"] + in_region["adjoint_ms"]) / sum(times)
    mode, far_entries, far_t_entries = P.cache_mode
    elem = WEIGHT_BYTES[args.form]
    stored_bytes = (far_t_entries if top == "forward" else far_entries) * elem
    traffic = ncu_traffic(f"{top}_{args.form}", stored_bytes) if mode == 2 else None

    # the single-GPU line also carries the per-form comparison, the parity with the reference
    # executable, the time to a corrected image, the CPU baseline, the FP64-oracle check, the
    # batch sub-record and the image quality; a multi-GPU run reports its timing only
    single = world == 1
    quality = image_quality(truth, g_host, corrected) if single else None
    forms = images = None
    if not args.no_forms and single:
        forms, images = compare_forms(args, rho, spacing, d_g, stream, l2_flush, value, corrected, P)
    parity = tti = None
    if single and not args.no_parity:
        parity, ref_job = parity_vs_prc_cu(P, rho, spacing, g_host, corrected, images or {}, args.iterations)
        tti = time_to_image(rho, spacing, g_host, args, ref_job)
        tti["command_line"] = cli_vs_prc_cu(rho, spacing, g_host, args.iterations)
    batch = None
    if single and not args.no_batch:
        batch = batch_record(frames=8, iterations=10, steps=2, warmup=1)
    shared = study = None
    if single and not args.no_batch and args.form != "traced":
        shared = shared_frames_record(P, truth, g_host, stream, l2_flush, args.iterations, value, corrected)
        if args.form == "fp32":
            study = study_batch_record(rho, truth, spacing, args.iterations, value)

    if world > 1:
        torch.distributed.barrier()
    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    cpu = None if args.no_cpu_baseline or not single else cpu_baseline(rho, spacing, g_host, sample_seconds=15.0)
    check = None if args.no_oracle_check or not single else oracle_check(rho, spacing, g_host, args)
    if check and args.oracle_full:
        check["full_volume"] = oracle_full_volume(rho, spacing, g_host, args, corrected, images or {})
    dram_frac = None
    if traffic:
        dram_frac = round(traffic / (region_ms[top] / 1e3) / 1e9 / peak, 4)
    line = {
        "metric": METRIC,
        "value": round(value, 3),
        "unit": "EM iters/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(total_ms / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": {"bf16": "bf16 (stored weights; f32 accumulation, f64 sums)",
                  "fp24": "f32 (24-bit stored weights; f32 accumulation, f64 sums)"}.get(args.form, "f32"),
        "data": data_how,
        "data_sha256": data_sha,
        "config": workload_config(args.grid, args.iterations, world),
        "details": {
            "form": {"fp32": "fp32 stored coefficient field (near block + far rays), the reference's numerics",
                     "bf16": "mixed precision: bf16 stored coefficient field, fp32 accumulation, fp64 sums",
                     "traced": "plain ray-traced projector: near cache + far rays re-marched every projection"}[
                         args.form],
            "n_active": n_active,
            "deposits_per_projection": deposits,
            "field_entries": {"source_major": far_entries, "target_major": far_t_entries},
            "voxels_per_s": round(value * n_vox, 1),
            "device_gb": round(P.device_bytes / 1e9, 2),
            "tile": "x".join(str(v) for v in pm.TILE_SHAPES.get(P.tile, (0, 0, 0))),
            "tile_tuning_s": None if tune_s is None else round(tune_s, 3),
            "first_handle_setup_s": round(setup_s, 4),
        },
        "e2e": {"value": round(e2e_value, 3), "unit": "EM iters/s",
                "h2d_bytes_per_step": int(g_host.nbytes), "d2h_bytes_per_step": int(g_host.nbytes)},
        "roofline": {"bound": "hbm", "kernel": f"project_kernel {top} ({args.form} form)",
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                     "traffic": traffic,
                     # measured DRAM bytes of the launch over its in-region time: the HBM fraction
                     # (the fixed accounting above charges 4 B per gathered target value, which
                     # the kernel reads from L1/L2, so `frac` can exceed 1)
                     "dram_frac": dram_frac,
                     "launch_ms": {k: round(v, 4) for k, v in region_ms.items()},
                     "launch_ms_alone": {k: round(v, 4) for k, v in launch_ms.items()},
                     "launches_timed": in_region["forward_launches"] + in_region["adjoint_launches"],
                     "projection_share_of_steps": round(projection_share, 4),
                     "algorithmic_bytes": alg_bytes,
                     # the whole MAP-EM iteration (both projections and the elementwise chain)
                     # over the mean iteration time of the timed steps
                     "iteration": iteration},
        "gpu_launches": launches_timed,
        "clocks": clock_info,
    }
    if parity:
        line["parity_vs_prc_cu"] = parity
    if tti:
        line["time_to_image"] = tti
    if forms:
        line["forms"] = forms
        line["targets"] = targets(forms, check)
    if quality:
        line["image_quality"] = quality
    if cpu:
        line["cpu_baseline"] = cpu
    if check:
        line["fp64_oracle_check"] = check
    if batch:
        line["batch"] = batch
    if shared:
        line["shared_density_frames"] = shared
    if study:
        line["study_batch"] = study
    print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


def nrmse(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2)))


def compare_forms(args, rho, spacing, d_g, stream, l2_flush, value_fp32, corrected_fp32, P_fp32):
    """EM iters/s of the other projector forms on the same data, and their agreement.  Returns
    (per-form record, per-form corrected image)."""
    import torch
    import prc_mlem_b200 as pm
    from prc_mlem_b200 import surrogate as sg
    out = {"fp32_field": {"iters_per_s": round(value_fp32, 3)}}
    images = {"fp32_field": corrected_fp32}
    for name, kw in projector_forms(pm, sg, sg.load_trained()):
        t_setup = time.perf_counter()
        Q = pm.Projector(ISOTOPE, rho, spacing, rays=RAYS, support_rho=SUPPORT_RHO, **kw)
        Q.synchronize()
        t_setup = time.perf_counter() - t_setup
        s = torch.cuda.ExternalStream(Q.stream)
        d_out = torch.empty_like(d_g)
        steps = max(1, min(args.steps, 3))
        Q.correct(d_g, d_out, args.iterations, BETA, GAMMA, True)
        Q.synchronize()
        ts = []
        for _ in range(steps):
            l2_flush()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            Q.correct(d_g, d_out, args.iterations, BETA, GAMMA, True)
            e1.record(s)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        v = args.iterations * steps / (sum(ts) / 1e3)
        img = d_out.cpu().numpy()
        images[name] = img
        out[name] = {"iters_per_s": round(v, 3), "nrmse_vs_fp32_field": nrmse(img, corrected_fp32),
                     "device_gb": round(Q.device_bytes / 1e9, 3), "setup_s": round(t_setup, 3)}
        if "surrogate" in kw:
            out[name]["exact_fallback_share"] = round(Q.fallbacks / (Q.n_active * RAYS), 4)
        Q.close()
    return out, images


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def parity_vs_prc_cu(P, rho, spacing, g, corrected, images, iterations):
    """The headline data run through the reference executable (prc.cu built for sm_100a, on the
    same GPU, outside the timed region): relative L2 of one forward and one adjoint projection
    of the measured data and of every form's corrected image against the reference's, on the
    full volume.  Returns (record, the reference's whole-job times)."""
    from oracle import ref_exe
    if not ref_exe.available():
        return {"unavailable": "oracle/_ref/prc was not built (needs the reference source)"}, None
    nz, ny, nx = rho.shape
    sp = spacing
    opts = ("--rays", str(RAYS), "--support-rho", str(SUPPORT_RHO))
    em = ref_exe.run("correct", ISOTOPE, g, rho, sp, *opts, "--iterations", str(iterations), "--beta", str(BETA),
                     "--gamma", str(GAMMA))
    fwd = ref_exe.run("forward", ISOTOPE, g, rho, sp, *opts)
    adj = ref_exe.run("adjoint", ISOTOPE, g, rho, sp, *opts)
    support = np.maximum(rho, np.float32(1e-3)) >= np.float32(SUPPORT_RHO)
    g_in = np.where(support, g, 0.0).astype(np.float32)
    out = {"what": f"relative L2 against prc.cu (sm_100a build) on the same {nx}x{ny}x{nz} data, full volume",
           "forward_fp32_field": rel_l2(P.forward_host(g_in), fwd["out"]),
           "adjoint_fp32_field": rel_l2(P.adjoint_host(g_in), adj["out"]),
           "corrected": {name: rel_l2(img, em["out"]) for name, img in ({"fp32_field": corrected} | images).items()},
           "tolerance_fp32": 1e-5}
    job = {"setup_s": em["setup_s"], "iterations_s": em["iterations_s"], "total_s": em["total_s"],
           "process_wall_s": round(em["wall_s"], 3)}
    return out, job


def cli_vs_prc_cu(rho, spacing, g, iterations):
    """The drop-in command line end to end on the headline data: this engine's `prc` executable
    and the reference executable with the same arguments (--mode correct, 128 rays, beta 0.03,
    gamma 20, support density 0.05, acceleration on), each a fresh process that reads the raw
    files, creates its CUDA context, builds the projector, iterates and writes the image.
    Reports each process's wall time and the total it prints (prc.cu:719-720), and the relative
    L2 distance of the two output images."""
    import tempfile
    from oracle import ref_exe
    import prc_mlem_b200 as pm
    if not (ref_exe.available() and pm.CLI_PATH.is_file()):
        return {"unavailable": "the reference executable or the prc command line was not built"}
    nz, ny, nx = rho.shape
    out = {}
    with tempfile.TemporaryDirectory(prefix="prc_cli_bench_") as d:
        d = Path(d)
        np.ascontiguousarray(rho, np.float32).tofile(d / "rho.raw")
        np.ascontiguousarray(g, np.float32).tofile(d / "g.raw")
        images = {}
        for name, exe in (("prc_cli", pm.CLI_PATH), ("prc_cu", ref_exe.EXE)):
            cmd = [str(exe), ISOTOPE, str(nx), str(ny), str(nz), *(repr(float(s)) for s in spacing), "--input",
                   str(d / "g.raw"), "--density", str(d / "rho.raw"), "--output", str(d / f"{name}.raw"), "--rays",
                   str(RAYS), "--iterations", str(iterations), "--beta", str(BETA), "--gamma", str(GAMMA),
                   "--support-rho", str(SUPPORT_RHO)]
            walls = []
            for _ in range(2):  # the second run sees warm file caches
                t0 = time.perf_counter()
                r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
                walls.append(time.perf_counter() - t0)
                if r.returncode != 0:
                    return {"unavailable": f"{name} failed: {r.stderr.strip()[:200]}"}
            import re
            total = re.search(r"total ([0-9.]+) s", r.stdout)
            norm = re.search(r"normalisation [^:]*: ([0-9.]+) s", r.stdout)
            out[name] = {"process_wall_s": round(min(walls), 3), "printed_total_s": float(total.group(1)) if total else None,
                         "printed_setup_s": float(norm.group(1)) if norm else None}
            images[name] = np.fromfile(d / f"{name}.raw", np.float32)
        out["speedup_process_wall"] = round(out["prc_cu"]["process_wall_s"] / out["prc_cli"]["process_wall_s"], 2)
        out["output_rel_l2"] = rel_l2(images["prc_cli"], images["prc_cu"])
    return out


def time_to_image(rho, spacing, g, args, ref_job):
    """Seconds from density and data in host memory to the corrected image in host memory, for
    a fresh handle in a warm CUDA context (library loaded, context created): prc_create (host
    clamp and source order, uploads, layout, normalisation, both field copies) plus
    prc_em_run_host (upload, the MAP-EM iterations, download).  Beside it the reference
    executable's whole job on the same data: its normalisation plus its iterations, by its own
    clock, and its total (which also counts reading the files and creating its CUDA context).
    Each form runs three times; the run of median total time is reported, with every total."""
    import prc_mlem_b200 as pm
    out = {}
    for name, kw in (("fp32_field", dict(cache=pm.PRC_CACHE_FULL)),
                     ("bf16_field", dict(cache=pm.PRC_CACHE_FULL, precision=pm.PRC_PRECISION_BF16))):
        runs = []
        for _ in range(3):
            t0 = time.perf_counter()
            Q = pm.Projector(ISOTOPE, rho, spacing, rays=RAYS, support_rho=SUPPORT_RHO, **kw)
            t1 = time.perf_counter()
            Q.correct_host(g, args.iterations, BETA, GAMMA, True)
            t2 = time.perf_counter()
            Q.close()
            runs.append({"seconds": round(t2 - t0, 4), "setup_s": round(t1 - t0, 4), "iterations_s": round(t2 - t1, 4)})
        runs.sort(key=lambda r: r["seconds"])
        out[name] = dict(runs[1], all_seconds=[r["seconds"] for r in runs])
    if ref_job and ref_job.get("setup_s") is not None:
        ref_s = ref_job["setup_s"] + ref_job["iterations_s"]
        out["prc_cu"] = dict(ref_job, seconds=round(ref_s, 3),
                             note="setup + iterations from its 2-decimal clock (prc.cu:644, 719-720)")
        out["speedup_fp32_field"] = round(ref_s / out["fp32_field"]["seconds"], 2)
        out["speedup_bf16_field"] = round(ref_s / out["bf16_field"]["seconds"], 2)
    return out


def targets(forms, check):
    """Every form's EM iterations/s as a multiple of the plain ray-traced projector (the
    reference's algorithm: near block cached, far rays re-marched every projection) and of the
    fp32 stored field, beside its FP64-oracle NRMSE.  "plain" always means the traced form."""
    traced = forms.get("traced", {}).get("iters_per_s")
    fp32 = forms["fp32_field"]["iters_per_s"]
    fp64 = (check or {}).get("forms", {})
    out = {"plain": "traced: the reference's algorithm on B200 (near cache, far rays re-marched)"}
    for name, f in forms.items():
        v = f["iters_per_s"]
        out[name] = {"iters_per_s": v,
                     "x_plain_traced": round(v / traced, 3) if traced else None,
                     "x_fp32_field": round(v / fp32, 3),
                     "nrmse_vs_fp64": fp64.get(name, {}).get("nrmse_vs_fp64")}
    return out


def image_quality(truth, measured, corrected):
    """What the correction gains, scored on the device against the known truth with the
    reference's metrics (prc_mlem_b200.evaluate): the measured data and the corrected image,
    both scaled by sum(truth) / sum(measured) into the truth's activity units."""
    from prc_mlem_b200 import evaluate
    ev = evaluate.Evaluator(truth)
    scale = float(truth.sum(dtype=np.float64) / measured.sum(dtype=np.float64))
    keys = ("nrmse", "ssim", "ssim_edge", "edge_nrmse", "rc_hot", "rc_min", "bg_cov", "ring", "halo")
    out = {"scaling": "both images x sum(truth) / sum(measured)",
           "hot_regions": ev.metric_settings["hot_region_count"]}
    for name, img in (("measured", measured), ("corrected", corrected)):
        m = ev(img.astype(np.float64) * scale)
        out[name] = {k: (None if m[k] is None else round(m[k], 5)) for k in keys}
    ev.close()
    return out


def projector_forms(pm, sg, net):
    """The projector forms compared with the headline fp32 field: (name, Projector keywords)."""
    forms = [("fp24_field", dict(cache=pm.PRC_CACHE_FULL, precision=pm.PRC_PRECISION_FP24)),
             ("bf16_field", dict(cache=pm.PRC_CACHE_FULL, precision=pm.PRC_PRECISION_BF16)),
             ("bf16_volumes", dict(cache=pm.PRC_CACHE_FULL, precision=pm.PRC_PRECISION_BF16_VOLUMES)),
             ("traced", dict(cache=pm.PRC_CACHE_NEAR, precision=pm.PRC_PRECISION_FP32)),
             ("radial_traced_bf16", dict(precision=pm.PRC_PRECISION_BF16, surrogate="traced"))]
    if net is not None:
        forms += [("learned_bf16", dict(precision=pm.PRC_PRECISION_BF16, surrogate=net,
                                        target_scale=sg.TARGET_SCALE)),
                  ("learned_judged_bf16", dict(precision=pm.PRC_PRECISION_BF16, surrogate=net,
                                               target_scale=sg.TARGET_SCALE, fallback_nrmse=JUDGE_THRESHOLD))]
    return forms


def oracle_check(rho, spacing, g, args):
    """Every projector form against the FP64 oracle (the CPU restatement of prc.cu with doubles
    throughout) on a central 64x48x32 crop of the workload: NRMSE of the corrected image after
    the benchmark's MAP-EM run, and the forward/adjoint identity residual
    |<Ax, y> - <x, A^T y>| / |<Ax, y>| on seeded random volumes."""
    import torch
    import prc_mlem_b200 as pm
    from prc_mlem_b200 import surrogate as sg
    from oracle import oracle
    nz, ny, nx = rho.shape
    cz, cy, cx = nz // 2, ny // 2, nx // 2
    sl = (slice(max(cz - 16, 0), cz + 16), slice(max(cy - 24, 0), cy + 24), slice(max(cx - 32, 0), cx + 32))
    rc, gc = np.ascontiguousarray(rho[sl]), np.ascontiguousarray(g[sl], dtype=np.float32)
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    O = oracle.Problem(ISOTOPE, rc, spacing, rays=RAYS, support_rho=SUPPORT_RHO, precision=64, threads=threads)
    O.normalize()
    ref = O.correct(gc, args.iterations, BETA, GAMMA, True)
    t_oracle = time.perf_counter() - t0
    rng = np.random.default_rng(3)
    support = np.maximum(rc, 1e-3) >= SUPPORT_RHO
    x = np.where(support, rng.random(rc.shape), 0.0).astype(np.float32)
    y = rng.random(rc.shape).astype(np.float32)
    forms = [("fp32_field", dict(cache=pm.PRC_CACHE_FULL, precision=pm.PRC_PRECISION_FP32))]
    forms += projector_forms(pm, sg, sg.load_trained())
    d_g = torch.from_numpy(gc).cuda()
    out = {}
    for name, kw in forms:
        Q = pm.Projector(ISOTOPE, rc, spacing, rays=RAYS, support_rho=SUPPORT_RHO, **kw)
        d_out = torch.empty_like(d_g)
        Q.correct(d_g, d_out, args.iterations, BETA, GAMMA, True)
        Q.synchronize()
        ax, aty = Q.forward_host(x).astype(np.float64), Q.adjoint_host(y).astype(np.float64)
        lhs = float(np.sum(ax * y))
        rhs = float(np.sum(np.where(support, aty, 0.0) * x))
        out[name] = {"nrmse_vs_fp64": nrmse(d_out.cpu().numpy(), ref),
                     "identity_residual": abs(lhs - rhs) / abs(lhs)}
        Q.close()
    return {"crop": f"{rc.shape[2]}x{rc.shape[1]}x{rc.shape[0]} voxels at the volume centre "
                    f"({int(support.sum())} tissue voxels)",
            "oracle_seconds": round(t_oracle, 1), "oracle_threads": threads, "forms": out}


def oracle_full_volume(rho, spacing, g, args, corrected, images):
    """The FP64 oracle's corrected image of the whole volume (minutes on all host cores) and the
    NRMSE of every form's full-volume corrected image against it."""
    from oracle import oracle
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    O = oracle.Problem(ISOTOPE, rho, spacing, rays=RAYS, support_rho=SUPPORT_RHO, precision=64, threads=threads)
    O.normalize()
    ref = O.correct(np.ascontiguousarray(g, np.float32), args.iterations, BETA, GAMMA, True)
    dt = time.perf_counter() - t0
    forms = {"fp32_field": corrected} | images
    return {"oracle_seconds": round(dt, 1), "oracle_threads": threads,
            "nrmse_vs_fp64": {name: nrmse(img, ref) for name, img in forms.items()}}


# ------------------------------------------------------------------------------- CPU baseline
def cpu_baseline(rho, spacing, g, sample_seconds=15.0, seed=7, extras=True):
    """The oracle's float restatement of prc.cu (near block cached, far rays re-marched each
    projection, as the reference does) on all host cores, over a random sample of sources.
    iters/s = 1 / (forward + adjoint time scaled to all sources + one RDP update).  With
    ``extras`` the record also times the reference's own CPU quadrature and the FP64
    restatement on the small configuration."""
    sys.path.insert(0, str(ROOT))
    from oracle import oracle
    threads = os.cpu_count() or 1
    full = oracle.Problem(ISOTOPE, rho, spacing, rays=RAYS, support_rho=SUPPORT_RHO, precision=32, threads=threads)
    n_active = full.n_active
    rng = np.random.default_rng(seed)
    frac = 0.002
    while True:
        sample = np.sort(rng.choice(n_active, size=max(64, int(n_active * frac)), replace=False))
        sub = oracle.Problem(ISOTOPE, rho, spacing, rays=RAYS, support_rho=SUPPORT_RHO, precision=32,
                             threads=threads)
        sub.active = np.ascontiguousarray(full.active[sample])
        sub.normalize()
        x = g.astype(np.float32)
        t0 = time.perf_counter()
        sub.forward(x)
        sub.adjoint(x)
        dt = time.perf_counter() - t0
        if dt >= 0.5 * sample_seconds or frac >= 1.0:
            break
        frac = min(1.0, frac * max(2.0, 0.6 * sample_seconds / max(dt, 1e-3)))
    t0 = time.perf_counter()
    full.update(g, g, BETA, GAMMA, 1e-6)
    t_update = time.perf_counter() - t0
    per_iter = dt * n_active / len(sample) + t_update
    info = {"value": round(1.0 / per_iter, 5), "unit": "EM iters/s", "cores": threads, "kind": "port",
            "sample": f"{len(sample)} of {n_active} sources ({100 * len(sample) / n_active:.2f}%): one forward "
                      f"and one adjoint projection ({dt:.1f} s), scaled to all sources, plus one full RDP "
                      f"update ({t_update:.2f} s)"}
    if extras:
        info["reference_quadrature"] = reference_quadrature()
        info["small_configuration_fp64"] = small_configuration_fp64(threads)
    return info


def small_configuration_fp64(threads: int) -> dict:
    """The FP64 restatement of prc.cu run end to end on the small configuration the reference's
    own CPU-runnable case uses: 32x32x24 at 2 mm, 18F, 32 rays; the truth blurred by the
    projector and Poisson-sampled at 1e6 counts, then --mode forward, --mode adjoint and
    --mode correct with beta 0, no acceleration, 4 iterations (each with its own setup)."""
    sys.path.insert(0, str(ROOT))
    from oracle import oracle
    from prc_mlem_b200 import phantoms
    rho, truth, spacing = phantoms.small_phantom(seed=1)
    t0 = time.perf_counter()
    P = oracle.Problem("18F", rho, spacing, rays=32, precision=64, threads=threads)
    g = phantoms.poisson_counts(P.forward(truth.astype(np.float64)).astype(np.float32), 1e6, seed=1)
    t_data = time.perf_counter() - t0
    t0 = time.perf_counter()
    for mode in ("forward", "adjoint", "correct"):
        Q = oracle.Problem("18F", rho, spacing, rays=32, precision=64, threads=threads)
        x = Q.clamp_input(g).astype(np.float64)
        if mode == "forward":
            Q.forward(x)
        elif mode == "adjoint":
            Q.adjoint(x)
        else:
            Q.correct(g, 4, beta=0.0, accelerate=False)
    return {"seconds": round(time.perf_counter() - t0, 4), "cores": threads, "kind": "port",
            "case": "32x32x24 at 2 mm, 18F, rays 32, 1e6 counts: forward, adjoint and 4 RL iterations "
                    f"(beta 0, no acceleration) in FP64, each with its own setup; data made in {t_data:.2f} s"}


def reference_quadrature(repeats=3):
    """The reference's own CPU computation (the FP64 homogeneous water-kernel quadrature of its
    tests/reference.py, restated in oracle/kernel_oracle.py): the 68Ga kernel at 2 mm voxels,
    half-width 6, 600 shells x 1000 directions, single-threaded NumPy; median of ``repeats``."""
    sys.path.insert(0, str(ROOT))
    from oracle import kernel_oracle
    branches = kernel_oracle.table_branches(ISOTOPE)
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        k = kernel_oracle.water_kernel(branches, (2.0, 2.0, 2.0), 6)
        times.append(time.perf_counter() - t0)
    return {"seconds": round(statistics.median(times), 4), "cores": 1, "kind": "port",
            "case": f"{ISOTOPE} water kernel, 2 mm voxels, half-width 6, 600 shells x 1000 directions "
                    f"(mass inside the box {k.sum():.6f})"}


def run_reference(args):
    """The reference's algorithm on the host cores (the oracle's float restatement of prc.cu:
    near block cached, far rays re-marched every projection), with the reference executable on
    the same GPU beside it.  Every timed step is one forward and one adjoint projection over a
    fixed random half of the sources (fewer only when many steps would exceed the arm's time
    budget), scaled to all
    sources, plus one full RDP update; the normalisation pass is timed once on that half and
    reported, scaled to all sources, as the setup.  Warm-up steps run 4 % of the half."""
    world, rank, _ = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT))
    from oracle import oracle
    rho, truth, spacing = make_workload(args.grid)
    g, data_how, data_sha = measured_data(rho, truth, spacing)
    threads = os.cpu_count() or 1
    full = oracle.Problem(ISOTOPE, rho, spacing, rays=RAYS, support_rho=SUPPORT_RHO, precision=32, threads=threads)
    n_active = full.n_active
    x = g.astype(np.float32)
    t0 = time.perf_counter()
    full.update(g, g, BETA, GAMMA, 1e-6)
    t_update = time.perf_counter() - t0

    # one fixed random half of the sources, normalised once (timed: the setup, scaled to all)
    rng = np.random.default_rng(101)
    half = np.sort(rng.choice(n_active, size=max(64, n_active // 2), replace=False))
    base = oracle.Problem(ISOTOPE, rho, spacing, rays=RAYS, support_rho=SUPPORT_RHO, precision=32, threads=threads)
    base.active = np.ascontiguousarray(full.active[half])
    t0 = time.perf_counter()
    base.normalize()
    setup_s = (time.perf_counter() - t0) * n_active / len(half)

    def step(frac, seed):
        """One forward and one adjoint projection over `frac` of the normalised half."""
        pick = np.arange(len(half))
        if frac < 1.0:
            pick = np.sort(np.random.default_rng(seed).choice(len(half), size=max(64, int(len(half) * frac)),
                                                              replace=False))
        sub = oracle.Problem(ISOTOPE, rho, spacing, rays=RAYS, support_rho=SUPPORT_RHO, precision=32,
                             threads=threads)
        sub.active = np.ascontiguousarray(base.active[pick])
        sub.W, sub.near = np.ascontiguousarray(base.W[pick]), np.ascontiguousarray(base.near[pick])
        t0 = time.perf_counter()
        sub.forward(x)
        sub.adjoint(x)
        spent = time.perf_counter() - t0
        return len(pick), spent * n_active / len(pick), spent

    for i in range(args.warmup):
        step(0.04, 11 + i)
    budget = REFERENCE_ARM_SECONDS  # host seconds of projection the timed steps may take together
    frac, vals, fracs = 1.0, [], []
    for i in range(args.steps):
        n_sample, pair_s, spent = step(frac, 1001 + i)
        vals.append(1.0 / (pair_s + t_update))
        fracs.append(n_sample / n_active)
        budget -= spent
        left = args.steps - i - 1
        if left and budget < left * spent:  # keep the arm within a few minutes for any --steps
            frac = max(0.1, frac * max(budget, 0.0) / (left * spent))
    value = statistics.mean(vals)
    per_iter = 1.0 / value
    info = {"value": round(value, 5), "unit": "EM iters/s", "cores": threads, "kind": "port",
            "sample": f"per step one forward and one adjoint projection over a random {100 * min(fracs):.0f}-"
                      f"{100 * max(fracs):.0f}% of the {n_active} sources, scaled to all sources, plus one full "
                      f"RDP update ({t_update:.2f} s); {args.steps} steps",
            "setup_s": round(setup_s, 2),
            "time_to_image_s": round(setup_s + args.iterations * per_iter, 2),
            "reference_quadrature": reference_quadrature(),
            "small_configuration_fp64": small_configuration_fp64(threads)}
    line = {
        "metric": METRIC, "impl": "reference", "value": round(value, 5), "unit": "EM iters/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": data_how,
        "data_sha256": data_sha,
        "config": workload_config(args.grid, args.iterations, world),
        "cpu_baseline": info,
        "e2e": {"value": round(value, 5), "unit": "EM iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_gpu": reference_gpu(rho, spacing, g, args.iterations),
    }
    print(json.dumps(line))


def reference_gpu(rho, spacing, g, iterations: int, rate_iterations: int = 60):
    """The reference executable itself (prc.cu compiled for sm_100a by oracle/build_ref.sh) on
    the same workload: the whole job of `iterations` MAP-EM iterations (normalisation plus
    iterations, by its own clock, and its total), and its iteration rate from a run of
    `rate_iterations` (its clock prints 2 decimals, so a short run cannot give the rate)."""
    sys.path.insert(0, str(ROOT))
    from oracle import ref_exe
    if not ref_exe.available():
        return {"unavailable": "oracle/_ref/prc was not built (needs the reference source)"}
    try:
        import torch
        if not torch.cuda.is_available():
            return {"unavailable": "no CUDA device"}
    except Exception:
        return {"unavailable": "no CUDA device"}
    sp = spacing
    opts = ("--rays", str(RAYS), "--beta", str(BETA), "--gamma", str(GAMMA), "--support-rho", str(SUPPORT_RHO))
    try:
        job = ref_exe.run("correct", ISOTOPE, g, rho, sp, *opts, "--iterations", str(iterations))
        rate = ref_exe.run("correct", ISOTOPE, g, rho, sp, *opts, "--iterations", str(rate_iterations))
    except (RuntimeError, OSError, subprocess.TimeoutExpired) as e:
        return {"unavailable": f"reference executable failed: {str(e)[:200]}"}
    return {"value": round(rate_iterations / rate["iterations_s"], 3), "unit": "EM iters/s",
            "rate_iterations": rate_iterations, "rate_iteration_seconds": rate["iterations_s"],
            "job": {"iterations": iterations, "setup_s": job["setup_s"], "iterations_s": job["iterations_s"],
                    "seconds": round(job["setup_s"] + job["iterations_s"], 3), "total_s": job["total_s"]},
            "what": "prc.cu built for sm_100a, timed by its own 2-decimal clock"}


def measured_data(rho, truth, spacing, P=None, use_reference=True):
    """The measured data both arms correct: the truth blurred by the plain projector with 128
    rays -- the reference executable's own forward projection where it is built, else the
    engine's fp32 field (`P`) -- and Poisson-sampled at 5e7 counts with seed 100 by the
    counter-based device sampler (prc_poisson: every count depends only on its own mean, so the
    last-bit noise of the reference's atomic forward changes no other voxel's count).
    Multi-GPU replicas use the engine (the reference executable runs on one device only).
    Returns (data, description, sha256 prefix of its bytes)."""
    import hashlib
    from oracle import ref_exe
    from prc_mlem_b200 import phantoms
    blur, how = None, None
    if use_reference and ref_exe.available():
        try:
            blur = ref_exe.run("forward", ISOTOPE, truth, rho, spacing, "--rays", str(RAYS),
                               "--support-rho", str(SUPPORT_RHO))["out"]
            how = "synthetic (seeded torso phantom, blurred by prc.cu's projector, Poisson 5e7 counts)"
        except (RuntimeError, OSError, subprocess.TimeoutExpired):
            blur = None
    if blur is None and P is not None:
        blur, how = P.forward_host(truth), "synthetic (seeded torso phantom, blurred by the fp32 field, Poisson 5e7)"
    if blur is None:  # projection cost does not depend on the activity values, only on the density
        blur, how = truth, "synthetic (seeded torso phantom, unblurred truth Poisson-sampled at 5e7 counts)"
    try:
        import torch
        cuda = torch.cuda.is_available()
    except ImportError:
        cuda = False
    if cuda:
        g = phantoms.poisson_counts_device(torch.from_numpy(np.ascontiguousarray(blur, np.float32)).cuda(), COUNTS,
                                           seed=100).cpu().numpy()
    else:
        g = phantoms.poisson_counts(blur, COUNTS, seed=100)
        how += " (host sampler: no CUDA device)"
    return g, how, hashlib.sha256(g.tobytes()).hexdigest()[:16]


# ------------------------------------------------------------------ frames sharing one density map
def shared_frames_record(P, truth, g_host, stream, l2_flush, iterations, single_value, corrected,
                         n_frames: int = 4, steps: int = 3, warmup: int = 1) -> dict:
    """The frames of one dynamic study share the density map (one CT), so they share the
    projector: frame 0 is the headline data, frames 1.. further Poisson draws (seeds 101..) of
    the same blur, all corrected by one prc_em_run_frames call per step (each projection one
    pass over the stored field for up to four frames).  Reports frame-iterations/s, the
    projection passes' mean device time against the single-volume launches, and frame 0's
    difference from the single-volume correction of the same data (bit-identical by design)."""
    import torch
    import prc_mlem_b200 as pm
    from prc_mlem_b200 import phantoms
    blur = torch.empty(g_host.size, dtype=torch.float32, device="cuda")
    d_truth = torch.from_numpy(np.ascontiguousarray(truth, np.float32)).cuda().reshape(-1)
    P.forward(d_truth, blur)
    P.synchronize()
    d_gs = [torch.from_numpy(g_host).cuda().reshape(-1)]
    d_gs += [phantoms.poisson_counts_device(blur, COUNTS, seed=100 + k).reshape(-1) for k in range(1, n_frames)]
    d_outs = [torch.empty_like(d_gs[0]) for _ in range(n_frames)]
    torch.cuda.synchronize()
    for _ in range(warmup):
        P.correct_frames(d_gs, d_outs, iterations, BETA, GAMMA, True)
    P.synchronize()
    times = []
    P.timing(True)
    for _ in range(steps):
        l2_flush()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        P.correct_frames(d_gs, d_outs, iterations, BETA, GAMMA, True)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    P.timing(False)
    passes = P.timing_read()
    total_s = sum(times) / 1e3
    value = n_frames * iterations * steps / total_s
    diff = float(np.max(np.abs(d_outs[0].cpu().numpy().reshape(corrected.shape) - corrected)))
    return {"value": round(value, 3), "unit": "EM frame-iterations/s",
            "frames_per_s": round(n_frames * steps / total_s, 3),
            "x_single_volume": round(value / single_value, 3),
            "steps": steps, "warmup": warmup, "ms_per_step": round(sum(times) / steps, 3),
            "config": {"workload": f"{n_frames} frames of the 128x128x159 68Ga torso sharing its density map, "
                                   f"{iterations} MAP-EM iterations each per step (beta {BETA}, gamma {GAMMA}, "
                                   "accel), fp32 stored field", "l2": "flushed before every step"},
            "pass_ms": {"forward": round(passes["forward_ms"] / max(passes["forward_launches"], 1), 4),
                        "adjoint": round(passes["adjoint_ms"] / max(passes["adjoint_launches"], 1), 4),
                        "frames_per_pass": min(n_frames, 4)},
            "frame0_max_abs_diff_vs_single_volume": diff}


def study_batch_record(rho, truth, spacing, iterations, single_value, n_frames: int = 8, steps: int = 3,
                       warmup: int = 1) -> dict:
    """A dynamic study through the batch API: n_frames frames of the torso passing the same density
    array (prc_batch_create shares one projector among them and the batched projections take them
    four at a time), the data n_frames Poisson draws of the same blur; one graph replay of
    `iterations` MAP-EM iterations of every frame per step."""
    import torch
    import prc_mlem_b200 as pm
    from prc_mlem_b200 import phantoms
    batch = pm.Batch([(ISOTOPE, rho, spacing)] * n_frames, rays=RAYS, support_rho=SUPPORT_RHO)
    stream = torch.cuda.ExternalStream(batch.stream)
    with pm.Projector(ISOTOPE, rho, spacing, rays=RAYS, support_rho=SUPPORT_RHO) as P:
        blur = torch.empty(truth.size, dtype=torch.float32, device="cuda")
        P.forward(torch.from_numpy(np.ascontiguousarray(truth, np.float32)).cuda().reshape(-1), blur)
        P.synchronize()
    gs = [phantoms.poisson_counts_device(blur, COUNTS, seed=300 + k) for k in range(n_frames)]
    outs = [torch.empty_like(g) for g in gs]
    torch.cuda.synchronize()
    for _ in range(warmup):
        batch.correct(gs, outs, iterations, BETA, GAMMA, True)
    batch.synchronize()
    times = []
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        batch.correct(gs, outs, iterations, BETA, GAMMA, True)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    total_s = sum(times) / 1e3
    value = n_frames * iterations * steps / total_s
    device_gb = [round(batch.device_bytes(i) / 1e9, 3) for i in (0, 1)]
    batch.close()
    return {"value": round(value, 3), "unit": "EM frame-iterations/s",
            "frames_per_s": round(n_frames * steps / total_s, 3), "x_single_volume": round(value / single_value, 3),
            "steps": steps, "warmup": warmup, "ms_per_step": round(sum(times) / steps, 3),
            "device_gb_owner_and_sharer": device_gb,
            "config": {"workload": f"{n_frames} frames of the 128x128x159 68Ga torso passing one density array to "
                                   f"prc_batch_create, {iterations} MAP-EM iterations each per step (beta {BETA}, "
                                   f"gamma {GAMMA}, accel), fp32 stored field, one graph replay per step"}}


# ------------------------------------------------------------------------------- batched frames
BATCH_GRIDS = ((64, 64, 64), (80, 96, 96), (159, 128, 128), (200, 192, 192))
BATCH_ISOTOPES = ("11C", "15O", "18F", "68Ga")


def batch_record(frames: int, iterations: int, steps: int, warmup: int, surrogate: bool = False,
                 clocks: bool = False) -> dict:
    """Dynamic-PET frames: grids drawn from {64^3, 96x96x80, 128x128x159, 192x192x200}, isotopes
    from {11C, 15O, 18F, 68Ga}, each the torso generator with its own seed and counts
    log-uniform in [1e5, 5e7]; `iterations` MAP-EM iterations (beta 0.03, gamma 20,
    accelerated) of every frame per step, all frames in one launch per phase inside one
    captured CUDA graph.  Returns the record (frames/s and its context)."""
    import torch
    import prc_mlem_b200 as pm
    from prc_mlem_b200 import phantoms, surrogate as sg
    torch.cuda.set_device(0)
    rng = np.random.default_rng(5)
    specs = []
    for i in range(frames):
        shape = BATCH_GRIDS[rng.integers(len(BATCH_GRIDS))]
        iso = BATCH_ISOTOPES[rng.integers(len(BATCH_ISOTOPES))]
        counts = float(np.exp(rng.uniform(np.log(1e5), np.log(5e7))))
        rho, truth, sp = phantoms.torso_phantom(seed=100 + i, shape=shape)
        specs.append((iso, rho, sp, truth, counts))
    net = sg.load_trained() if surrogate else None
    t0 = time.perf_counter()
    batch = pm.Batch([(iso, rho, sp) for iso, rho, sp, _, _ in specs], precision=pm.PRC_PRECISION_BF16,
                     surrogate=net, target_scale=sg.TARGET_SCALE, fallback_nrmse=JUDGE_THRESHOLD if net else 0.0)
    setup_s = time.perf_counter() - t0
    gs, outs = [], []
    for i, (iso, rho, sp, truth, counts) in enumerate(specs):
        d_t = torch.from_numpy(truth).cuda()
        d_b = torch.empty_like(d_t)
        batch.forward(i, d_t, d_b)
        gs.append(phantoms.poisson_counts_device(d_b, counts, seed=200 + i))
        outs.append(torch.empty_like(d_t))
    torch.cuda.synchronize()  # the counts are drawn on torch's stream, the batch runs on its own
    stream = torch.cuda.ExternalStream(batch.stream)
    for _ in range(warmup):
        batch.correct(gs, outs, iterations, BETA, GAMMA, True)
    batch.synchronize()
    sampler = ClockSampler(0) if clocks else None
    if sampler:
        sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        batch.correct(gs, outs, iterations, BETA, GAMMA, True)
    e1.record(stream)
    e1.synchronize()
    batch.synchronize()
    clock_info = sampler.stop() if sampler else None
    ms = e0.elapsed_time(e1)
    frames_per_s = frames * steps / (ms / 1e3)
    # the launch structure: one graph replay against the same launches made one by one
    prof = batch.profile(gs, outs, iterations, BETA, GAMMA, True)
    prof["gap_ms"] = round(prof["graph_ms"] - prof["launches_ms"], 4)
    prof["gap_share"] = round(prof["gap_ms"] / prof["graph_ms"], 5)
    # per-frame NRMSE against the plain method (fp32 weights, reference numerics), first 4 frames
    nrmse_list = []
    for i in range(min(4, frames)):
        iso, rho, sp, truth, counts = specs[i]
        with pm.Projector(iso, rho, sp, cache=pm.PRC_CACHE_NEAR) as P:
            d = torch.empty_like(gs[i])
            P.correct(gs[i], d, iterations, BETA, GAMMA, True)
            P.synchronize()
            nrmse_list.append(nrmse(outs[i].cpu().numpy(), d.cpu().numpy()))
    modes = collections.Counter(batch.cache_mode(i)[0] for i in range(frames))
    rec = {"value": round(frames_per_s, 3), "unit": "frames/s", "steps": steps, "warmup": warmup,
           "ms_per_step": round(ms / steps, 3), "em_iters_per_s": round(frames_per_s * iterations, 2),
           "dtype": "f32 (bf16 stored weights)",
           "config": {"workload": f"{frames} frames, grids {BATCH_GRIDS}, isotopes {BATCH_ISOTOPES}, torso "
                                  f"phantoms, counts log-uniform 1e5-5e7, {iterations} MAP-EM iterations, beta 0.03, "
                                  "gamma 20, accel",
                      "frames": [f"{iso} {rho.shape[2]}x{rho.shape[1]}x{rho.shape[0]}" for iso, rho, *_ in specs],
                      "projector_forms": {str(k): v for k, v in modes.items()},
                      "surrogate": bool(net), "autotuned": {"warps_per_block": batch.warps},
                      "setup_s": round(setup_s, 2)},
           "nrmse_vs_plain_first_frames": nrmse_list,
           "schedule": {"what": "one CUDA-graph replay of the run vs the same kernel launches timed one by one "
                                "with CUDA events; the gap bounds what one persistent kernel per iteration could save",
                        **{k: (round(v, 4) if isinstance(v, float) else v) for k, v in prof.items()}}}
    if clock_info:
        rec["clocks"] = clock_info
    batch.close()
    return rec


def run_batch(args):
    rec = batch_record(args.frames, 10, args.steps, args.warmup, surrogate=args.surrogate, clocks=True)
    rec = {"metric": "batched dynamic-PET frames per second (10 MAP-EM iterations each)", "n_gpus": 1,
           "higher_is_better": True} | rec
    print(json.dumps(rec))


def run_surrogate_eval(args):
    """The learned surrogate's evaluation: the small phantom's geometry on the 128x128x159 grid,
    data = the plain projector's blur of its activity, Poisson-sampled at 5e7 counts, 6-iteration
    MAP-EM for each isotope the network was trained on.  Per form: EM iters/s, NRMSE of the
    corrected image against the plain fp32 field (full volume) and against the FP64 oracle (a
    central 64x48x32 crop), and the share of sources the tracer's judge sent back to exact
    weights.  The crop comparison runs every form on the cropped volume and data, as the oracle
    does, so both see the same problem."""
    import torch
    import prc_mlem_b200 as pm
    from prc_mlem_b200 import phantoms, surrogate as sg
    from oracle import oracle
    world, rank, _ = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(0)
    rho, truth, spacing = phantoms.scaled_small_phantom(seed=1, shape=tuple(args.grid))
    nz, ny, nx = rho.shape
    sl = (slice(nz // 2 - 16, nz // 2 + 16), slice(ny // 2 - 24, ny // 2 + 24), slice(nx // 2 - 32, nx // 2 + 32))
    net = sg.load_trained()
    results = {}
    for iso in sg.ISOTOPES:
        forms = [("fp32_field", dict(cache=pm.PRC_CACHE_FULL)),
                 ("bf16_field", dict(cache=pm.PRC_CACHE_FULL, precision=pm.PRC_PRECISION_BF16)),
                 ("traced", dict(cache=pm.PRC_CACHE_NEAR)),
                 ("radial_traced_bf16", dict(precision=pm.PRC_PRECISION_BF16, surrogate="traced"))]
        if net is not None:
            forms += [("learned_bf16", dict(precision=pm.PRC_PRECISION_BF16, surrogate=net,
                                            target_scale=sg.TARGET_SCALE)),
                      ("learned_judged_bf16", dict(precision=pm.PRC_PRECISION_BF16, surrogate=net,
                                                   target_scale=sg.TARGET_SCALE, fallback_nrmse=JUDGE_THRESHOLD))]
        out, plain = {}, None
        g = None
        for name, kw in forms:
            Q = pm.Projector(iso, rho, spacing, rays=RAYS, support_rho=SUPPORT_RHO, **kw)
            if g is None:  # the data: the plain projector's blur of the activity, Poisson-sampled
                g = phantoms.poisson_counts_device(torch.from_numpy(Q.forward_host(truth)).cuda(), COUNTS,
                                                   seed=5).cpu().numpy()
                d_g = torch.from_numpy(g).cuda()
                d_out = torch.empty_like(d_g)
            s = torch.cuda.ExternalStream(Q.stream)
            Q.correct(d_g, d_out, args.iterations, BETA, GAMMA, True)
            Q.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            for _ in range(3):
                Q.correct(d_g, d_out, args.iterations, BETA, GAMMA, True)
            e1.record(s)
            e1.synchronize()
            img = d_out.cpu().numpy()
            if plain is None:
                plain = img
            out[name] = {"iters_per_s": round(3 * args.iterations / (e0.elapsed_time(e1) / 1e3), 2),
                         "nrmse_vs_fp32_field": nrmse(img, plain)}
            if "surrogate" in kw:
                out[name]["exact_fallback_share"] = round(Q.fallbacks / (Q.n_active * RAYS), 4)
            Q.close()
            with pm.Projector(iso, np.ascontiguousarray(rho[sl]), spacing, rays=RAYS, support_rho=SUPPORT_RHO,
                              **kw) as C:
                out[name]["crop_image"] = C.correct_host(np.ascontiguousarray(g[sl]), args.iterations, BETA, GAMMA,
                                                         True)
        O = oracle.Problem(iso, np.ascontiguousarray(rho[sl]), spacing, rays=RAYS, support_rho=SUPPORT_RHO,
                           precision=64, threads=os.cpu_count() or 1)
        ref = O.correct(np.ascontiguousarray(g[sl]), args.iterations, BETA, GAMMA, True)
        for name in out:
            out[name]["nrmse_vs_fp64_crop"] = nrmse(out[name].pop("crop_image"), ref)
        results[iso] = out
    print(json.dumps({"workload": f"surrogate evaluation: small phantom geometry on {nx}x{ny}x{nz} at "
                                  f"{spacing[0]}x{spacing[1]}x{spacing[2]} mm, {args.iterations} MAP-EM iterations, "
                                  f"beta {BETA}, gamma {GAMMA:g}, Poisson {COUNTS:g} counts",
                      "network": "trained" if net is not None else "absent", "isotopes": results}))


def run_tiles(args):
    """Stored-field projections per source tile shape, fp32 and bf16 weights, on the torso: mean
    device time of ten forward and ten adjoint projections (after three warm-up pairs) and of
    one MAP-EM iteration (a 6-iteration correction / 6), and the stored entries."""
    import torch
    import prc_mlem_b200 as pm
    torch.cuda.set_device(0)
    rho, truth, spacing = make_workload(args.grid)
    d = torch.from_numpy(truth).cuda()
    out = {}
    for prec_name, prec in (("fp32", pm.PRC_PRECISION_FP32), ("bf16", pm.PRC_PRECISION_BF16)):
        for tile, shape in pm.TILE_SHAPES.items():
            if args.tile != "auto" and "x".join(map(str, shape)) != args.tile:
                continue
            P = pm.Projector(ISOTOPE, rho, spacing, rays=RAYS, support_rho=SUPPORT_RHO, precision=prec, tile=tile)
            o = torch.empty_like(d)
            s = torch.cuda.ExternalStream(P.stream)
            for _ in range(3):
                P.forward(d, o)
                P.adjoint(d, o)
            P.synchronize()
            rec = {}
            for name, fn in (("forward_ms", P.forward), ("adjoint_ms", P.adjoint)):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(s)
                for _ in range(10):
                    fn(d, o)
                e1.record(s)
                e1.synchronize()
                rec[name] = round(e0.elapsed_time(e1) / 10, 4)
            P.forward(d, o)
            g = o.clone()
            P.correct(g, o, args.iterations, BETA, GAMMA, True)
            P.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            P.correct(g, o, args.iterations, BETA, GAMMA, True)
            e1.record(s)
            e1.synchronize()
            rec["em_iteration_ms"] = round(e0.elapsed_time(e1) / args.iterations, 4)
            rec["stored_entries"] = P.cache_mode[1]
            out[f"{prec_name} {'x'.join(map(str, shape))}"] = rec
            P.close()
    nz, ny, nx = args.grid
    print(json.dumps({"workload": f"torso {nx}x{ny}x{nz}, {ISOTOPE}, rays {RAYS}", "tiles": out}))


def run_frames(args):
    """Frames sharing one density map on the torso (--grid, --form): the mean device time of ten
    forward and ten adjoint projections of 1, 2 and 4 frames per call (after two warm-up calls),
    per frame and against the single-volume launch, and one MAP-EM run of --frames frames
    (--iterations each) against as many single-volume runs."""
    import torch
    import prc_mlem_b200 as pm
    torch.cuda.set_device(0)
    rho, truth, spacing = make_workload(args.grid)
    cache, prec = FORMS[args.form]
    P = pm.Projector(ISOTOPE, rho, spacing, rays=RAYS, support_rho=SUPPORT_RHO, cache=cache, precision=prec)
    s = torch.cuda.ExternalStream(P.stream)
    d = torch.from_numpy(truth).cuda()
    n = max(1, args.frames)
    ins = [d * (1.0 + 0.1 * k) for k in range(max(n, 4))]
    outs = [torch.empty_like(d) for _ in ins]
    torch.cuda.synchronize()

    def timed(fn, reps=10, warm=2):
        for _ in range(warm):
            fn()
        P.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(reps):
            fn()
        e1.record(s)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    single = {"forward_ms": round(timed(lambda: P.forward(ins[0], outs[0])), 4),
              "adjoint_ms": round(timed(lambda: P.adjoint(ins[0], outs[0])), 4)}
    per_call = {}
    for k in (1, 2, 4):
        f = timed(lambda: P.forward_frames(ins[:k], outs[:k]))
        a = timed(lambda: P.adjoint_frames(ins[:k], outs[:k]))
        per_call[str(k)] = {"forward_ms": round(f, 4), "adjoint_ms": round(a, 4),
                            "forward_ms_per_frame": round(f / k, 4), "adjoint_ms_per_frame": round(a / k, 4)}
    gs = [torch.empty_like(d) for _ in range(n)]
    for k in range(n):
        P.forward(ins[k], gs[k])
    em_outs = [torch.empty_like(d) for _ in range(n)]
    shared = timed(lambda: P.correct_frames(gs, em_outs, args.iterations, BETA, GAMMA, True), reps=2, warm=1)

    def one_by_one():
        for k in range(n):
            P.correct(gs[k], em_outs[k], args.iterations, BETA, GAMMA, True)
    alone = timed(one_by_one, reps=2, warm=1)
    nz, ny, nx = args.grid
    print(json.dumps({"workload": f"torso {nx}x{ny}x{nz}, {ISOTOPE}, rays {RAYS}, {args.form} stored field",
                      "single_volume": single, "frames_per_call": per_call,
                      "map_em": {"frames": n, "iterations": args.iterations,
                                 "shared_ms": round(shared, 3), "one_by_one_ms": round(alone, 3),
                                 "speedup": round(alone / shared, 3)}}))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "surrogate":
        run_surrogate_eval(args)
    elif args.workload == "tiles":
        run_tiles(args)
    elif args.workload == "frames":
        run_frames(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
