#!/usr/bin/env python
"""Throughput of the fused near-field SAR backprojection + surface-normal vote.

Workload (one "step"): the 128^3-voxel, 128x128-antenna, 256-frequency scene
(2 mm voxel and antenna pitch, 77-81 GHz, 20k scatterers on a box U cylinder at
z = 0.45 m, 15 dB) -- backprojection fused with the normal vote over the whole grid
(image + vote), then the mask / unit-normal epilogue.  8.8e12 voxel*antenna*frequency
updates per step.  Inputs are synthetic (seeded); they are resident in HBM before the
timed region; the 126 MB L2 is flushed (256 MB write) before every step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints ONE JSON line on rank 0.  ``--impl reference`` times the reference's own CPU
imager (src/data_processing/cpp/imaging.cpp, built from source into oracle/_ref) on the
host cores on a bounded voxel sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "G voxel·ant·freq updates/s, mixed vs plain FP32 on 1 B200 at ≤1e-4 L2 err"  # fused image + normal vote
UNIT = "G updates/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--plain-steps", type=int, default=1)
    ap.add_argument("--nufft-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="target CPU seconds of the bounded reference/CPU sample")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-interp", action="store_true",
                    help="skip the interpolated-mode leg (reference kernels, bit-exact and "
                         "fast forms)")
    ap.add_argument("--no-reference-cuda", action="store_true",
                    help="skip the reference CUDA kernel's full matched filter")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--no-next-rows", action="store_true",
                    help="skip the isosurface-channel and RSDF legs")
    ap.add_argument("--variant", default=None,
                    help="force a mixed kernel variant by name instead of autotuning")
    ap.add_argument("--aperture", type=int, default=128,
                    help="aperture side (antennas); smaller values make a profiling case "
                         "with the same kernel and voxel grid (the default is the workload)")
    return ap.parse_args()


# ----------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu_index = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="mmn_clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu_index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4)
                          if r[5 + k].lower().startswith("active")})
        loaded = sorted(sm)[len(sm) // 4:] if len(sm) >= 4 else sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows
                                   if r[3].replace(".", "").isdigit()) if rows else None}


# --------------------------------------------------------------------- the scene
def load_scene(device, aperture=128):
    from mmnorm_b200 import scenes
    sc = scenes.config1(sign=-1, device=device)
    if aperture != 128:
        # profiling case: the central aperture x aperture antennas of the same scene
        n0 = (128 - aperture) // 2
        idx = (np.arange(n0, n0 + aperture)[:, None] * 128 +
               np.arange(n0, n0 + aperture)[None, :]).ravel()
        sc.antenna_locs = np.ascontiguousarray(sc.antenna_locs[idx])
        sc.meas = np.ascontiguousarray(sc.meas[idx])
        sc.name = sc.name.replace("ap128", "ap%d" % aperture)
    return sc


def cpu_sample_axes(sc, n_voxels_target, cores):
    """A voxel sub-grid of the workload's grid: `cores` x-slices (the reference imager's
    OpenMP loop runs over x) spread over the grid, one y row, z columns as needed."""
    nx = max(1, min(len(sc.x_locs), cores))
    xi = np.linspace(0, len(sc.x_locs) - 1, nx).round().astype(int)
    nz = max(1, min(len(sc.z_locs), int(math.ceil(n_voxels_target / nx))))
    zi = np.linspace(0, len(sc.z_locs) - 1, nz).round().astype(int)
    yi = np.array([len(sc.y_locs) // 2])
    return sc.x_locs[xi], sc.y_locs[yi], sc.z_locs[zi]


def time_reference_imager(sc, steps, warmup, target_seconds):
    """Reference imager on host cores; returns (updates/s, info dict)."""
    from oracle import ref_imager
    cores = os.cpu_count() or 1
    A, F = sc.meas.shape
    meas = sc.meas[:, :, None]
    rxo = np.zeros((1, 3), np.float32)
    # calibrate: one voxel per x-slice
    x, y, z = cpu_sample_axes(sc, cores, cores)
    cal = ref_imager.time_sample(x, y, z, sc.antenna_locs, meas, rxo, sc.slope, sc.f_lo,
                                 steps=1, warmup=0, threads=cores)
    per = max(1e-6, cal["step_seconds"][0] - cal["conversion_seconds"])
    nvox_cal = len(x) * len(y) * len(z)
    n_target = int(nvox_cal * target_seconds / per)
    x, y, z = cpu_sample_axes(sc, max(nvox_cal, n_target), cores)
    res = ref_imager.time_sample(x, y, z, sc.antenna_locs, meas, rxo, sc.slope, sc.f_lo,
                                 steps=steps, warmup=warmup, threads=cores)
    nvox = len(x) * len(y) * len(z)
    upd = nvox * A * F
    compute = [max(1e-9, t - res["conversion_seconds"]) for t in res["step_seconds"]]
    rate = upd / statistics.median(compute)
    info = {"voxels": nvox, "updates_per_step": upd, "step_seconds": res["step_seconds"],
            "conversion_seconds": res["conversion_seconds"], "threads": res["threads"],
            "sample": "%d voxels (%d x-slices x %d y x %d z) of the 128^3 grid, all %d antennas "
                      "x %d freqs; reference imager (imaging.cpp) built from source, "
                      "OMP_NUM_THREADS=%d; rate excludes the per-call pybind11 input "
                      "conversion (%.2f s, timed on a 1-voxel call)"
                      % (nvox, len(x), len(y), len(z), A, F, res["threads"],
                         res["conversion_seconds"])}
    return rate, info


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    try:
        from oracle import ref_imager
        if not ref_imager.available():
            from oracle import build as ob
            ob.build_ref()
        if not ref_imager.available():
            print(json.dumps({"impl": "reference", "unavailable":
                              "reference imager not built (oracle/build.py needs the mmNorm "
                              "checkout at build time)"}))
            return 0
    except Exception as e:  # pragma: no cover
        print(json.dumps({"impl": "reference", "unavailable": str(e)[:200]}))
        return 0
    sc = load_scene("cuda" if _has_cuda() else None)
    per_step = max(2.0, args.cpu_seconds / 3.0)
    rate, info = time_reference_imager(sc, max(1, args.steps), max(0, args.warmup), per_step)
    value = rate / 1e9
    ms = 1e3 * statistics.median(info["step_seconds"])
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded point-scatterer scene)",
        "config": {"workload": sc.name + " (128^3 voxels @2 mm, 128x128 antennas @2 mm, "
                   "256 freqs 77-81 GHz)", "voxels": sc.num_voxels,
                   "antennas": int(sc.meas.shape[0]), "freqs": int(sc.meas.shape[1]),
                   "parallelism": "host OpenMP", "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": info["threads"],
                         "kind": "reference", "sample": info["sample"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def _has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


# ------------------------------------------------------------------- our arm
def ours_arm(args):
    import torch
    import torch.distributed as dist

    from mmnorm_b200 import _lib, autotune, ops, shard

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=dev)
    lib = _lib.load()
    _lib.check(lib.mmn_check_device(local), "mmn_check_device")

    sc = load_scene(dev, args.aperture)
    A, F = sc.meas.shape
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    # N GPUs: the grid grows by one 128-plane slab per GPU along x (same pitch, centred
    # on the scene) and every rank images its own slab (voxel-slab sharding, weak scaling)
    nx_total = len(sc.x_locs) * world
    if world > 1:
        pitch = float(sc.x_locs[1] - sc.x_locs[0])
        x_all = (float(np.mean(sc.x_locs)) +
                 (np.arange(nx_total) - (nx_total - 1) / 2.0) * pitch).astype(np.float32)
        x0, x1 = shard.split_bounds(nx_total, world, rank)
        xs = t(x_all[x0:x1])
    else:
        xs = t(sc.x_locs)
    ys, zs = t(sc.y_locs), t(sc.z_locs)
    V = xs.numel() * ys.numel() * zs.numel()
    updates = V * A * F
    ant, rxo = t(sc.antenna_locs), t(np.zeros((1, 3), np.float32))
    meas = t(sc.meas)
    if args.variant:
        names = [v["name"] for v in ops.variants("mixed")]
        ops.set_variant("mixed", names.index(args.variant))
        tuned = {"best": names.index(args.variant), "times_ms": None}
    else:
        tuned = autotune.tune(xs, ys, zs, ant, rxo, meas, sc.wavelength, sc.slope, mode="mixed")
    variant = ops.variants("mixed")[tuned["best"]]
    prob = ops.make_problem(xs, ys, zs, ant, rxo, meas, sc.wavelength, sc.slope)
    ws = torch.empty(ops.workspace_bytes(prob, "mixed"), dtype=torch.uint8, device=dev)
    plan = ops.plan_info(prob, "mixed")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    max_abs = torch.empty(1, dtype=torch.float32, device=dev)

    def step(mode="mixed", ev=None, workspace=None):
        flush.fill_(1)
        if ev is not None:
            ev[0].record(stream)
        img, vote = ops.backproject(xs, ys, zs, ant, rxo, meas, sc.wavelength, sc.slope,
                                    mode=mode, workspace=ws if workspace is None else workspace)
        if ev is not None:
            ev[1].record(stream)
        # mask threshold: 5 % of max|I| over the whole grid (one float all-reduced)
        ops.image_max_abs(img, out=max_abs)
        if world > 1:
            dist.all_reduce(max_abs, op=dist.ReduceOp.MAX)
        normals, mask = ops.surface_normals_from_max(img, vote, max_abs, 0.05)
        return img, vote, normals, mask

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # FP32 peak probe (the roofline denominator), right before the timed region
    probe_out = torch.empty(148 * 8 * 256, dtype=torch.float32, device=dev)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    blocks, iters = sms * 8, 20000
    for _ in range(2):
        _lib.check(lib.mmn_fp32_peak_probe(blocks, 200, ops._vp(probe_out), ops._stream(dev)),
                   "probe")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    probe_rates = []
    for _ in range(3):
        e0.record(stream)
        _lib.check(lib.mmn_fp32_peak_probe(blocks, iters, ops._vp(probe_out), ops._stream(dev)),
                   "probe")
        e1.record(stream)
        torch.cuda.synchronize()
        probe_rates.append(blocks * 256.0 * iters * 32 / (e0.elapsed_time(e1) * 1e-3))
    fp32_peak = max(probe_rates)

    for _ in range(max(3, args.warmup)):
        step()
    clocks = ClockSampler(local)
    kernel_events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                     for _ in range(args.steps)]
    barrier()
    clocks.start()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for k in range(args.steps):
        step(ev=kernel_events[k])
    t1.record(stream)
    barrier()
    clk = clocks.stop()
    total_ms = t0.elapsed_time(t1)
    if world > 1:
        tt = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total_ms = float(tt.item())
    value = world * updates * args.steps / (total_ms * 1e-3) / 1e9
    kern_ms = [a.elapsed_time(b) for a, b in kernel_events]
    kern_avg_s = statistics.mean(kern_ms) * 1e-3

    # outputs on a seeded 4096-voxel subset, for the accuracy report against the FP64 oracle
    acc_idx = np.sort(np.random.default_rng(2).choice(V, 4096, replace=False))
    acc_t = torch.as_tensor(acc_idx, device=dev)

    def subset(img, vote):
        I = img.reshape(-1)[acc_t].cpu().numpy()
        W = vote.reshape(3, -1)[:, acc_t].cpu().numpy().T
        return (I, W), float(img.abs().max())

    acc_mixed = acc_plain = None
    if rank == 0 and world == 1 and not args.no_accuracy:
        img_a, vote_a, _, _ = step()
        acc_mixed = subset(img_a, vote_a)
        del img_a, vote_a
    # the library's count for backproject (prep_antennas, stage_meas when the form needs a
    # staged copy, bp_fwd_kernel, bp_reduce_partials when split) + max_abs + normals
    launches_per_step = plan["launches"] + 2

    out = {}
    if rank == 0 and world == 1 and args.plain_steps > 0:
        # plain FP32 sincos-per-sample form on the same workload
        ptuned = autotune.tune(xs, ys, zs, ant, rxo, meas, sc.wavelength, sc.slope,
                               mode="plain", max_antennas=256)
        step("plain")
        pe = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.plain_steps)]
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for k in range(args.plain_steps):
            step("plain", ev=pe[k])
        p1.record(stream)
        torch.cuda.synchronize()
        pms = p0.elapsed_time(p1) / args.plain_steps
        pval = updates / (pms * 1e-3) / 1e9
        if not args.no_accuracy:
            img_a, vote_a, _, _ = step("plain")
            acc_plain = subset(img_a, vote_a)
            del img_a, vote_a
        out["plain"] = {"value": pval, "unit": UNIT, "ms_per_step": pms,
                        "kernel_ms": statistics.mean(a.elapsed_time(b) for a, b in pe),
                        "mixed_over_plain": value / pval,
                        "variant": ops.variants("plain")[ptuned["best"]]["name"]}

    if rank == 0 and world == 1 and args.nufft_steps > 0:
        # the same sums by 8-tap interpolation from per-antenna oversampled grids (a type-2
        # non-uniform FFT): not the mixed recurrence, so reported beside it, with its
        # distance from the mixed form's outputs on this workload
        img_m, vote_m, _, _ = step()
        img_m, vote_m = img_m.clone(), vote_m.clone()
        ws_nu = torch.empty(lib.mmn_backproject_nufft_workspace_bytes(ctypes.byref(prob)),
                            dtype=torch.uint8, device=dev)
        img_n, vote_n, _, _ = step("nufft", workspace=ws_nu)
        rel = lambda a, b: float((a.to(torch.complex128) - b.to(torch.complex128)).norm() /
                                 b.to(torch.complex128).norm())
        rel_img, rel_vote = rel(img_n, img_m), rel(vote_n, vote_m)
        del img_m, vote_m, img_n, vote_n
        ne = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.nufft_steps)]
        torch.cuda.synchronize()
        n0, n1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n0.record(stream)
        for k in range(args.nufft_steps):
            step("nufft", ev=ne[k], workspace=ws_nu)
        n1.record(stream)
        torch.cuda.synchronize()
        nms = n0.elapsed_time(n1) / args.nufft_steps
        nval = updates / (nms * 1e-3) / 1e9
        out["nufft"] = {"value": nval, "unit": UNIT + " equivalent (interpolated sums)",
                        "ms_per_step": nms,
                        "kernel_ms": statistics.mean(a.elapsed_time(b) for a, b in ne),
                        "over_mixed": nval / value,
                        "rel_l2_vs_mixed": {"image": rel_img, "vote": rel_vote}}

    adjoint = None
    if rank == 0 and world == 1 and not args.no_adjoint:
        adjoint = time_adjoint(dev)
    batched = None
    if rank == 0 and world == 1 and not args.no_batched:
        batched = time_batched(dev)

    # end to end through the public API: pinned host inputs -> device -> image + normals
    # -> pinned host outputs, every step
    e2e = None
    if not args.no_e2e:
        # every rank: its slab's inputs from pinned host memory, the step, its image and
        # normals back to pinned host memory; the mask's max|I| all-reduced as in the step
        h_meas = torch.empty(meas.shape, dtype=meas.dtype, pin_memory=True)
        h_meas.copy_(torch.as_tensor(sc.meas))
        h_ant = torch.as_tensor(sc.antenna_locs).pin_memory()
        h_axes = [xs.cpu().pin_memory()] + [torch.as_tensor(a).pin_memory()
                                            for a in (sc.y_locs, sc.z_locs)]
        h_rxo = torch.zeros((1, 3), dtype=torch.float32).pin_memory()
        h_img = torch.empty(V, dtype=torch.complex64, pin_memory=True)
        h_nrm = torch.empty((V, 3), dtype=torch.float32, pin_memory=True)
        n_e2e = max(1, min(args.steps, 3))

        def e2e_step():
            flush.fill_(1)
            d_meas = h_meas.to(dev, non_blocking=True)
            d_ant = h_ant.to(dev, non_blocking=True)
            d_axes = [a.to(dev, non_blocking=True) for a in h_axes]
            d_rxo = h_rxo.to(dev, non_blocking=True)
            img, vote = ops.backproject(*d_axes, d_ant, d_rxo, d_meas, sc.wavelength, sc.slope,
                                        mode="mixed")
            mx = ops.image_max_abs(img)
            if world > 1:
                dist.all_reduce(mx, op=dist.ReduceOp.MAX)
            normals, mask = ops.surface_normals_from_max(img, vote, mx, 0.05)
            h_img.copy_(img.reshape(-1), non_blocking=True)
            h_nrm.copy_(normals.reshape(-1, 3), non_blocking=True)
            torch.cuda.synchronize()

        e2e_step()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        s0.record(stream)
        for _ in range(n_e2e):
            e2e_step()
        s1.record(stream)
        barrier()
        ems = s0.elapsed_time(s1) / n_e2e
        if world > 1:
            et = torch.tensor([ems], device=dev, dtype=torch.float64)
            dist.all_reduce(et, op=dist.ReduceOp.MAX)
            ems = float(et.item())
        h2d = (h_meas.numel() * 8 + h_ant.numel() * 4 + sum(a.numel() for a in h_axes) * 4
               + h_rxo.numel() * 4)
        d2h = h_img.numel() * 8 + h_nrm.numel() * 4
        e2e = {"value": world * updates / (ems * 1e-3) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": h2d * world, "d2h_bytes_per_step": d2h * world,
               "ms_per_step": ems,
               "path": "pinned host -> ops.backproject + image_max_abs (+ all-reduce) + "
                       "surface_normals_from_max (C ABI) -> pinned host image + unit normals"}

    # the reference-facing call a mmNorm user makes (image_processor.py:383-396's image and
    # normals in one call, numpy in and out), on rank 0 of a single-GPU run
    e2e_dropin = None
    if rank == 0 and world == 1 and not args.no_e2e:
        from mmnorm_b200 import pipeline
        radar = sc.meas[:, :, None]
        args_d = (sc.x_locs, sc.y_locs, sc.z_locs, sc.antenna_locs.astype(np.float64), radar,
                  np.zeros((1, 3)), sc.slope, sc.wavelength, sc.slope * (F - 1), F)
        pipeline.surface_normals(*args_d, use_4_rx=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pipeline.surface_normals(*args_d, use_4_rx=True)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        e2e_dropin = {"value": updates / dt / 1e9, "unit": UNIT, "seconds": dt,
                      "path": "pipeline.surface_normals (image_cuda + normal_estimates_cuda "
                              "semantics): numpy inputs -> complex64 image, float64 unit "
                              "normals with NaN, phase centres; wall clock, one call"}

    interp = None
    if rank == 0 and world == 1 and not args.no_interp:
        interp = time_interp(dev, sc)
    reference_cuda = None
    if rank == 0 and world == 1 and not args.no_reference_cuda and args.aperture == 128:
        reference_cuda = time_reference_cuda_full(dev, sc)
    next_rows = None
    if rank == 0 and world == 1 and not args.no_next_rows:
        next_rows = time_next_rows(dev)
    accuracy = None
    if acc_mixed is not None:
        accuracy = accuracy_report(dev, sc, acc_idx, acc_mixed[0],
                                   acc_plain[0] if acc_plain else None, acc_mixed[1],
                                   acc_plain[1] if acc_plain else None)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import ref_imager
            if ref_imager.available():
                rate, info = time_reference_imager(sc, 1, 0, args.cpu_seconds)
                cpu = {"value": rate / 1e9, "unit": UNIT, "cores": info["threads"],
                       "kind": "reference", "sample": info["sample"]}
        except Exception as e:  # pragma: no cover
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                   "sample": "failed: %s" % str(e)[:200]}

    sms = torch.cuda.get_device_properties(dev).multi_processor_count

    def lane_bounds(rate, updates_per_sm_clock):
        """Fraction of an SM-count x clock x issue-width bound, at the sampled loaded clock
        and at the maximum clock."""
        out = {}
        for label, mhz in (("at_sampled_clock", clk.get("sm_mhz")),
                           ("at_max_clock", clk.get("sm_max_mhz"))):
            if mhz:
                bound = sms * mhz * 1e6 * updates_per_sm_clock
                out[label] = {"sm_mhz": mhz, "bound_G_updates_per_s": bound / 1e9,
                              "frac": rate / bound}
        return out

    if "plain" in out:
        # 16 SFU results per SM per clock, sin + cos per update
        out["plain"]["sfu_bound"] = lane_bounds(updates / (out["plain"]["kernel_ms"] * 1e-3),
                                                16 / 2)

    numpy_cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the same formula in NumPy (FP64 and FP32) on all host cores, a seeded voxel sample
        try:
            from oracle import numpy_baseline
            idx = np.sort(np.random.default_rng(5).choice(sc.num_voxels, 8192, replace=False))
            res = {}
            for prec in ("f64", "f32"):
                r = numpy_baseline.time_sample(sc.voxel_centres(idx), sc.antenna_locs,
                                               np.zeros((1, 3), np.float32), sc.meas,
                                               sc.wavelength, sc.slope,
                                               target_seconds=0.4 * args.cpu_seconds,
                                               precision=prec)
                res[prec] = {"value": r["updates_per_s"] / 1e9, "unit": UNIT,
                             "cores": r["workers"], "kind": "port",
                             "sample": "%d seeded random voxels of the 128^3 grid x all %d "
                                       "antennas x %d freqs, %s NumPy (oracle.full_np) in "
                                       "%d spawn processes, %.1f s"
                                       % (r["voxels"], A, F, prec.upper(), r["workers"],
                                          r["seconds"])}
            numpy_cpu = dict(res["f64"], f32=res["f32"])
        except Exception as e:  # pragma: no cover
            numpy_cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                         "sample": "failed: %s" % str(e)[:200]}

    if rank == 0:
        flops = 8.0 * updates          # one complex multiply-add (4 FFMA) per update
        achieved = flops / kern_avg_s / 1e12
        peak = fp32_peak / 1e12
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup),
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "precision": precision_text(variant["name"]),
            "data": "synthetic (seeded point-scatterer scene, exp(-j4pi f r/c)/r^2, 15 dB)",
            "config": {"workload": sc.name + " (128^3 voxels @2 mm, 128x128 antennas @2 mm, "
                       "256 freqs 77-81 GHz; image + vote + unit normals)",
                       "voxels": V * world, "voxels_per_gpu": V, "antennas": A, "freqs": F,
                       "parallelism": ("voxel slabs: %d x-planes of a %d x %d x %d grid per "
                                       "GPU, one all-reduce(MAX) of max|I| per step"
                                       % (xs.numel(), nx_total, ys.numel(), zs.numel()))
                       if world > 1 else "single GPU",
                       "l2": "flushed before every step (256 MB write)",
                       "plan": plan, "variant": variant["name"],
                       "autotune_ms": tuned["times_ms"]},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak,
                         "traffic": FWD_DRAM_BYTES_PER_LAUNCH.get(variant["name"]) if args.aperture == 128
                         else None,
                         "traffic_source": "one full-size ncu capture of this variant "
                                           "(profiles/bp_fwd_kernel_dram_boxcyl128.md)",
                         "kernel": "bp_fwd_kernel " + variant["name"],
                         "flops_per_update": 8,
                         "peak_source": "FP32 FFMA probe (mmn_fp32_peak_probe) timed in this "
                                        "run; MEASURED_PEAKS.json has no FP32 figure",
                         "kernel_ms": statistics.mean(kern_ms),
                         # 128 FP32 lanes per SM per clock.  The Horner form costs 4 FMA
                         # lane-ops per update; a phasor-rotation form (rotate, then
                         # multiply-add) costs 8, so this kernel can exceed that bound
                         "fp32_lane_bound_4_ops": lane_bounds(updates / kern_avg_s, 128 / 4),
                         "fp32_lane_bound_8_ops": lane_bounds(updates / kern_avg_s, 128 / 8)},
            "clocks": clk,
            "e2e": e2e,
            "e2e_dropin": e2e_dropin,
            "gpu_launches": launches_per_step * args.steps,
            "cpu_baseline": cpu,
            "numpy_baseline": numpy_cpu,
            "adjoint": adjoint,
            "batched": batched,
            "interp": interp,
            "reference_cuda": reference_cuda,
            "accuracy": accuracy,
            "next_rows": next_rows,
        }
        line.update(out)
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def time_adjoint(dev):
    """Forward vs backward cost on the differentiation workload (64^3 voxels @3 mm,
    64x64 antennas @3 mm, 128 frequencies, sphere scene): device time of the fused
    forward (image + vote) and of the adjoint (measurement + position gradients)."""
    import torch
    from mmnorm_b200 import ops, scenes
    sc = scenes.config3(sign=+1, device=dev)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    args = [t(sc.x_locs), t(sc.y_locs), t(sc.z_locs), t(sc.antenna_locs),
            t(np.zeros((1, 3), np.float32)), t(sc.meas)]
    rng = np.random.default_rng(3)
    pos = t(rng.normal(0, 5e-4, sc.antenna_locs.shape).astype(np.float32))
    V = sc.num_voxels
    gI = t((rng.standard_normal(V) + 1j * rng.standard_normal(V)).astype(np.complex64))
    gW = t((rng.standard_normal((3, V)) + 1j * rng.standard_normal((3, V))).astype(np.complex64))
    stream = torch.cuda.current_stream(dev)

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return best

    fwd = timed(lambda: ops.backproject(*args, sc.wavelength, sc.slope, pos_offsets=pos))
    bwd = timed(lambda: ops.backproject_backward(*args, sc.wavelength, sc.slope, gI, gW,
                                                 pos_offsets=pos))
    bwd_m = timed(lambda: ops.backproject_backward(*args, sc.wavelength, sc.slope, gI, gW,
                                                   pos_offsets=pos, want_pos=False))
    bwd_p = timed(lambda: ops.backproject_backward(*args, sc.wavelength, sc.slope, gI, gW,
                                                   pos_offsets=pos, want_meas=False))
    # a loss on the image only (no vote term): the passes skip the vote terms
    bwd_i = timed(lambda: ops.backproject_backward(*args, sc.wavelength, sc.slope, gI, None,
                                                   pos_offsets=pos))
    # both passes in their sum-over-samples / sum-over-voxels forms, for comparison
    ops.set_position_pass("horner")
    ops.set_measurement_pass("horner")
    try:
        hor = timed(lambda: ops.backproject_backward(*args, sc.wavelength, sc.slope, gI, gW,
                                                     pos_offsets=pos))
        hor_m = timed(lambda: ops.backproject_backward(*args, sc.wavelength, sc.slope, gI, gW,
                                                       pos_offsets=pos, want_pos=False))
        hor_p = timed(lambda: ops.backproject_backward(*args, sc.wavelength, sc.slope, gI, gW,
                                                       pos_offsets=pos, want_meas=False))
    finally:
        ops.set_position_pass("interp")
        ops.set_measurement_pass("interp")
    return {"workload": sc.name + " (64^3 voxels @3 mm, 64x64 antennas @3 mm, 128 freqs)",
            "forward_ms": fwd, "backward_ms": bwd, "backward_over_forward": bwd / fwd,
            "backward_meas_ms": bwd_m, "backward_pos_ms": bwd_p,
            "passes": "interpolation form (8-cell kernel, 2x oversampled per-antenna grids): "
                      "type-2 gather for the position pass, type-1 spread for the "
                      "measurement pass",
            "backward_image_loss_ms": bwd_i, "backward_image_loss_over_forward": bwd_i / fwd,
            "horner_passes": {"backward_ms": hor, "backward_meas_ms": hor_m,
                              "backward_pos_ms": hor_p, "backward_over_forward": hor / fwd}}


def time_batched(dev, replays=3):
    """24 uneven objects (grids 32^3-96^3, apertures 32^2-96^2 at 2-4 mm, 64-256
    frequencies) in one persistent, graph-captured launch: aggregate updates/s, the same
    objects launched one by one, and the worst per-object deviation between the two."""
    import torch
    from mmnorm_b200 import autotune, ops, scenes
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    scs = scenes.config4_objects(sign=-1, device=dev)
    objs = [dict(x_locs=t(sc.x_locs), y_locs=t(sc.y_locs), z_locs=t(sc.z_locs),
                 antenna_locs=t(sc.antenna_locs), rx_offsets=t(np.zeros((1, 3), np.float32)),
                 meas=t(sc.meas), wavelength=sc.wavelength, slope=sc.slope) for sc in scs]
    updates = sum(sc.updates for sc in scs)
    single_variant = ops.current_variant("mixed")
    tuned = autotune.tune_batched(objs)
    plan = ops.BatchPlan(objs, items_per_slot=tuned["best"])
    plan.capture()
    plan.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(replays):
        plan.replay()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / replays
    # one by one, same kernels, for the comparison and the per-object check
    worst = 0.0
    i0, i1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    i0.record()
    singles = [ops.backproject(o["x_locs"], o["y_locs"], o["z_locs"], o["antenna_locs"],
                               o["rx_offsets"], o["meas"], o["wavelength"], o["slope"])
               for o in objs]
    i1.record()
    torch.cuda.synchronize()
    ms_single = i0.elapsed_time(i1)
    for (img, vote), (si, sv) in zip(plan.results(), singles):
        for a, b in ((img, si), (vote, sv)):
            worst = max(worst, float((a - b).abs().norm() / b.abs().norm()))
    info = plan.info()
    ops.set_variant("mixed", single_variant)  # the other legs keep the workload's pick
    return {"objects": len(objs), "updates": updates, "ms": ms,
            "value": updates / (ms * 1e-3) / 1e9, "unit": UNIT,
            "one_by_one_ms": ms_single, "one_by_one_value": updates / (ms_single * 1e-3) / 1e9,
            "max_rel_l2_vs_one_by_one": worst, "items": info["items"], "ctas": info["ctas"],
            "items_per_slot": tuned["best"], "variant": tuned["variant"],
            "autotune_ms": tuned["times_ms"],
            "graph": "captured once, replayed"}


def _event_ms(fn, reps=3, warm=1):
    """CUDA-event times (ms) of `fn` on the current stream: `warm` untimed calls, then
    `reps` timed ones; returns the list."""
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    out = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        out.append(e0.elapsed_time(e1))
    return out


def _wall_ms(fn, reps=2, warm=1):
    """Host wall-clock times (ms) of a synchronous call, synchronised on both sides."""
    import torch
    for _ in range(warm):
        fn()
    out = []
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        out.append(1e3 * (time.perf_counter() - t0))
    return out


def _central_antennas(n_side, full_side=128):
    n0 = (full_side - n_side) // 2
    return (np.arange(n0, n0 + n_side)[:, None] * full_side +
            np.arange(n0, n0 + n_side)[None, :]).ravel()


def time_reference_cuda_full(dev, sc, target_ms=1000.0):
    """The reference's own CUDA kernel (cuda_image, full matched filter: FP32 range, FP64
    phase and FP64 sin + cos per update, imaging_gpu.cu:106-117), compiled unmodified for
    sm_100a and launched as py_image_gpu.py:272-274 does (block 512, grid V/512 + 1), on the
    WHOLE 128^3 grid -- so it fills the GPU as it would in use -- with a central n x n
    subset of the aperture sized so that one reference launch takes about `target_ms`.
    mmn_cuda_image (the drop-in entry with the reference's argument list, mixed form) runs
    on the same inputs.  Kernel-only CUDA-event times, and end to end: the reference with
    its per-call pycuda transfers (allocation + synchronous copies from pageable memory,
    oracle/ref_cuda.cuda_image_in_out), ours through mmn_cuda_image from the same pageable
    arrays."""
    import torch
    from mmnorm_b200 import _lib, ops
    from oracle import ref_cuda
    if not ref_cuda.available():
        return {"unavailable": "reference cubins not built (oracle/build.py needs the mmNorm "
                               "checkout at build time)"}
    nx, ny, nz = sc.grid_shape
    V = nx * ny * nz
    F = sc.meas.shape[1]
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    x, y, z = t(sc.x_locs), t(sc.y_locs), t(sc.z_locs)
    rxo = t(np.zeros(3, np.float32))
    wl, sl = np.float32(sc.wavelength), np.float32(sc.slope)
    lib = _lib.load()
    vp = ops._vp

    def inputs(n_side):
        idx = _central_antennas(n_side)
        ant = np.ascontiguousarray(sc.antenna_locs[idx])
        m = sc.meas[idx]
        return (idx.size, ant, np.ascontiguousarray(m.real.reshape(-1)),
                np.ascontiguousarray(m.imag.reshape(-1)))

    def ref_kernel_ms(n_side, reps):
        A, ant, mr, mi = inputs(n_side)
        pr, pi = torch.zeros(V, device=dev), torch.zeros(V, device=dev)
        ta, tr, ti_ = t(ant.reshape(-1)), t(mr), t(mi)
        ms = _event_ms(lambda: ref_cuda.cuda_image(pr, pi, x, y, z, ta, tr, ti_, rxo, sl, wl,
                                                   0.0, nx, ny, nz, A, 1, F, 0, 0),
                       reps=reps, warm=0 if reps == 1 else 1)
        return ms, (pr, pi)

    # calibrate on 4 x 4 antennas, then size the subset for ~target_ms per launch
    cal, _ = ref_kernel_ms(4, 1)
    n_side = int(max(4, min(128, math.floor(math.sqrt(16 * target_ms / max(cal[0], 1e-3))))))
    A, ant, mr, mi = inputs(n_side)
    ref_ms, (pr, pi) = ref_kernel_ms(n_side, 2)
    ta, tr, ti_ = t(ant.reshape(-1)), t(mr), t(mi)
    ws_n = lib.mmn_cuda_image_workspace_bytes_for(nx, ny, nz, A, F, 0, -1, 0)
    ws = torch.empty(ws_n, dtype=torch.uint8, device=dev)
    qr, qi = torch.zeros(V, device=dev), torch.zeros(V, device=dev)

    def ours():
        _lib.check(lib.mmn_cuda_image(vp(qr), vp(qi), vp(x), vp(y), vp(z), vp(ta), vp(tr),
                                      vp(ti_), vp(rxo), float(sl), float(wl), 0.0, nx, ny, nz,
                                      A, 1, F, 0, 0, 0, -1, vp(ws), ws_n, ops._stream(dev)),
                   "mmn_cuda_image")

    ours_ms = _event_ms(ours, reps=3)
    upd = V * A * F
    a = pr.cpu().numpy().astype(np.float64) + 1j * pi.cpu().numpy()
    b = qr.cpu().numpy().astype(np.float64) + 1j * qi.cpu().numpy()
    rel = float(np.linalg.norm(a - b) / np.linalg.norm(a))
    # end to end, host numpy in and out every call
    hx, hy, hz = sc.x_locs, sc.y_locs, sc.z_locs
    hant, hrxo = ant.reshape(-1), np.zeros(3, np.float32)
    ref_e2e = _wall_ms(lambda: ref_cuda.cuda_image_in_out(hx, hy, hz, hant, mr, mi, hrxo, sl, wl,
                                                          0.0, A, 1, F, 0, 0), reps=1, warm=0)
    out_r, out_i = np.empty(V, np.float32), np.empty(V, np.float32)

    def ours_e2e():
        dx, dy, dz, da, dr, di, do = (torch.from_numpy(np.asarray(h)).to(dev)
                                      for h in (hx, hy, hz, hant, mr, mi, hrxo))
        ox, oi = torch.empty(V, device=dev), torch.empty(V, device=dev)
        w = torch.empty(ws_n, dtype=torch.uint8, device=dev)
        _lib.check(lib.mmn_cuda_image(vp(ox), vp(oi), vp(dx), vp(dy), vp(dz), vp(da), vp(dr),
                                      vp(di), vp(do), float(sl), float(wl), 0.0, nx, ny, nz, A,
                                      1, F, 0, 0, 0, -1, vp(w), ws_n, ops._stream(dev)),
                   "mmn_cuda_image")
        out_r[:] = ox.cpu().numpy()
        out_i[:] = oi.cpu().numpy()

    ours_e2e_ms = _wall_ms(ours_e2e, reps=3)
    r_ms, o_ms = min(ref_ms), min(ours_ms)
    re_ms, oe_ms = min(ref_e2e), min(ours_e2e_ms)
    return {
        "what": "reference cuda_image full matched filter vs mmn_cuda_image (mixed) on the "
                "whole 128^3 grid with the central %dx%d antennas x %d freqs" % (n_side, n_side, F),
        "antennas": A, "updates": upd, "launch": "reference: block 512, grid %d" % (V // 512 + 1),
        "reference_kernel_ms": r_ms, "reference_G_updates_per_s": upd / r_ms / 1e6,
        "ours_kernel_ms": o_ms, "ours_G_updates_per_s": upd / o_ms / 1e6,
        "kernel_speedup": r_ms / o_ms,
        "reference_e2e_ms": re_ms, "reference_e2e_G_updates_per_s": upd / re_ms / 1e6,
        "ours_e2e_ms": oe_ms, "ours_e2e_G_updates_per_s": upd / oe_ms / 1e6,
        "e2e_speedup": re_ms / oe_ms,
        "e2e_path": "reference: pycuda drv.In/Out pattern (cuMemAlloc + synchronous copies from "
                    "pageable numpy, launch, copy back, free); ours: mmn_cuda_image with torch "
                    "device buffers from the same pageable arrays; host wall clock",
        "rel_l2_ours_vs_reference": rel}


def time_interp(dev, sc, nbins=4096):
    """Interpolated mode, the reference's shipped default (src/utils/params.json:4), on the
    whole workload: the 256-sample measurements zero-padded to a 4096-bin range FFT
    (image_processor.py:22-35, here torch.fft on the device), 2.1M voxels x 16384 antennas.
    The reference's own cuda_image (interpolated branch) and cuda_sn_est against this
    library's bit-exact kernels and the fast form, kernel-only CUDA events; the fast form
    also fused with the vote in one pass; end to end with the reference's per-call pycuda
    transfers vs ours from the same pageable arrays."""
    import torch
    from mmnorm_b200 import _lib, ops
    from oracle import ref_cuda
    nx, ny, nz = sc.grid_shape
    V = nx * ny * nz
    A, F = sc.meas.shape
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    x, y, z = t(sc.x_locs), t(sc.y_locs), t(sc.z_locs)
    ant = t(sc.antenna_locs)
    rxo = t(np.zeros((1, 3), np.float32))
    pad = torch.zeros((A, nbins), dtype=torch.complex64, device=dev)
    pad[:, :F] = t(sc.meas)
    fft = torch.fft.fft(pad, dim=1)
    del pad
    mr, mi = fft.real.contiguous().reshape(-1), fft.imag.contiguous().reshape(-1)
    fsp = np.float32(3e8 / (2 * (sc.f_hi - sc.f_lo)) * F / nbins)
    wl, sl = np.float32(sc.wavelength), np.float32(sc.slope)
    lib = _lib.load()
    vp = ops._vp
    ws = torch.empty(256, dtype=torch.uint8, device=dev)
    qr, qi = torch.zeros(V, device=dev), torch.zeros(V, device=dev)

    def ours(flag, out_r=qr, out_i=qi):
        _lib.check(lib.mmn_cuda_image(vp(out_r), vp(out_i), vp(x), vp(y), vp(z), vp(ant),
                                      vp(mr), vp(mi), vp(rxo), float(sl), float(wl), float(fsp),
                                      nx, ny, nz, A, 1, nbins, 0, 0, flag, -1, vp(ws), 256,
                                      ops._stream(dev)),
                   "mmn_cuda_image")

    pairs = V * A
    out = {"what": "interpolated mode, 128^3 voxels x 16384 antennas, %d-bin range FFT" % nbins,
           "pairs": pairs}
    exact_ms = _event_ms(lambda: ours(1))
    exact = torch.complex(qr, qi).clone()
    rel = lambda a, b: float((a.to(torch.complex128) - b.to(torch.complex128)).norm() /
                             b.to(torch.complex128).norm())
    forms = {}
    for form in ("scalar", "packed"):  # the default form last
        ops.set_interp_fast_form(form)
        f_ms = _event_ms(lambda: ours(2))
        forms[form] = {"ms": min(f_ms),
                       "rel_l2_vs_exact": rel(torch.complex(qr, qi), exact)}
    fast_ms = [forms["packed"]["ms"]]
    fast = torch.complex(qr, qi).clone()
    out["fast_forms"] = forms
    out["ours_exact_ms"] = min(exact_ms)
    out["ours_fast_ms"] = min(fast_ms)
    out["fast_rel_l2_vs_exact"] = rel(fast, exact)
    img_f, vote_f = ops.backproject(x, y, z, ant, rxo, fft, float(wl), float(sl),
                                    mode="interp_fast", fft_spacing=float(fsp))
    fused_ms = _event_ms(lambda: ops.backproject(x, y, z, ant, rxo, fft, float(wl), float(sl),
                                                 mode="interp_fast", fft_spacing=float(fsp)))
    out["ours_fast_fused_image_vote_ms"] = min(fused_ms)
    del img_f, vote_f
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    # 3 MUFU results per pair (square-root seed, sine, cosine) at 16 per SM per clock
    out["fast_mufu_bound"] = {"mufu_per_pair": 3, "sm_count": sms,
                              "bound_pairs_per_s_at_1965MHz": sms * 16 / 3 * 1.965e9,
                              "frac": pairs / (min(fast_ms) * 1e-3) / (sms * 16 / 3 * 1.965e9)}
    if ref_cuda.available():
        pr, pi = torch.zeros(V, device=dev), torch.zeros(V, device=dev)
        ref_ms = _event_ms(lambda: ref_cuda.cuda_image(pr, pi, x, y, z, ant.reshape(-1), mr, mi,
                                                       rxo.reshape(-1), sl, wl, fsp, nx, ny, nz,
                                                       A, 1, nbins, 0, 1))
        torch.cuda.synchronize()
        out["reference_kernel_ms"] = min(ref_ms)
        out["exact_bit_identical_to_reference"] = bool(torch.equal(pr, exact.real) and
                                                       torch.equal(pi, exact.imag))
        out["exact_speedup"] = min(ref_ms) / min(exact_ms)
        out["fast_speedup"] = min(ref_ms) / min(fast_ms)
        out["fast_rel_l2_vs_reference"] = rel(fast, torch.complex(pr, pi))
        # normal vote over the masked voxels (py_sn_est_gpu.py:326-333)
        img = torch.complex(pr, pi).reshape(nx, ny, nz)
        mag = img.abs()
        coords = torch.nonzero(mag > mag.max() * 0.05).to(torch.int32)
        nv = int(coords.shape[0])
        vx, vy, vz = (coords[:, k].contiguous() for k in range(3))
        out["normals"] = {"valid_voxels": nv}
        outs = {}
        for which in ("reference", "exact", "fast"):
            n = [torch.zeros(nv, device=dev) for _ in range(3)]
            if which == "reference":
                fn = lambda n=n: ref_cuda.cuda_sn_est(*n, vx, vy, vz, pr, pi, x, y, z,
                                                      ant.reshape(-1), mr, mi, rxo.reshape(-1),
                                                      sl, wl, fsp, nx, ny, nz, A, 1, nv, nbins,
                                                      0)
            else:
                entry = lib.mmn_cuda_sn_est if which == "exact" else lib.mmn_cuda_sn_est_fast
                fn = lambda n=n, entry=entry: _lib.check(entry(
                    vp(n[0]), vp(n[1]), vp(n[2]), vp(vx), vp(vy), vp(vz), vp(pr), vp(pi), vp(x),
                    vp(y), vp(z), vp(ant), vp(mr), vp(mi), vp(rxo), float(sl), float(wl),
                    float(fsp), nx, ny, nz, A, 1, nv, nbins, 0, 0, -1, vp(ws), 256,
                    ops._stream(dev)), "mmn_cuda_sn_est")
            out["normals"][which + "_ms"] = min(_event_ms(fn))
            outs[which] = torch.stack(n, 1)
        out["normals"]["exact_bit_identical_to_reference"] = bool(
            torch.equal(outs["exact"], outs["reference"]))
        out["normals"]["fast_rel_l2_vs_reference"] = rel(outs["fast"], outs["reference"])
        out["normals"]["fast_speedup"] = out["normals"]["reference_ms"] / out["normals"]["fast_ms"]
        # end to end (image), host numpy in and out every call
        hx, hy, hz = sc.x_locs, sc.y_locs, sc.z_locs
        hant = np.ascontiguousarray(sc.antenna_locs.reshape(-1))
        hmr, hmi = mr.cpu().numpy(), mi.cpu().numpy()
        hrxo = np.zeros(3, np.float32)
        ref_e2e = _wall_ms(lambda: ref_cuda.cuda_image_in_out(hx, hy, hz, hant, hmr, hmi, hrxo, sl,
                                                              wl, fsp, A, 1, nbins, 0, 1))
        o_r, o_i = np.empty(V, np.float32), np.empty(V, np.float32)

        def ours_e2e(flag):
            dx, dy, dz, da, dr, di, do = (torch.from_numpy(np.asarray(h)).to(dev)
                                          for h in (hx, hy, hz, hant, hmr, hmi, hrxo))
            ox, oi = torch.empty(V, device=dev), torch.empty(V, device=dev)
            _lib.check(lib.mmn_cuda_image(vp(ox), vp(oi), vp(dx), vp(dy), vp(dz), vp(da),
                                          vp(dr), vp(di), vp(do), float(sl), float(wl),
                                          float(fsp), nx, ny, nz, A, 1, nbins, 0, 0, flag, -1,
                                          vp(ws), 256, ops._stream(dev)), "mmn_cuda_image")
            o_r[:] = ox.cpu().numpy()
            o_i[:] = oi.cpu().numpy()

        out["e2e"] = {"reference_ms": min(ref_e2e),
                      "ours_exact_ms": min(_wall_ms(lambda: ours_e2e(1))),
                      "ours_fast_ms": min(_wall_ms(lambda: ours_e2e(2))),
                      "h2d_bytes": int(hmr.nbytes + hmi.nbytes + hant.nbytes + 4 * (nx + ny + nz)),
                      "d2h_bytes": 8 * V,
                      "path": "reference: pycuda drv.In/Out pattern; ours: mmn_cuda_image from "
                              "the same pageable arrays; host wall clock"}
        out["e2e"]["fast_speedup"] = out["e2e"]["reference_ms"] / out["e2e"]["ours_fast_ms"]
        del hmr, hmi
        out["stage_tail"] = time_stage_tail(dev, sc, nbins)
    else:
        out["reference"] = "unavailable: reference cubins not built"
    return out


def time_stage_tail(dev, sc, nbins):
    """The whole tail of generate_mmwave_surface_normals in interpolated mode
    (image_processor.py:383-396), host arrays in and out, three ways: the reference's
    (numpy range FFT + reference_dropin_calls: its two CUDA kernels with their per-call
    transfers and its host steps); the same numpy FFT followed by this library's drop-in
    image_cuda / normal_estimates_cuda in their place (what swapping the two imports at
    image_processor.py:10-14 gives); and stage1.generate_mmwave_surface_normals (range FFT,
    image and normals on the device).  Bit-exact and fast forms; host wall clock, and the
    agreement of the outputs with the reference's.  The reference's host steps are restated
    in oracle/ref_pipeline.py."""
    from mmnorm_b200 import py_image_gpu, py_sn_est_gpu, stage1
    from oracle.ref_pipeline import range_fft_host, reference_dropin_calls
    A, S = sc.meas.shape
    radar = np.ascontiguousarray(sc.meas.reshape(A, S, 1))
    rxo = np.zeros((1, 3), np.float32)
    x, y, z = sc.x_locs, sc.y_locs, sc.z_locs
    locs = np.asarray(sc.antenna_locs, np.float32)
    wl, sl = np.float32(sc.wavelength), np.float32(sc.slope)
    bw = sc.f_hi - sc.f_lo
    res = {}

    def ref():
        bins = range_fft_host(radar, nbins)
        res["ref"] = reference_dropin_calls(x, y, z, locs, bins, rxo, sl, wl, bw, S)

    def dropin(precision):
        bins = range_fft_host(radar, nbins)
        img, _ = py_image_gpu.image_cuda(x, y, z, locs, bins, rxo, float(sl), float(wl), bw, S,
                                         use_4_rx=True, use_interpolated_processing=True,
                                         precision=precision)
        nrm = py_sn_est_gpu.normal_estimates_cuda(img, x, y, z, locs, bins, rxo, float(sl),
                                                  float(wl), bw, S, use_4_rx=True,
                                                  precision=precision)
        nrm /= np.linalg.norm(nrm, axis=-1)[..., np.newaxis].repeat(3, axis=-1)
        res["dropin_" + precision] = (img, nrm)

    def ours(precision):
        out = stage1.generate_mmwave_surface_normals(
            x, y, z, locs, radar, rxo, float(sl), float(wl), bw, S, is_ti_radar=False,
            use_interpolated_processing=True, precision=precision)
        res["stage1_" + precision] = (out[0], out[2])

    fft_ms = min(_wall_ms(lambda: range_fft_host(radar, nbins), reps=2, warm=0))
    ref_ms = min(_wall_ms(ref, reps=2, warm=0))
    out = {"what": "generate_mmwave_surface_normals tail, interpolated mode: %d-bin range FFT, "
                   "image, normals at 5 %% of max|I|, unit normalisation; host arrays in and out"
                   % nbins,
           "reference_ms": ref_ms, "numpy_fft_ms": fft_ms,
           "reference": "numpy FFT + the reference's cuda_image / cuda_sn_est built from "
                        "source, pycuda transfer pattern, its host steps"}
    for key, prec in (("exact", "exact"), ("fast", "fast")):
        out["dropin_%s_ms" % key] = min(_wall_ms(lambda: dropin(prec), reps=2, warm=1))
    out["ours_exact_ms"] = min(_wall_ms(lambda: ours("mixed"), reps=3, warm=1))
    out["ours_fast_ms"] = min(_wall_ms(lambda: ours("fast"), reps=3, warm=1))
    for k in ("dropin_exact", "dropin_fast", "ours_exact", "ours_fast"):
        out[k.replace("ours", "stage1") + "_speedup" if k.startswith("ours") else
            k + "_speedup"] = ref_ms / out[k + "_ms"]
    out["exact_speedup"], out["fast_speedup"] = (out["stage1_exact_speedup"],
                                                 out["stage1_fast_speedup"])
    img_r, nrm_r = res["ref"]
    for key in ("dropin_exact", "dropin_fast", "stage1_mixed", "stage1_fast"):
        img_o, nrm_o = res[key]
        both = np.isfinite(nrm_o).all(-1) & np.isfinite(nrm_r).all(-1)
        cosang = np.clip(np.sum(nrm_o[both] * nrm_r[both], axis=-1), -1.0, 1.0)
        out[key + "_vs_reference"] = {
            "image_rel_l2": float(np.linalg.norm(img_o - img_r) / np.linalg.norm(img_r)),
            "normal_deg_median": float(np.median(np.degrees(np.arccos(cosang)))),
            "mask_agreement": float(np.mean(np.isfinite(nrm_o).all(-1) ==
                                            np.isfinite(nrm_r).all(-1)))}
    return out


def time_next_rows(dev):
    """The steps after the normals, each beside the reference's own path on the same GPU
    or host: (1) isosurface channel simulation at the reference's ray settings (2048 x 2048
    rays, 80 degree fields of view, 512 wavelengths over 77.5-80.5 GHz, TI offset) on a
    200 x 220 x 120 grid at 1 mm holding the RSDF of a 4 cm sphere on a +-8 mm shell, 8
    antennas, against the reference's ray-marching extension (built from source) plus the
    torch steps of _simulate_channels (isosurface_optimization.py:116-208); (2) the RSDF of
    a 3-voxel spherical cap on a 64^3 grid against the sequential breadth-first search of
    sdf.py:122-224 (the restatement pinned to the reference's outputs), and on a 128^3 grid.
    Host wall clock, synchronised, after a warm-up."""
    import torch
    from mmnorm_b200 import isosurface, rsdf
    from oracle import iso_oracle as IO
    from oracle import rsdf_oracle as RO
    C = 2.99792458e8
    out = {}
    vs = 0.001
    x = -0.05 + vs * np.arange(200)
    y = -0.06 + vs * np.arange(220)
    z = -0.40 + vs * np.arange(120)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    r = np.sqrt((X - 0.05) ** 2 + (Y - 0.05) ** 2 + (Z + 0.33) ** 2) - 0.04
    sdf = np.where(np.abs(r) < 0.008, r, -50.0).astype(np.float32)[..., None]
    bbox = [x[0], y[0], z[0], x[-1], y[-1], z[-1]]
    wl = C / np.arange(77.5e9, 80.5e9, 3e9 / 512)
    rng = np.random.default_rng(0)
    A = 8
    loc = np.stack([rng.uniform(0.0, 0.1, A), rng.uniform(0.0, 0.1, A), np.zeros(A)], 1)
    dirs = np.tile(np.array([[0, 0, 1.0]], np.float32), (A, 1))
    W = H = 2048
    fov = 80.0
    scene = isosurface.make_scene(sdf, bbox, vs, wl, W, H, fov, fov, True)
    taus = torch.zeros((1, 1))
    ch = None

    def ours():
        nonlocal ch
        ch = isosurface.simulate_channels_batch(scene, taus, loc, dirs)

    t_ours = min(_wall_ms(ours, reps=3))
    iso = {"grid": list(sdf.shape[:3]), "rays": W * H, "antennas": A, "wavelengths": len(wl),
           "ours_ms": t_ours}
    if IO.available():
        grid = torch.as_tensor(sdf, device=dev)
        wl_t = torch.as_tensor(wl, device=dev)
        refs = []

        def ref():
            refs.clear()
            for a in range(A):
                refs.append(IO.simulate_channels(bbox, vs, W, H, fov, fov, grid,
                                                 torch.as_tensor(loc[a]), dirs[a], wl_t,
                                                 torch.zeros(1), True))

        iso["reference_ms"] = min(_wall_ms(ref, reps=2))
        iso["speedup"] = iso["reference_ms"] / t_ours
        iso["max_rel_l2"] = max(float((ch[0, a] - refs[a]).abs().norm() / refs[a].abs().norm())
                                for a in range(A))
        iso["reference"] = "ray_tracing.cpp + ray_tracing_kernel.cu built from source, torch steps"
    else:
        iso["reference"] = "unavailable: reference ray-marching extension not built"
    out["isosurface"] = iso
    for n in (64, 128):
        c = (n - 1) / 2
        g = np.indices((n, n, n)).astype(np.float64)
        rr = np.sqrt(((g - c) ** 2).sum(0))
        shell = (rr > n * 0.35) & (rr < n * 0.35 + 3) & (g[2] < c + n * 0.1)
        nrm = np.stack([(g[k] - c) / np.maximum(rr, 1e-9) for k in range(3)], -1)
        nrm[~shell] = np.nan
        xs = np.arange(n) * 0.002
        res = {}

        def ours_rsdf():
            res["out"] = rsdf.compute_rsdf(nrm, xs, xs, xs)

        rec = {"voxels_in_mask": int(shell.sum()), "ours_ms": min(_wall_ms(ours_rsdf, reps=2))}
        if n == 64:
            out_g, lab, valid, _ = res["out"]
            t0 = time.perf_counter()
            ref = RO.rsdf(nrm, RO.coords(xs, xs, xs), lab, valid, xs)
            rec["sequential_search_ms"] = 1e3 * (time.perf_counter() - t0)
            rec["speedup"] = rec["sequential_search_ms"] / rec["ours_ms"]
            rec["bit_identical"] = bool(np.array_equal(np.nan_to_num(ref, nan=7.0),
                                                       np.nan_to_num(out_g, nan=7.0)))
        out["rsdf_cap%d" % n] = rec
    return out



def accuracy_report(dev, sc, idx, sub_mixed, sub_plain, max_mixed, max_plain):
    """Relative L2 error of the complex image and the vote, and the median / 95th
    percentile normal angle over the masked voxels, of the mixed and plain forms against
    the FP64 oracle: the workload on a seeded random 4096-voxel subset (from the step's own
    outputs), and config 2 (the 48^3 sphere scene of config 0, 32x32 antennas, 64
    frequencies) on its seeded 4096-voxel subset."""
    import torch
    from mmnorm_b200 import ops, scenes
    from oracle import oracle as O

    def stats(I, W, Io, Wo, max_full):
        sel = np.abs(Io) > 0.05 * max_full
        _, _, raw_o = O.normals_from_vote(Io, Wo, 0.0)
        _, _, raw = O.normals_from_vote(I.astype(np.complex128), W.astype(np.complex128), 0.0)
        ang = O.angle_deg(raw[sel], raw_o[sel])
        return {"image_rel_l2": O.rel_l2(I, Io), "vote_rel_l2": O.rel_l2(W, Wo),
                "normal_deg_median": float(np.median(ang)) if ang.size else None,
                "normal_deg_p95": float(np.percentile(ang, 95)) if ang.size else None,
                "masked_voxels": int(sel.sum())}

    rxo = np.zeros((1, 3))
    t0 = time.perf_counter()
    Io, Wo = O.full(sc.voxel_centres(idx), sc.antenna_locs, rxo, sc.meas, sc.wavelength,
                    sc.slope, phase_mode=1)
    out = {"workload_subset": {"voxels": int(len(idx)), "sign": -1,
                               "mixed": stats(*sub_mixed, Io, Wo, max_mixed)}}
    if sub_plain is not None:
        out["workload_subset"]["plain"] = stats(*sub_plain, Io, Wo, max_plain)
    sc2 = scenes.config0(sign=-1)
    idx2 = np.sort(np.random.default_rng(2).choice(sc2.num_voxels, 4096, replace=False))
    Io2, Wo2 = O.full(sc2.voxel_centres(idx2), sc2.antenna_locs, rxo, sc2.meas, sc2.wavelength,
                      sc2.slope, phase_mode=1)
    tt = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    out["config2"] = {"scene": sc2.name, "voxels": 4096}
    for mode in ("mixed", "plain"):
        img, vote = ops.backproject(tt(sc2.x_locs), tt(sc2.y_locs), tt(sc2.z_locs),
                                    tt(sc2.antenna_locs), tt(np.zeros((1, 3), np.float32)),
                                    tt(sc2.meas), sc2.wavelength, sc2.slope, mode=mode)
        I = img.cpu().numpy().ravel()
        W = vote.cpu().numpy().reshape(3, -1).T
        out["config2"][mode] = stats(I[idx2], W[idx2], Io2, Wo2, float(np.abs(I).max()))
    out["oracle"] = "FP64 C restatement (oracle/bp_oracle.c) on float32-rounded inputs"
    out["oracle_seconds"] = time.perf_counter() - t0
    return out



# DRAM bytes (read + write) of one forward launch at the full workload, by kernel variant:
# one ncu capture of dram__bytes_read.sum + dram__bytes_write.sum on one full-size launch
# (a one-pass metric set, checked on the small case first), summarised in
# profiles/bp_fwd_kernel_dram_boxcyl128.md.  Variants without a capture report null.
FWD_DRAM_BYTES_PER_LAUNCH = {"mixed_antpair_fx2_t1_n256": 38597632 + 37433856,
                             "mixed_clen64_fx2_t4_n128_s24": 40073728 + 36137728,
                             "mixed_clen64_fx2_t4_n128": 40509696 + 36157440,
                             "mixed_clen64eo_fx2_t2_n256": 39280640 + 35329024,
                             "mixed_clen_fx2_t4_n128_s24": 40404992 + 36330240}


def precision_text(variant_name):
    """The arithmetic of a mixed-form kernel variant, for the bench line."""
    if "clen64eo" in variant_name:
        blk = 64
        rec = ("FP32 second-order (Clenshaw) recurrence split into even- and odd-sample "
               "chains in z^2, b_k = m_k + 2cos(2 theta) b_{k+1} - b_{k+2}, h = E + z O; "
               "first-order Horner where |cos 2theta| > 0.98 and on a row's last partial "
               "block")
    elif "clen" in variant_name:
        blk = 64 if "clen64" in variant_name else 32
        rec = ("FP32 second-order (Clenshaw) rotation recurrence b_t = m_t + 2cos(theta) "
               "b_{t+1} - b_{t+2}, first-order Horner where |cos theta| > 0.98")
    elif "split" in variant_name:
        blk = 32
        rec = ("FP32 first-order Horner rotation recurrence, two 16-sample chains per block "
               "joined by z^16")
    else:
        blk = 32
        rec = "FP32 first-order Horner rotation recurrence"
    return ("mixed: FP64 range and phase wrap; %s; re-anchored every %d samples; FP32 "
            "accumulation" % (rec, blk))


def main():
    args = parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    return ours_arm(args)


if __name__ == "__main__":
    sys.exit(main())
