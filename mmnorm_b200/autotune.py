"""Autotuner for the forward kernels' launch shape (voxels per thread x threads per CTA;
the antenna stage size and the antenna split follow from the plan).

Each candidate variant is timed with CUDA events on a reduced copy of the problem: the
same voxel grid and sample count with at most ``max_antennas`` antennas, which keeps the
per-update work of every variant identical to the full problem while bounding the tuning
time.  The winner is cached per (device, mode, padded sample count, voxel-count bucket)
in memory and, optionally, in a JSON file.
"""
from __future__ import annotations

import json
import math
import os

import torch

from . import ops

_cache: dict = {}


def _key(device, mode, nvox, nsamples):
    name = torch.cuda.get_device_name(device)
    fp = (nsamples + 31) // 32 * 32
    vb = int(math.log2(max(1, nvox)))
    return "%s|%s|F%d|V2^%d" % (name, mode, fp, vb)


def load_cache(path):
    if path and os.path.exists(path):
        with open(path) as f:
            _cache.update(json.load(f))


def save_cache(path):
    if path:
        with open(path, "w") as f:
            json.dump(_cache, f, indent=1, sort_keys=True)


# Variant families by accuracy (image relative L2 against FP64 at the 128^3 / 16384-antenna
# / 256-sample workload): the first-order Horner forms ~2.6e-6, the split second-order
# form ~3.4e-6, the single-chain second-order forms 6.8e-6 (32-sample blocks) and 8.8e-6
# (64-sample blocks) -- all within the 1e-4 bound; the faster forms carry more error.
ACCURATE_FORMS = ("mixed_clen64eo_", "mixed_antpair_", "mixed_ffma2_", "mixed_ffma_",
                  "mixed_split_")


def tune(x_locs, y_locs, z_locs, antenna_locs, rx_offsets, meas, wavelength, slope, *,
         mode="mixed", max_antennas=1024, repeats=2, apply=True, verbose=False,
         candidates=None):
    """Times the variants of ``mode`` and (if ``apply``) selects the fastest.
    ``candidates``: variant-name prefixes to consider (default: every variant), e.g.
    ``ACCURATE_FORMS`` to keep the image error near 3e-6 instead of 9e-6.

    The caller's selection is kept when ``apply`` is false, and restored if timing fails.

    Returns {"key", "best", "times_ms": {variant index: ms}}."""
    pool = [v for v in ops.variants(mode)
            if candidates is None or v["name"].startswith(tuple(candidates))]
    if not pool:
        raise ValueError("no %s variant matches the candidates %r" % (mode, candidates))
    dev = meas.device
    nvox = x_locs.numel() * y_locs.numel() * z_locs.numel()
    key = _key(dev, mode, nvox, meas.shape[1])
    if candidates is not None:
        key += "|" + ",".join(sorted(candidates))
    if key in _cache:
        res = _cache[key]
        if apply:
            ops.set_variant(mode, res["best"])
        return res
    A = meas.shape[0]
    n = min(A, max_antennas)
    sel = torch.linspace(0, A - 1, n, device=dev).round().long() if n < A else None
    ant = antenna_locs[sel].contiguous() if sel is not None else antenna_locs
    m = meas[sel].contiguous() if sel is not None else meas
    times = {}
    stream = torch.cuda.current_stream(dev)
    prev = ops.current_variant(mode)
    try:
        for v in pool:
            idx = v["index"]
            ops.set_variant(mode, idx)
            ops.backproject(x_locs, y_locs, z_locs, ant, rx_offsets, m, wavelength, slope,
                            mode=mode)
            best = float("inf")
            for _ in range(repeats):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                ops.backproject(x_locs, y_locs, z_locs, ant, rx_offsets, m, wavelength, slope,
                                mode=mode)
                e1.record(stream)
                torch.cuda.synchronize(dev)
                best = min(best, e0.elapsed_time(e1))
            times[idx] = best
            if verbose:
                print("autotune %s variant %d (%s): %.3f ms" % (mode, idx, v, best))
    finally:
        ops.set_variant(mode, prev)
    best_idx = min(times, key=times.get)
    res = {"key": key, "best": best_idx, "times_ms": {str(k): t for k, t in times.items()},
           "variants": ops.variants(mode), "antennas_timed": n}
    _cache[key] = res
    if apply:
        ops.set_variant(mode, best_idx)
    return res


def tune_batched(objects, options=(4, 8, 16), variants=None, repeats=1, apply=True):
    """Times the batched persistent launch for each (mixed kernel variant, work granularity
    in items per resident CTA) and returns {"best": items_per_slot, "variant": name,
    "times_ms": {"name|items": ms}}.  ``variants``: names to try (default: the current
    variant and the fastest of each block length among the second-order and Horner forms
    that the single-object autotuner would consider), since the objects' sample counts and
    grids differ from the single-object problems the variants were tuned on.  With ``apply`` the
    winning variant is made current (a BatchPlan takes the current variant when built)."""
    names = [v["name"] for v in ops.variants("mixed")]
    cur = ops.current_variant("mixed")
    if variants is None:
        variants = [names[cur]]
        for cand in ("mixed_clen64_fx2_t4_n128_s24", "mixed_clen_fx2_t4_n128_s24",
                     "mixed_antpair_fx2_t1_n256"):
            if cand in names and cand not in variants:
                variants.append(cand)
    times = {}
    for name in variants:
        ops.set_variant("mixed", names.index(name))
        for ips in options:
            plan = ops.BatchPlan(objects, items_per_slot=ips)
            plan.run()
            torch.cuda.synchronize()
            best = float("inf")
            for _ in range(repeats):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                plan.run()
                e1.record()
                torch.cuda.synchronize()
                best = min(best, e0.elapsed_time(e1))
            times[(name, ips)] = best
            del plan
    best_name, best_ips = min(times, key=times.get)
    ops.set_variant("mixed", names.index(best_name) if apply else cur)
    return {"best": best_ips, "variant": best_name,
            "times_ms": {"%s|%d" % k: v for k, v in times.items()}}


def tune_position(x_locs, y_locs, z_locs, antenna_locs, rx_offsets, meas, wavelength, slope,
                  grad_image, grad_vote=None, *, max_antennas=1024, repeats=2, apply=True):
    """Times every launch shape of the interpolation-form position pass (the adjoint's
    antenna-offset gradient) on a reduced copy of the problem -- the same grid and sample
    count, at most ``max_antennas`` antennas, the caller's upstream gradients -- and (if
    ``apply``) selects the fastest.  Cached like ``tune``.

    Returns {"key", "best", "times_ms": {variant index: ms}, "variants": names}."""
    dev = meas.device
    nvox = x_locs.numel() * y_locs.numel() * z_locs.numel()
    key = _key(dev, "position" + ("_vote" if grad_vote is not None else ""), nvox,
               meas.shape[1])
    if key in _cache:
        res = _cache[key]
        if apply:
            ops.set_position_variant(res["best"])
        return res
    A = meas.shape[0]
    n = min(A, max_antennas)
    sel = torch.linspace(0, A - 1, n, device=dev).round().long() if n < A else None
    ant = antenna_locs[sel].contiguous() if sel is not None else antenna_locs
    m = meas[sel].contiguous() if sel is not None else meas
    names = ops.position_variants()
    stream = torch.cuda.current_stream(dev)
    times = {}

    def run():
        ops.backproject_backward(x_locs, y_locs, z_locs, ant, rx_offsets, m, wavelength,
                                 slope, grad_image, grad_vote, want_meas=False)

    prev = ops.current_position_variant()
    try:
        for idx in range(len(names)):
            ops.set_position_variant(idx)
            run()
            best = float("inf")
            for _ in range(repeats):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                run()
                e1.record(stream)
                torch.cuda.synchronize(dev)
                best = min(best, e0.elapsed_time(e1))
            times[idx] = best
    finally:
        ops.set_position_variant(prev)
    best_idx = min(times, key=times.get)
    res = {"key": key, "best": best_idx, "times_ms": {str(k): t for k, t in times.items()},
           "variants": names, "antennas_timed": n}
    _cache[key] = res
    if apply:
        ops.set_position_variant(best_idx)
    return res
