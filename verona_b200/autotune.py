"""Autotuner of the batch kernel: the tile variant (2D tile and 1D pencil
shape) and CTAs per SM of one persistent launch.

A grid search over the candidates, timed with CUDA events on the batch's own
problems; the batch state is checkpointed before and restored after, so
tuning leaves the solution unchanged. Results are cached per (GPU, batch
signature) in a JSON file: $VB_TUNE_CACHE, else ~/.cache/verona_b200/batch_tuning.json.
"""
from __future__ import annotations

import json
import os

from .batch import Batch, variants


def cache_path() -> str:
    return os.environ.get("VB_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "verona_b200",
                                                           "batch_tuning.json")


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _gpu_key():
    import torch

    p = torch.cuda.get_device_properties(torch.cuda.current_device())
    return f"{p.name}/sm{p.major}{p.minor}/{p.multi_processor_count}"


def tune_batch(b: Batch, steps: int = 2, ctas_candidates=(0, 1, 2), use_cache: bool = True, path: str | None = None,
               log=None) -> dict:
    """Pick and apply the fastest (variant, CTAs per SM); returns the choice
    with the timings of every candidate (ms per step)."""
    import torch

    path = path or cache_path()
    key = f"{_gpu_key()}/{b.signature()}"
    if use_cache:
        hit = _load(path).get(key)
        if hit:
            b.set_tuning(hit["variant"], hit["ctas_per_sm"])
            return dict(hit, cached=True)
    shapes = variants(b.precision)
    stream = torch.cuda.current_stream()
    b.checkpoint()
    results = []
    for v in range(len(shapes)):
        for c in ctas_candidates:
            b.set_tuning(v, c)
            b.step(1)  # builds the graph, warms the caches
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            b.step(steps)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
            results.append({"variant": v, "shape": shapes[v], "ctas_per_sm": c, "grid": b.tuning["grid"],
                            "ms_per_step": ms})
            if log:
                log(f"variant {v} {shapes[v]} ctas/SM {c}: {ms:.3f} ms/step")
            b.rollback()
    b.reset_counters()
    best = min(results, key=lambda r: r["ms_per_step"])
    b.set_tuning(best["variant"], best["ctas_per_sm"])
    choice = {"variant": best["variant"], "ctas_per_sm": best["ctas_per_sm"], "shape": best["shape"],
              "ms_per_step": best["ms_per_step"]}
    if use_cache:
        data = _load(path)
        data[key] = choice
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1)
        os.replace(tmp, path)
    return dict(choice, cached=False, candidates=results)
