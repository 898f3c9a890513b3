"""Autotuning with a persistent cache of earlier measurements.

fe_autotune times every candidate shape of the tunable kernels (radix digit
width and keys per thread, the inference grid, threads per block and
persistence of the neighbour kernels) on the context's own device and data
and applies the fastest.  `tune` keeps those choices in a JSON file
keyed by GPU model, SM count, problem size class and key width, so that a
later context of the same class on the same kind of GPU applies the cached
choice without timing anything.
"""
from __future__ import annotations

import json
import math
import os

from . import _abi


def device_key(device: int = 0) -> str:
    """GPU model and SM count of `device` ("unknown" without torch/CUDA)."""
    try:
        import torch
        p = torch.cuda.get_device_properties(device)
        return f"{p.name}|sm{p.multi_processor_count}"
    except Exception:
        return "unknown"


def cache_key(device: str, n: int, table_size: int, learned: bool) -> str:
    size_class = max(0, math.ceil(math.log2(max(n, 1))))
    key_bits = max(1, math.ceil(math.log2(max(table_size, 2))))
    return f"{device}|n2^{size_class}|k{key_bits}|{'learned' if learned else 'plain'}"


def load_cache(path: str | None) -> dict:
    if not path or not os.path.exists(path):
        return {}
    try:
        with open(path) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


def save_cache(path: str, cache: dict) -> None:
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def tune(data, cache_path: str | None = None, *, learned: bool = False,
         device: str | None = None) -> dict:
    """Applies the cached shapes for `data`'s class, or measures them with
    fe_autotune (and stores them when cache_path is given).  Returns
    {"source": "cache" | "measured", "tuning": {...}, "report": {...}?}."""
    dev = device if device is not None else device_key()
    key = cache_key(dev, data.count, data.table_size, learned)
    cache = load_cache(cache_path)
    if key in cache:
        c = cache[key]
        data.set_tuning(_abi.FeTuning.from_dict(c))
        return {"source": "cache", "key": key, "tuning": dict(c)}
    report = data.autotune()
    rd = report.as_dict()
    chosen = rd["chosen"]
    if cache_path:
        cache[key] = chosen
        save_cache(cache_path, cache)
    return {"source": "measured", "key": key, "tuning": chosen, "report": rd}
