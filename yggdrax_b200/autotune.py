"""Autotuner for the pipeline's launch shapes.

The library exposes a few process-wide knobs (``ygx_tune_set``): how the
onesweep sort ranks a tile's keys (warp ballots, per-warp peer tables, or a
per-pass choice by how concentrated the pass's digits are, with its
threshold), its tile shape (keys per thread, CTAs per SM) and its digit
width (8 bits, or 11 bits where that cuts passes: 6 instead of 8 for the
63-bit Morton codes), how many CTAs per SM the traversal walk runs, the
warps per CTA of the leaf refit, and the CTAs per SM of the short-row
finalize.  None of them changes a result.  This module measures candidate
settings on the caller's own workload with CUDA events and keeps the
fastest:

* the 8-bit pass's knobs on the sort of the workload's Morton codes alone (a
  short, low-noise measurement), then
* the other knobs one at a time (coordinate descent) on the whole step --
  the digit width among them, because at 8 bits the Morton encode also
  builds the sort's digit histograms while the 11-bit sort counts its own,
  so only the whole step compares the two fairly.

Results are cached per device and workload signature in a JSON file
(``$YGGDRAX_B200_TUNE_CACHE``, default ``~/.cache/yggdrax_b200/tune.json``)
so a process pays for tuning once.  The reference has no counterpart.
"""

from __future__ import annotations

import json
import os
from typing import Callable, Dict, Iterable, Optional

import numpy as np
import torch

from . import _lib as L

KNOBS = ("sort_rank", "sort_skew", "sort_tile", "sort_bits", "walk_blocks", "refit_warps",
         "row_grid")
SPACE: Dict[str, tuple] = {
    "sort_rank": (0, 1, 2),
    "sort_tile": (0, 1, 2, 3),
    "sort_bits": (8, 11),
    "sort_skew": (8, 16, 32, 64, 128),
    "walk_blocks": (3, 4, 5, 6),
    "refit_warps": (2, 4, 8),
    "row_grid": (4, 8, 16, 32),
}


def current() -> dict:
    """The knobs' present values."""
    lib = L.lib()
    out = {}
    for k in KNOBS:
        v = np.zeros(1, np.int32)
        L.check(lib.ygx_tune_get(L.TUNE[k], v.ctypes.data), "ygx_tune_get")
        out[k] = int(v[0])
    return out


def apply(cfg: dict) -> None:
    """Set the knobs named in ``cfg`` (ValueError on an illegal value)."""
    lib = L.lib()
    for k, v in cfg.items():
        if k not in L.TUNE:
            raise ValueError(f"unknown knob '{k}'")
        if lib.ygx_tune_set(L.TUNE[k], int(v)) != 0:
            raise ValueError(f"illegal value {v} for knob '{k}'")


def _cache_path() -> str:
    return os.environ.get("YGGDRAX_B200_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "yggdrax_b200",
                                       "tune.json"))


def _load_cache() -> dict:
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store_cache(key: str, cfg: dict) -> None:
    data = _load_cache()
    data[key] = cfg
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # an unwritable cache only costs a re-tune


def signature(dev: torch.device, kind: str, n: int, **params) -> str:
    """Cache key: device name, workload kind, size bucket (power of two) and
    the parameters that change the work (leaf size, MAC, theta, sets)."""
    name = torch.cuda.get_device_name(dev).replace(" ", "_")
    bucket = int(np.ceil(np.log2(max(n, 1))))
    extra = ",".join(f"{k}={params[k]}" for k in sorted(params))
    return f"{name}|{kind}|n2^{bucket}|{extra}"


def time_ms(fn: Callable[[], object], dev: torch.device, reps: int = 3, warmup: int = 1) -> float:
    """Median CUDA-event time of ``fn`` on the current stream."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize(dev)
    ts = []
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize(dev)
        ts.append(a.elapsed_time(b))
    return float(np.median(ts))


def _sort_step(codes: torch.Tensor, dev: torch.device) -> Callable[[], None]:
    lib = L.lib()
    n = int(codes.numel())
    ws = L.workspace(lib.ygx_sort_pairs_workspace_size(n), dev)
    ko = torch.empty_like(codes)
    vo = torch.empty(n, dtype=torch.int32, device=dev)
    st = L.stream_handle(dev)

    def run():
        L.check(lib.ygx_sort_pairs(L.ptr(codes), None, n, 0, 63, L.ptr(ko), L.ptr(vo),
                                   L.ptr(ws), ws.numel(), st), "ygx_sort_pairs")
    return run


def tune(step: Callable[[], object], dev: torch.device, *, codes: Optional[torch.Tensor] = None,
         knobs: Iterable[str] = ("sort_bits", "walk_blocks", "refit_warps", "row_grid"),
         reps: int = 3,
         log: Optional[list] = None) -> dict:
    """Choose knob values for ``step`` (a callable that runs the workload
    once).  With ``codes`` (the workload's Morton codes) the sort knobs are
    chosen first on the sort alone.  Returns the chosen configuration (also
    applied); ``log`` (a list) receives every (config, ms) measured."""
    best = current()
    if codes is not None:
        run = _sort_step(codes, dev)
        results = []
        best["sort_bits"] = 8  # the rank and tile knobs shape the 8-bit pass
        for rank in SPACE["sort_rank"]:
            for skew in (SPACE["sort_skew"] if rank == 2 else (best["sort_skew"],)):
                cfg = dict(best, sort_rank=rank, sort_skew=skew)
                apply(cfg)
                ms = time_ms(run, dev, reps=max(reps, 5))
                results.append((ms, cfg))
                if log is not None:
                    log.append({"stage": "sort", "config": cfg, "ms": ms})
        best = min(results, key=lambda r: r[0])[1]
        base_sort = min(r[0] for r in results)
        for tile in SPACE["sort_tile"]:
            if tile == best["sort_tile"]:
                continue
            cfg = dict(best, sort_tile=tile)
            apply(cfg)
            ms = time_ms(run, dev, reps=max(reps, 5))
            if log is not None:
                log.append({"stage": "sort", "config": cfg, "ms": ms})
            if ms < base_sort * 0.99:
                best, base_sort = cfg, ms
        apply(best)
    base = time_ms(step, dev, reps=reps)
    if log is not None:
        log.append({"stage": "step", "config": dict(best), "ms": base})
    for k in knobs:
        start = best[k]  # already measured (base)
        for v in SPACE[k]:
            if v == start:
                continue
            cfg = dict(best, **{k: v})
            apply(cfg)
            ms = time_ms(step, dev, reps=reps)
            if log is not None:
                log.append({"stage": "step", "config": cfg, "ms": ms})
            if ms < base * 0.99:  # keep a change only for a clear gain
                best, base = cfg, ms
        apply(best)
    return best


def tuned(key: str, step: Callable[[], object], dev: torch.device, *,
          codes: Optional[torch.Tensor] = None, retune: bool = False, **kw) -> dict:
    """The cached configuration for ``key`` (applied), tuning it first when
    it is not cached (or ``retune``)."""
    cache = _load_cache()
    if not retune and key in cache:
        cfg = {k: int(v) for k, v in cache[key].items() if k in KNOBS}
        apply(cfg)
        return cfg
    cfg = tune(step, dev, codes=codes, **kw)
    _store_cache(key, cfg)
    return cfg


__all__ = ["KNOBS", "SPACE", "current", "apply", "signature", "time_ms", "tune", "tuned"]
