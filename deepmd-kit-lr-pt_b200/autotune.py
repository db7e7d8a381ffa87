"""Autotuner of the tile-shape knobs (include/dpb200.h: dpb_tune_*).

The knobs pick launch shapes that the launchers read at launch time: atoms
(warps) per CTA of the fused descriptor kernels and of the batched env /
force kernels, the N tile of the tensor-core fitting GEMM, rows per group and
warps per CTA of the training kernels. ``tune`` times the options on the
caller's own step (CUDA events around replays of its captured graph, the
graph captured again after every change) by coordinate descent and leaves
the fastest shapes set; results are cached per GPU and workload signature in
a JSON file (``$DPB_TUNE_CACHE``, default ``~/.cache/deepmd_kit_lr_pt_b200/
tune.json``) so later runs of the same workload apply them without timing.
"""

from __future__ import annotations

import ctypes
import json
import os

import numpy as np
import torch

from . import _capi


def names() -> list[str]:
    lib = _capi.lib()
    return [lib.dpb_tune_name(i).decode() for i in range(lib.dpb_tune_count())]


def get(name: str) -> int:
    v = _capi.lib().dpb_tune_get(name.encode())
    if v < 0:
        raise _capi.DPBInvalidArgument(f"unknown tile knob {name!r}")
    return v


def options(name: str) -> list[int]:
    buf = (ctypes.c_int * 16)()
    n = _capi.lib().dpb_tune_options(name.encode(), buf, 16)
    if n < 0:
        raise _capi.DPBInvalidArgument(f"unknown tile knob {name!r}")
    return list(buf[:n])


def set_knob(name: str, value: int) -> None:
    _capi.call("dpb_tune_set", name.encode(), int(value))


def current(knobs=None) -> dict:
    return {k: get(k) for k in (knobs or names())}


def apply(values: dict) -> None:
    for k, v in values.items():
        set_knob(k, v)


def _cache_path() -> str:
    return os.environ.get("DPB_TUNE_CACHE", os.path.join(
        os.path.expanduser("~"), ".cache", "deepmd_kit_lr_pt_b200", "tune.json"))


def _key(signature: str, device) -> str:
    return f"{torch.cuda.get_device_name(device)}|{signature}"


def load_cached(signature: str, device=None) -> dict | None:
    try:
        with open(_cache_path()) as f:
            return json.load(f).get(_key(signature, device))
    except (OSError, ValueError):
        return None


def _store(signature: str, device, result: dict) -> None:
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        try:
            with open(path) as f:
                data = json.load(f)
        except (OSError, ValueError):
            data = {}
        data[_key(signature, device)] = result
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home: the result is still returned and applied


def time_step(run_step, reps: int = 10, warmup: int = 3, device=None) -> float:
    """Median milliseconds of run_step() over reps timed calls (CUDA events on
    the current stream)."""
    for _ in range(warmup):
        run_step()
    torch.cuda.synchronize(device)
    ev = []
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        run_step()
        b.record()
        ev.append((a, b))
    torch.cuda.synchronize(device)
    return float(np.median([a.elapsed_time(b) for a, b in ev]))


def tune(run_step, recapture, knobs, signature: str | None = None, reps: int = 10,
         warmup: int = 3, sweeps: int = 2, margin: float = 0.01, device=None,
         use_cache: bool = True) -> dict:
    """Coordinate descent over ``knobs``: for each knob try every option with
    the others fixed (recapture(), then the median of ``reps`` timed
    run_step() calls), keep an option only if it is faster by more than
    ``margin``; repeat up to ``sweeps`` times. Leaves the best shapes set and
    the step captured with them. Returns {"knobs", "ms", "baseline_ms",
    "history", "cached"}."""
    knobs = list(knobs)
    if use_cache and signature is not None:
        hit = load_cached(signature, device)
        if hit is not None and set(hit.get("knobs", {})) == set(knobs):
            apply(hit["knobs"])
            recapture()
            return dict(hit, cached=True)
    best = current(knobs)
    recapture()
    t_best = time_step(run_step, reps, warmup, device)
    baseline = t_best
    history = [{"knobs": dict(best), "ms": t_best}]
    for _ in range(sweeps):
        changed = False
        for k in knobs:
            for v in options(k):
                if v == best[k]:
                    continue
                set_knob(k, v)
                recapture()
                t = time_step(run_step, reps, warmup, device)
                history.append({"knobs": dict(best, **{k: v}), "ms": t})
                if t < t_best * (1.0 - margin):
                    best[k], t_best, changed = v, t, True
            set_knob(k, best[k])
        if not changed:
            break
    apply(best)
    recapture()
    result = {"knobs": best, "ms": t_best, "baseline_ms": baseline, "history": history}
    if signature is not None:
        _store(signature, device, result)
    return dict(result, cached=False)
