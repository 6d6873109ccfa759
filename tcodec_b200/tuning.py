"""Autotuner of the CTU engine's knobs for one frame size.

The engine has two knobs that change how long a batched step takes and never
what it produces (include/tcodec_b200.h, tcb_engine_set_tuning):

* search_window: radius R of the motion search's SAD tables (2..5);
* queue_order: how a batch step merges its streams' CTU wavefronts
  (diagonal-major or staggered).

Their best values depend on the frame size and on the content (how far the
searches walk, how many streams share a step), so `tune_engine` measures
them: it runs a batch of `streams` streams of the caller's frames (device
resident, so only the engine and the host steps are timed) for every
combination, times `steps` steps after `warmup` untimed ones with CUDA
events on the batch's stream, keeps the fastest (ties go to the default),
and records it in the library's table with tcb_engine_set_tuning.  Every
later encoder, batch and server of that frame size in the process uses it.

Reported back: the chosen pair and the milliseconds per step of every
combination.
"""
from __future__ import annotations

import ctypes
import itertools
from typing import Dict, List, Sequence, Tuple

from . import api

WINDOWS = (3, 4, 5)
ORDERS = (api.QUEUE_DIAGONAL, api.QUEUE_STAGGERED)


def _ms_per_step(lib, cfg, dev_frames, streams: int, steps: int, warmup: int) -> float:
    """Device time per batched step of `streams` streams, stream s encoding
    frames s, s + 1, ... of dev_frames ((y, cb, cr) CUDA tensors)."""
    import torch
    batch = api.BatchEncoder(lib, [cfg] * streams)
    try:
        stream = torch.cuda.ExternalStream(lib.tcb_batch_stream(batch.h))

        def step(t):
            planes = [tuple((f.data_ptr(), f.shape[1]) for f in dev_frames[(s + t) % len(dev_frames)])
                      for s in range(streams)]
            batch.encode(planes, on_device=True)

        for t in range(warmup):
            step(t)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for t in range(warmup, warmup + steps):
            step(t)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps
    finally:
        batch.close()


def tune_engine(lib: ctypes.CDLL, cfg: api.Config, frames: Sequence, streams: int = 32, steps: int = 3,
                warmup: int = 5, windows: Sequence[int] = WINDOWS,
                orders: Sequence[int] = ORDERS) -> Dict:
    """Time every (search_window, queue_order) on `streams` streams of
    `frames` ((y, cb, cr) numpy planes of cfg's size) and record the fastest
    for cfg.width x cfg.height.  Returns {"chosen": (window, order),
    "ms_per_step": {(window, order): ms}, "streams": streams}."""
    import numpy as np
    import torch
    lib = api.bind_b200(lib)
    W, H = cfg.width, cfg.height
    dev = [tuple(torch.from_numpy(np.ascontiguousarray(p)).cuda() for p in f) for f in frames]
    before = api.engine_tuning(lib, W, H)
    times: Dict[Tuple[int, int], float] = {}
    try:
        for w, o in itertools.product(windows, orders):
            api.set_engine_tuning(lib, W, H, w, o)
            times[(w, o)] = _ms_per_step(lib, cfg, dev, streams, steps, warmup)
    except Exception:
        api.set_engine_tuning(lib, W, H, *before)
        raise
    default = (4, api.QUEUE_DIAGONAL)
    best = min(times, key=lambda k: (times[k], k != default))
    api.set_engine_tuning(lib, W, H, *best)
    return {"chosen": best, "ms_per_step": times, "streams": streams}


def describe(result: Dict) -> Dict:
    """JSON-friendly form of a tune_engine result."""
    names = {api.QUEUE_DIAGONAL: "diagonal", api.QUEUE_STAGGERED: "staggered"}
    w, o = result["chosen"]
    return {"search_window": w, "queue_order": names[o], "streams": result["streams"],
            "ms_per_step": {f"R{k[0]}/{names[k[1]]}": round(v, 2) for k, v in sorted(result["ms_per_step"].items())}}


def choice_table(lib: ctypes.CDLL, sizes: List[Tuple[int, int]]) -> Dict[Tuple[int, int], Tuple[int, int]]:
    """The (search_window, queue_order) the library uses for each size."""
    return {s: api.engine_tuning(lib, *s) for s in sizes}
