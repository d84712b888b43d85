"""Autotuner for the launch shapes of the quartet kernels.

Each class kernel of the J/K build (and of the gradient) runs a grid-stride
loop over its selected quartets; its launch shape is the block size (64 or
128 threads: 2 or 4 warps of 32 quartets each per step) and the grid cap in
resident blocks per SM (how many quartets a block takes in total, and how
evenly the tail of a class spreads over the 148 SMs).  The best shape
depends on the class (register footprint, primitive count per quartet) and
on the workload (how many quartets survive screening), so it is measured:
every candidate shape is applied to all classes at once, one build is timed
per class with CUDA events (``dftk_jk_timing``), and each class keeps its
fastest shape.  Results are cached in memory per (device, workload
signature) and can be saved to / loaded from a JSON file.

The J/K family has a third dimension, the tile: how many consecutive
32-quartet work items a warp takes per step of its loop (1, 2, 4, 8), i.e.
how long a warp stays on neighbouring list entries (shared bra pairs); with
the shapes chosen, every tile is timed the same way and each class keeps its
fastest.
"""
from __future__ import annotations

import ctypes
import json
import os
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib

FAMILY_JK, FAMILY_GRAD = 0, 1
N_QCLASS = 6
CANDIDATES: Tuple[Tuple[int, int], ...] = ((128, 4), (128, 8), (128, 16), (128, 32), (64, 8), (64, 16), (64, 32))
TILES: Tuple[int, ...] = (1, 2, 4, 8)

_cache: Dict[str, Dict] = {}


def get_shapes(family: int, fp32: bool = False) -> List[Tuple[int, int]]:
    out = []
    for c in range(N_QCLASS):
        t, b = ctypes.c_int(), ctypes.c_int()
        _lib.call("dftk_get_launch", family, c, int(fp32), ctypes.byref(t), ctypes.byref(b))
        out.append((t.value, b.value))
    return out


def set_shapes(family: int, shapes: Sequence[Tuple[int, int]], fp32: bool = False) -> None:
    for c, (t, b) in enumerate(shapes):
        _lib.call("dftk_set_launch", family, c, int(fp32), int(t), int(b))


def get_tiles(fp32: bool = False) -> List[int]:
    out = []
    for c in range(N_QCLASS):
        t = ctypes.c_int()
        _lib.call("dftk_get_tile", c, int(fp32), ctypes.byref(t))
        out.append(t.value)
    return out


def set_tiles(tiles: Sequence[int], fp32: bool = False) -> None:
    for c, t in enumerate(tiles):
        _lib.call("dftk_set_tile", c, int(fp32), int(t))


def _signature(engine, family: int, fp32: bool) -> str:
    name = torch.cuda.get_device_name(engine.device)
    totals = [int(np.log2(max(t, 1))) for t in engine.quartet_totals()]  # size bucket per class
    return json.dumps([name, family, int(fp32), totals])


def _time_classes(run, repeats: int, fp32: bool = False) -> np.ndarray:
    """Per-class kernel ms of `run()` (median of `repeats`), via the timing hook
    (slots 0..5 hold the FP64 class launches, 6..11 the FP32 ones)."""
    ms = []
    _lib.call("dftk_jk_timing", 1)
    try:
        for _ in range(repeats):
            run()
            buf = (ctypes.c_float * 12)()
            _lib.call("dftk_jk_timing_read", buf, 12)
            o = N_QCLASS if fp32 else 0
            ms.append(np.array(buf[o:o + N_QCLASS]))
    finally:
        _lib.call("dftk_jk_timing", 0)
    return np.median(np.stack(ms), axis=0)


def tune(engine, run, family: int = FAMILY_JK, fp32: bool = False,
         candidates: Sequence[Tuple[int, int]] = CANDIDATES, repeats: int = 3, apply: bool = True) -> Dict:
    """Measure every candidate shape for every class of ``family`` while
    ``run()`` issues one build (or gradient) on ``engine``; keep per class the
    fastest.  Returns {"shapes": [...], "ms": {...}, "default_ms": [...]}."""
    key = _signature(engine, family, fp32)
    if key in _cache:
        res = _cache[key]
        if apply:
            set_shapes(family, res["shapes"], fp32)
            if "tiles" in res:
                set_tiles(res["tiles"], fp32)
        return res
    default = get_shapes(family, fp32)
    run()  # warm-up
    torch.cuda.synchronize(engine.device)
    table = {}
    try:
        for cand in candidates:
            set_shapes(family, [cand] * N_QCLASS, fp32)
            table[cand] = _time_classes(run, repeats, fp32)
        set_shapes(family, default, fp32)
        base = _time_classes(run, repeats, fp32)
    finally:
        set_shapes(family, default, fp32)
    best = []
    for c in range(N_QCLASS):
        cand = min(candidates, key=lambda k: table[k][c])
        best.append(cand if table[cand][c] < base[c] else tuple(default[c]))
    tuned = [float(table[best[c]][c]) if best[c] in table else float(base[c]) for c in range(N_QCLASS)]
    res = {"shapes": [list(b) for b in best],
           "ms": {f"{t}x{b}": [float(x) for x in v] for (t, b), v in table.items()},
           "default_ms": [float(x) for x in base],
           "tuned_ms": tuned}
    if family == FAMILY_JK:
        # the tile, with the chosen shapes in place
        set_shapes(family, res["shapes"], fp32)
        default_tiles = get_tiles(fp32)
        ttab = {}
        try:
            for t in TILES:
                set_tiles([t] * N_QCLASS, fp32)
                ttab[t] = _time_classes(run, repeats, fp32)
        finally:
            set_tiles(default_tiles, fp32)
            set_shapes(family, default, fp32)
        tiles = [min(TILES, key=lambda t: ttab[t][c]) for c in range(N_QCLASS)]
        res["tiles"] = tiles
        res["tile_ms"] = {str(t): [float(x) for x in v] for t, v in ttab.items()}
        res["tuned_ms"] = [min(tuned[c], float(ttab[tiles[c]][c])) for c in range(N_QCLASS)]
    _cache[key] = res
    if apply:
        set_shapes(family, res["shapes"], fp32)
        if "tiles" in res:
            set_tiles(res["tiles"], fp32)
    return res


def tune_jk(engine, D: torch.Tensor, D_a: Optional[torch.Tensor] = None, tau: float = 1e-14, **kw) -> Dict:
    """Tune the FP64 J/K class kernels on one build of ``engine`` at density D."""
    return tune(engine, lambda: engine.jk(D, D_a, tau=tau), FAMILY_JK, False, **kw)


def tune_jk_mixed(engine, dD: torch.Tensor, tau: float = 1e-12, tau_fp32: float = 1e-6, **kw) -> Dict:
    """Tune the FP32 class kernels of the mixed build on one incremental build
    of density difference dD (the FP64 part keeps its shapes)."""
    return tune(engine, lambda: engine.jk(2.0 * dD, dD, mixed=True, tau=tau, tau_fp32=tau_fp32), FAMILY_JK, True,
                **kw)


def save(path: str) -> None:
    with open(path, "w") as fh:
        json.dump(_cache, fh)


def load(path: str) -> None:
    if os.path.exists(path):
        with open(path) as fh:
            _cache.update(json.load(fh))
