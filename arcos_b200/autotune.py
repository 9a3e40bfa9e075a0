"""Tile-shape autotuner for the stencil kernel.

Shapes 0-2 are the tiled fused kernel (tiles of 32 columns by WY*RPW rows,
one block per tile); shapes 3-5 the marching kernel (one warp per 31-column
strip and segment of 16, 32 or 64 rows).  Which is fastest depends on the
grid sizes (work units against SM count, halo share) and on the number of
species.  The tuner times a few device-timed steps with
each shape on the caller's own problem and keeps the fastest.  Timing runs
advance the simulation (the state moves on by the tuning steps).
"""
from __future__ import annotations

from typing import Dict, Optional

from ._lib import check

N_TILE_SHAPES = 6
TILE_SHAPES = {0: "tiles of 32 x 16 cells, 128 threads", 1: "tiles of 32 x 32 cells, 256 threads",
               2: "tiles of 32 x 16 cells, 256 threads",
               3: "marching warps, 31-column strips, segments of 16 rows",
               4: "marching warps, 31-column strips, segments of 32 rows",
               5: "marching warps, 31-column strips, segments of 64 rows"}


def autotune_tiles(tree, steps: int = 6, h: float = 50.0, stream=None) -> Dict[int, float]:
    """Times ``steps`` fused RK2 steps (even) per tile shape on ``tree`` (a
    CdrTree of single-grid families with a fixed field) and selects the
    fastest.  Returns {shape: ms per step}."""
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    steps += steps & 1
    L, h_ = tree.L, tree.h
    times = {}
    for cfg in range(N_TILE_SHAPES):
        tree.set_tile(cfg)
        check(L.arcos_run_prepare(h_, h))
        check(L.arcos_run_enqueue(h_, 2))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        check(L.arcos_run_enqueue(h_, steps))
        e1.record(s)
        e1.synchronize()
        times[cfg] = e0.elapsed_time(e1) / steps
    best = min(times, key=times.get)
    tree.set_tile(best)
    return times


TREE_SHAPES = (0, 1, 2, 3, 4, 5)   # the lean batched step: tiled k_fused (0-2) or k_march (3-5)


def autotune_tree(tree, steps: int = 4, h: float = 50.0, stream=None,
                  shapes=TREE_SHAPES) -> Dict[int, float]:
    """Times ``steps`` batched steps of a refinement tree (arcos_run, one
    CUDA graph per step) per shape and selects the fastest.  Shapes 0-2 run
    the lean step with the tiled fused kernel, 3-5 with k_march (segments of
    16, 32, 64 rows).  Returns {shape: ms per step}; the state advances."""
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    times = {}
    for cfg in shapes:
        tree.set_tile(cfg)
        tree.run(1, h)                      # capture the step graph
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        tree.run(steps, h)
        e1.record(s)
        e1.synchronize()
        times[cfg] = e0.elapsed_time(e1) / steps
    best = min(times, key=times.get)
    tree.set_tile(best)
    return times
