"""Launch-shape autotuner for the tracking kernel.

The tracking kernel is a persistent grid whose warps claim `chunk` histories per atomic
ticket and refill finished lanes at every event boundary.  Its speed depends on:
  block_size     threads per block (64..256; the kernel is compiled for <= 256)
  blocks_per_sm  resident blocks requested per SM (grid = blocks_per_sm x SMs)
  chunk          histories claimed per warp ticket (refill cadence / bank tile)
  smem_cells     stage the per-cell (sigma_a, sigma_s) table in shared memory
  prefetch       lanes copy their next history's bank record to shared memory ahead of need
                 (not in the default grid: slower on every workload measured)
The tuner replays the engine's last transport on a snapshot of the census bank for every
candidate (the Philox streams make each trial the identical work), times the tracking
phase with CUDA events, restores the census and installs the fastest shape.
"""
from __future__ import annotations

import itertools

import torch

from .engine import Bank, Engine

DEFAULT_GRID = {
    "block_size": (128, 256),
    "blocks_per_sm": (2, 4, 8),  # 2: small banks, where fewer resident lanes keep warps fuller
    "chunk": (512, 1024, 2048, 4096, 8192),
    "smem_cells": (0, 1),
}


def _snapshot(bank: Bank) -> dict:
    n = bank.size
    snap = {k: getattr(bank, k)[:n].clone() for k in Bank.FIELDS_F + ("cell",)}
    if bank.multigroup:
        snap["group"] = bank.group[:n].clone()
    snap["_n"] = n
    return snap


def _restore(bank: Bank, snap: dict) -> None:
    n = snap["_n"]
    bank.size = n
    for k, v in snap.items():
        if k != "_n":
            getattr(bank, k)[:n].copy_(v)


def candidates(engine: Engine, grid: dict | None = None) -> list[dict]:
    g = dict(DEFAULT_GRID if grid is None else grid)
    # the shared-memory table costs 8 B/cell/group: only for tables that leave room for >= 2 blocks
    if engine.nc * engine.ng * 8 > 108 * 1024:
        g["smem_cells"] = (0,)
    keys = list(g)
    return [dict(zip(keys, vals)) for vals in itertools.product(*(g[k] for k in keys))]


def tune_tracking(engine: Engine, transport_args: tuple, transport_kwargs: dict, grid: dict | None = None,
                  repeats: int = 2) -> dict:
    """Time every candidate launch shape on the current census; install and return the best.

    transport_args / transport_kwargs: the arguments of Engine.transport_async for one step
    (the material fields, source parameters and step index of a representative step).
    """
    snap = _snapshot(engine.bank)
    saved = dict(engine.launch)
    results = []
    for cand in candidates(engine, grid):
        engine.launch.update(cand)
        best = float("inf")
        for _ in range(repeats):
            _restore(engine.bank, snap)
            engine._census_dev_valid = False
            engine.transport_async(*transport_args, **transport_kwargs)
            torch.cuda.current_stream(engine.device).synchronize()
            best = min(best, engine.phase_times()[1])
        results.append((best, cand))
    _restore(engine.bank, snap)
    engine._census_dev_valid = False
    results.sort(key=lambda r: r[0])
    engine.launch = dict(saved)
    engine.launch.update(results[0][1])
    return {"best": results[0][1], "best_ms": results[0][0], "worst_ms": results[-1][0],
            "trials": [(round(t, 4), c) for t, c in results]}
