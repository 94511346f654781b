"""Autotuner for the round execution mode and tile shape.

For one resolution N and dtype it times short rounds of every candidate
(mode in {resident, persistent, graph}) x (tile shape) on the current GPU and
keeps the fastest; resident candidates whose tiles do not all fit on the GPU
at once (or whose tile shape has no resident kernel) are skipped.  Results are cached per (GPU name, N, dtype) in a JSON file
(``$LICOM_BT_TUNE_CACHE``, default ``~/.cache/licom4py_gpu_b200/tune.json``).
Without constants to time with, a static heuristic is returned.
"""

from __future__ import annotations

import json
import os
from typing import Dict, Optional, Sequence

import torch

TILES = ((7, 32), (8, 32), (15, 32), (16, 32), (8, 16), (16, 16))
MODES = ("resident", "persistent", "graph")


def _cache_path() -> str:
    return os.environ.get("LICOM_BT_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "licom4py_gpu_b200", "tune.json"))


def _load_cache() -> Dict[str, dict]:
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(key: str, cfg: dict) -> None:
    cache = _load_cache()
    cache[key] = cfg
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1)
        os.replace(tmp, path)
    except OSError:
        pass


def heuristic(n: int) -> dict:
    """Static choice from B200 measurements: CUDA graphs everywhere (at C48-C96
    the graph with programmatic launch beat the tile-resident and persistent
    rounds), small tiles for small grids."""
    if n <= 96:
        return {"mode": "graph", "tile": [8, 16], "source": "heuristic"}
    if n <= 192:
        return {"mode": "graph", "tile": [8, 32], "source": "heuristic"}
    return {"mode": "graph", "tile": [16, 32], "source": "heuristic"}


def _key(n: int, dtype: torch.dtype, device) -> str:
    name = torch.cuda.get_device_name(device)
    return f"{name}|C{n}|{str(dtype).replace('torch.', '')}"


def tune(n: int, dtype: torch.dtype, consts: Sequence, device=None, nbb: int = 40, reps: int = 3,
         modes: Sequence[str] = MODES, tiles: Sequence = TILES) -> dict:
    """Time every (mode, tile) candidate on ``nbb``-substep rounds; return and cache the best."""
    from .fields import harmonic_state  # noqa: F401  (keeps the import graph explicit)
    from .plan import BtPlan
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    m = n + 6
    g = torch.Generator(device="cpu").manual_seed(0)
    h = (torch.randn((6, m, m), generator=g, dtype=torch.float64) * 0.5).to(dev, dtype)
    u = (torch.randn((6, m, m), generator=g, dtype=torch.float64) * 0.1).to(dev, dtype)
    v = (torch.randn((6, m, m), generator=g, dtype=torch.float64) * 0.1).to(dev, dtype)
    ins = [h, h, u, v, u, v]
    dtb = 0.05 * 1.231 * 6.3712e6 / n / (9.8 * 5000.0) ** 0.5  # small, stable step for timing
    results = []
    for mode in modes:
        for tile in tiles:
            p = BtPlan(consts, dtype=dtype, device=dev, tile=tile, mode=mode)
            out = None
            try:
                try:
                    out = p.round(*ins, nbb=nbb, dtb=dtb, diag=False)
                except NotImplementedError:  # resident mode: shape without a kernel, or too many tiles
                    continue
                torch.cuda.synchronize(dev)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                for _ in range(reps):
                    p.round(*ins, nbb=nbb, dtb=dtb, diag=False, out=out)
                b.record()
                torch.cuda.synchronize(dev)
                ms = a.elapsed_time(b) / reps
                results.append({"mode": mode, "tile": list(tile), "ms_per_round": ms,
                                "cell_updates_per_s": 6 * n * n * nbb / (ms * 1e-3)})
            finally:
                p.close()
    best = min(results, key=lambda r: r["ms_per_round"])
    cfg = {"mode": best["mode"], "tile": best["tile"], "source": "tuned", "nbb": nbb, "candidates": results}
    _store(_key(n, dtype, dev), cfg)
    return cfg


def choose_config(n: int, dtype: torch.dtype = torch.float64, consts: Optional[Sequence] = None,
                  device=None, retune: bool = False) -> dict:
    """Cached tuned config, else tune when constants are given, else the heuristic."""
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    if not retune:
        cfg = _load_cache().get(_key(n, dtype, dev))
        if cfg is not None:
            return cfg
    if consts is None:
        return heuristic(n)
    return tune(n, dtype, consts, dev)


# ---- batched rounds ----------------------------------------------------------
BATCH_MODES = ("persistent", "stream")
BATCH_CTAS = (0, 148, 296)  # persistent grid caps tried (0 = as many CTAs as fit)


def _mix_key(specs, dtype: torch.dtype, rk: int, device) -> str:
    counts: Dict[int, int] = {}
    for s in specs:
        counts[s.n] = counts.get(s.n, 0) + 1
    mix = ",".join(f"C{n}x{c}" for n, c in sorted(counts.items()))
    return f"{torch.cuda.get_device_name(device)}|batch|{str(dtype).replace('torch.', '')}|rk{rk}|{mix}"


def tune_batch(ens, nsub: int = 48, reps: int = 2, modes: Sequence[str] = BATCH_MODES,
               tiles: Sequence = TILES, ctas: Sequence[int] = BATCH_CTAS) -> dict:
    """Time batched rounds of the ensemble ``ens`` for every (mode, tile, grid
    cap) candidate and cache the fastest.  The trial keeps the mix and its
    retirement pattern at a shorter length: member k runs
    max(1, nsub * nsub_k / max nsub) substeps."""
    from .batch import BtBatch
    longest = max(s.nsub for s in ens.specs)
    trial = [max(1, round(nsub * s.nsub / longest)) for s in ens.specs]
    work = sum(6 * s.n * s.n * k for s, k in zip(ens.specs, trial))
    results = []
    for mode in modes:
        for tile in tiles:
            for cap in (ctas if mode == "persistent" else (0,)):
                b = BtBatch(ens.dtype, max_members=len(ens.specs), device=ens.device, mode=mode, tile=tile)
                try:
                    b.set_max_ctas(cap)
                    times = []
                    for r in range(reps + 1):
                        mem = ens.members()
                        for m, k in zip(mem, trial):
                            m.remaining = k
                        torch.cuda.synchronize(ens.device)
                        a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        a.record()
                        b.advance(mem)
                        z.record()
                        torch.cuda.synchronize(ens.device)
                        if r > 0:
                            times.append(a.elapsed_time(z))
                    b.check_device_error()
                    ms = min(times)
                    results.append({"mode": mode, "tile": list(tile), "max_ctas": cap, "ms": ms,
                                    "cell_updates_per_s": work / (ms * 1e-3)})
                finally:
                    b.close()
    best = min(results, key=lambda r: r["ms"])
    cfg = {"mode": best["mode"], "tile": best["tile"], "max_ctas": best["max_ctas"], "source": "tuned",
           "trial_substeps": nsub, "candidates": results}
    _store(_mix_key(ens.specs, ens.dtype, ens.rk, ens.device), cfg)
    return cfg


def choose_batch_config(ens, retune: bool = False) -> dict:
    """Cached tuned batch config for this mix, else tune it now."""
    if not retune:
        cfg = _load_cache().get(_mix_key(ens.specs, ens.dtype, ens.rk, ens.device))
        if cfg is not None:
            return cfg
    return tune_batch(ens)
