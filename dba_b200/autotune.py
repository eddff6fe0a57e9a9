"""Autotuner for the batched dendrite sweep.

The batch kernel's DBA block edge (8 or 16 cells) trades halo overhead and
per-block work against activity granularity; its threads per CTA (128, 256 or
512) trade blocks processed per pass against occupancy; its launch form
(persistent: one cooperative launch of up to 48 steps with a grid barrier
between steps; or one launch per step, both replayed from CUDA graphs) trades
the barrier's cost against launch gaps; and the number of steps advanced
between tip checks (`chunk`) trades host synchronisation against overshoot past
each run's stopping point.  `tune()` times every (block edge, threads, launch
form) on a short seeded mixed workload (the sweep's grid sizes and parameter
ranges, every slot admitted at once, a fixed number of steps) and returns the
fastest by active cell-updates per second, caching the choice per GPU and
precision in a JSON file (DBA_AUTOTUNE_CACHE, default
~/.cache/dba_b200/autotune.json).
"""
import json
import os
import time

from . import engine, serve

CANDIDATE_BLOCKS = (8, 16)
CANDIDATE_THREADS = (128, 256, 512)
CANDIDATE_PERSISTENT = (1, 0)
CANDIDATE_CHUNKS = (48, 96, 192)
SHORTEST_RUN_STEPS = 960


def _cache_path():
    return os.environ.get("DBA_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "dba_b200", "autotune.json"))


def _device_key(precision):
    """Cache key of the current CUDA device: its name, compute capability and SM
    count (so different GPUs on one host, or a non-zero current device, each get
    their own entry), and the precision."""
    import torch
    dev = torch.cuda.current_device()
    p = torch.cuda.get_device_properties(dev)
    return f"{p.name}|sm{p.major}{p.minor}|{p.multi_processor_count}sms|prec{precision}"


def time_candidate(block, threads=256, precision=1, persistent=1, nslots=24, steps=480, seed=5):
    """Active cell-updates per second of one (block edge, threads, launch form) on a mixed batch."""
    reqs = serve.sweep_requests(n=nslots, rate=0.0, seed=seed, edges=(128, 256, 512))
    b = engine.Batch(precision=precision, block=block, max_slots=nslots, block_capacity=1 << 17, threads=threads)
    try:
        b.set_option(engine.BATCH_PERSISTENT, persistent)
        for r in reqs:
            if b.add(serve.request_config(r, precision, block)) is None:
                break
        b.step(96)                      # warm-up: graph capture, clocks
        b.sync()
        a0 = b.info().active_block_steps
        t0 = time.perf_counter()
        b.step(steps)
        b.sync()
        dt = time.perf_counter() - t0
        cells = (b.info().active_block_steps - a0) * block * block
    finally:
        b.close()
    return cells / dt


def tune(precision=1, use_cache=True, verbose=False):
    key = _device_key(precision)
    path = _cache_path()
    cache = {}
    if use_cache and os.path.exists(path):
        try:
            cache = json.load(open(path))
        except Exception:
            cache = {}
        if key in cache:
            return cache[key]
    scores = {}
    for blk in CANDIDATE_BLOCKS:
        for nt in CANDIDATE_THREADS:
            for pers in CANDIDATE_PERSISTENT:
                scores[(blk, nt, pers)] = time_candidate(blk, nt, precision, persistent=pers)
                if verbose:
                    print(f"block {blk} threads {nt} persistent {pers}: {scores[(blk, nt, pers)]:.3e} cell-updates/s",
                          flush=True)
    best_block, best_threads, best_pers = max(scores, key=scores.get)
    # chunk: the largest (fewest host syncs) whose mean overshoot past the stop, chunk / 2,
    # stays within 5 % of the shortest runs of the sweep (a 128^2 grid stops after ~960 steps)
    best_chunk = max(c for c in CANDIDATE_CHUNKS if c / 2 <= 0.05 * SHORTEST_RUN_STEPS)
    choice = {"block": int(best_block), "threads": int(best_threads), "persistent": int(best_pers),
              "chunk": int(best_chunk), "scores": {f"{b}x{t}x{'p' if q else 's'}": v for (b, t, q), v in scores.items()}}
    if use_cache:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        cache[key] = choice
        with open(path, "w") as f:
            json.dump(cache, f, indent=1)
    return choice
