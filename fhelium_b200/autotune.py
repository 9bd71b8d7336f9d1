"""Measured choice of the launch knobs of a batched workload.

The knobs a run can change without recompiling:

* ``ks_order`` (FHB_TUNE_KS_ORDER): the work order of the key-switch
  clusters, 0 = the limbs of one ciphertext back to back (the digits of one
  ciphertext stay in L2 while its limbs are processed), 1 = one limb across
  the batch back to back (the key rows of one prime are shared by the whole
  batch, which pays when every item uses the same key), 2 = one limb across
  a group of four ciphertexts, group by group (both the key rows of the limb
  and the group's digits stay in L2);
* ``streams``: how many graph branches the mixed-batch executor spreads its
  (kind, level) groups over, i.e. how many groups run side by side;
* for the descriptor-driven mixed batch (``MixedItemsExecutor``): the
  key-switch work order inside each (level, key) group of items (0 = the
  rows of one item back to back, 2 = one row across the group) and the
  scratch limit of a chunk of items (fewer, larger chunks launch fewer
  times but hold more scratch);
* ``ntt_forward_ept`` / ``ntt_inverse_ept`` (FHB_TUNE_NTT_{FORWARD,INVERSE}_EPT):
  residues per thread of the standalone transforms, i.e. the NTT's register
  radix and tile: 8 residues (radix-8 passes, 1024 threads per CTA at
  N = 2^16) or 16 (radix-16 passes, 512 threads).

The cluster width (CTAs per polynomial) is fixed per ring degree when the
library is compiled; every runtime knob above is picked here by timing the
caller's own workload (CUDA-graph replays for batches).  Winners are cached in a JSON file keyed by device,
ring, modulus chain and workload shape, so a later process with the same
workload skips the search.  The reference has no autotuner (its launch
shapes are fixed in csrc/ops/ntt/cuda/*.cu).
"""

from __future__ import annotations

import hashlib
import json
import os
import threading
from typing import Iterable

import torch

_LOCK = threading.Lock()


def default_cache_path() -> str:
    env = os.environ.get("FHB200_AUTOTUNE_CACHE")
    if env:
        return env
    return os.path.join(os.path.expanduser("~"), ".cache", "fhelium_b200", "autotune.json")


def _load(path: str) -> dict:
    try:
        with open(path) as f:
            data = json.load(f)
        return data if isinstance(data, dict) else {}
    except (OSError, ValueError):
        return {}


def _store(path: str, key: str, entry: dict) -> None:
    with _LOCK:
        data = _load(path)
        data[key] = entry
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        tmp = f"{path}.{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)


def workload_key(engine, executor) -> str:
    """Device + ring + chain + the multiset of (kind, level, items) groups."""
    shape = sorted((g.kind, g.level, g.items) for g in executor.groups)
    digest = hashlib.sha256(json.dumps(shape).encode()).hexdigest()[:16]
    chain = hashlib.sha256(json.dumps([int(m) for m in engine.moduli]).encode()).hexdigest()[:12]
    dev = torch.cuda.get_device_name(engine.device)
    return f"{dev}|logN={engine.log_n}|q={engine.num_q}|p={engine.num_p}|chain={chain}|mixed={digest}"


def time_replays(run, device, *, warmup: int = 1, repeats: int = 3) -> float:
    """Median milliseconds of `run()` on the current stream (CUDA events)."""
    for _ in range(warmup):
        run()
    stream = torch.cuda.current_stream(device)
    times = []
    for _ in range(repeats):
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        start.record(stream)
        run()
        stop.record(stream)
        stop.synchronize()
        times.append(start.elapsed_time(stop))
    times.sort()
    return times[len(times) // 2]


def tune_ntt(ctx, x: torch.Tensor, rows: int, row_start: int = 0, *, candidates: Iterable[int] = (8, 16),
             repeats: int = 5, cache_path: str | None = None, use_cache: bool = True) -> dict:
    """Pick residues per thread of the forward and of the inverse NTT for
    polynomials shaped like `x` ([..., rows, N] residues of prime ids
    [row_start, row_start + rows) on ctx's device) and leave `ctx` set to the
    winners.  Returns ``{"forward_ept", "inverse_ept", "forward_ms", ...}``."""
    from . import _native as nat
    cache_path = cache_path or default_cache_path()
    n = x.size(-1)
    batch = x.numel() // (rows * n)
    dev = x.device
    bits = 32 if x.element_size() == 4 else 64
    key = f"{torch.cuda.get_device_name(dev)}|ntt|bits={bits}|N={n}|rows={rows}|row_start={row_start}|batch={batch}"
    if use_cache:
        hit = _load(cache_path).get(key)
        if hit and {"forward_ept", "inverse_ept"} <= set(hit):
            ctx.set_tuning(nat.TUNE_NTT_FORWARD_EPT, int(hit["forward_ept"]))
            ctx.set_tuning(nat.TUNE_NTT_INVERSE_EPT, int(hit["inverse_ept"]))
            return dict(hit, cached=True)
    y = torch.empty_like(x)
    z = torch.empty_like(x)
    st = torch.cuda.current_stream(dev).cuda_stream
    fwd = lambda: ctx.call("fhb_forward_ntt", x.data_ptr(), y.data_ptr(), batch, rows, row_start, 0, st)
    inv = lambda: ctx.call("fhb_inverse_ntt", y.data_ptr(), z.data_ptr(), batch, rows, row_start, 2, st)
    entry: dict = {"candidates": {}}
    for name, param, fn in (("forward", nat.TUNE_NTT_FORWARD_EPT, fwd), ("inverse", nat.TUNE_NTT_INVERSE_EPT, inv)):
        times = {}
        for ept in candidates:
            ctx.set_tuning(param, int(ept))
            times[int(ept)] = time_replays(fn, dev, warmup=2, repeats=repeats)
        best = min(times, key=times.get)
        ctx.set_tuning(param, best)
        entry[f"{name}_ept"] = best
        entry[f"{name}_ms"] = times[best]
        entry["candidates"][name] = {str(k): v for k, v in times.items()}
    _store(cache_path, key, entry)
    return dict(entry, cached=False)


def tune_mixed_batch(engine, executor, *, ks_orders: Iterable[int] = (0, 1, 2), streams: Iterable[int] = (1, 2, 3, 4),
                     repeats: int = 3, cache_path: str | None = None, use_cache: bool = True) -> dict:
    """Pick (ks_order, streams) for `executor` by timing graph replays.

    Leaves the executor configured with the winner and returns
    ``{"ks_order", "streams", "ms", "candidates": [...], "cached": bool}``.
    """
    cache_path = cache_path or default_cache_path()
    key = workload_key(engine, executor)
    if use_cache:
        hit = _load(cache_path).get(key)
        if hit and {"ks_order", "streams"} <= set(hit):
            executor.configure(streams=int(hit["streams"]), ks_order=int(hit["ks_order"]))
            return dict(hit, cached=True)
    results = []
    for order in ks_orders:
        for s in streams:
            executor.configure(streams=s, ks_order=order)
            ms = time_replays(executor.run, engine.device, repeats=repeats)
            results.append({"ks_order": int(order), "streams": int(s), "ms": ms})
    best = min(results, key=lambda r: r["ms"])
    executor.configure(streams=best["streams"], ks_order=best["ks_order"])
    entry = dict(best, candidates=results)
    _store(cache_path, key, entry)
    return dict(entry, cached=False)


def items_workload_key(engine, ciphertexts, ops) -> str:
    """Device + ring + chain + the multiset of (kind, level) items."""
    shape = sorted((op.kind, ciphertexts[op.index].level) for op in ops)
    digest = hashlib.sha256(json.dumps(shape).encode()).hexdigest()[:16]
    chain = hashlib.sha256(json.dumps([int(m) for m in engine.moduli]).encode()).hexdigest()[:12]
    dev = torch.cuda.get_device_name(engine.device)
    return f"{dev}|logN={engine.log_n}|q={engine.num_q}|p={engine.num_p}|chain={chain}|items={digest}"


def tune_items(engine, ciphertexts, ops, *, ks_orders: Iterable[int] = (0, 2),
               limits: Iterable[int] = (4 << 30, 8 << 30, 16 << 30), repeats: int = 3,
               cache_path: str | None = None, use_cache: bool = True):
    """Pick (ks_order, max_scratch_bytes) of a MixedItemsExecutor for this
    batch by timing graph replays of each candidate (built one at a time).
    Returns ``(executor, entry)``: the executor built with the winner and
    ``{"ks_order", "max_scratch_bytes", "ms", "candidates", "cached"}``."""
    from .batch import MixedItemsExecutor
    cache_path = cache_path or default_cache_path()
    key = items_workload_key(engine, ciphertexts, ops)
    if use_cache:
        hit = _load(cache_path).get(key)
        if hit and {"ks_order", "max_scratch_bytes"} <= set(hit):
            ex = MixedItemsExecutor(engine, ciphertexts, ops, ks_order=int(hit["ks_order"]),
                                    max_scratch_bytes=int(hit["max_scratch_bytes"]))
            return ex, dict(hit, cached=True)
    results = []
    for order in ks_orders:
        for limit in limits:
            ex = MixedItemsExecutor(engine, ciphertexts, ops, ks_order=int(order), max_scratch_bytes=int(limit))
            ms = time_replays(ex.run, engine.device, repeats=repeats)
            results.append({"ks_order": int(order), "max_scratch_bytes": int(limit), "chunks": len(ex.chunks),
                            "ms": ms})
            del ex
            torch.cuda.empty_cache()
    best = min(results, key=lambda r: r["ms"])
    entry = dict(best, candidates=results)
    _store(cache_path, key, entry)
    ex = MixedItemsExecutor(engine, ciphertexts, ops, ks_order=best["ks_order"],
                            max_scratch_bytes=best["max_scratch_bytes"])
    return ex, dict(entry, cached=False)
