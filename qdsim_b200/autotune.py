"""Autotuner for the batched eigensolve.

Picks, for one batch of dots, the kernels' tile parameters and the solver's
parameters by timing solves of the batch itself on the GPU:
 - ``chunk_rows``: rows per CTA of every row-parallel kernel (SpMM, Gram,
   orthogonalisation, update), which also sets how many per-chunk partial
   sums the reductions add up;
 - ``block``: the LOBPCG block width B, the vector-row width every kernel is
   compiled for (B / 4 threads per row in the SpMMs, the Gram tile grid);
 - ``shift_ev``: the DST preconditioner's shift;
 - ``tol32`` / ``stag_window``: the FP32 -> FP64 hand-over of the mixed mode.
The search is coordinate descent over a small candidate set (one parameter at
a time, the others fixed at the best values found so far); a configuration
only counts if every dot converges.  Results are cached in a JSON file keyed by the
GPU name and a signature of the batch (dot sizes, nonzeros, k, tolerance), so
a later run of the same batch shape reads the tuned values instead of
re-tuning.

Usage: ``python -m qdsim_b200.autotune --dots 256 [--cache PATH]`` tunes the
batched sweep; ``load(...)`` / ``tune(...)`` serve other batches.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import time
from pathlib import Path

import numpy as np

DEFAULT_CACHE = Path(__file__).resolve().parent / "tuned.json"
DEFAULTS = {"block": 12, "shift_ev": 0.02, "stag_window": 12, "tol32": 1e-7,
            "chunk_rows": 1024}
SPACE = {
    "chunk_rows": [512, 1024, 2048, 4096],
    "shift_ev": [0.01, 0.02, 0.04],
    "block": [12, 16],
    "stag_window": [8, 12, 20],
    "tol32": [3e-8, 1e-7, 3e-7],
}
ORDER = ("chunk_rows", "shift_ev", "block", "stag_window", "tol32")


def solve_kwargs(cfg, tol, precision="mixed", max_iter=4000):
    """Keyword arguments of ``DeviceBatch.solve`` for a configuration."""
    return dict(b=int(cfg["block"]), precision=precision, tol=tol, max_iter=max_iter,
                tol32=cfg["tol32"], stag_window=cfg["stag_window"],
                chunk_rows=int(cfg.get("chunk_rows", DEFAULTS["chunk_rows"])))


def signature(host_batch, k: int, tol: float, gpu_name: str) -> str:
    h = hashlib.sha1()
    h.update(np.asarray(host_batch.rows_per_dot, np.int64).tobytes())
    h.update(np.asarray(host_batch.nnz_per_dot, np.int64).tobytes())
    h.update(f"{host_batch.order}|{k}|{tol:.3e}|{gpu_name}".encode())
    return h.hexdigest()[:16]


def _gpu_name(device) -> str:
    import torch
    return torch.cuda.get_device_name(device)


def load(host_batch, k: int, tol: float, device="cuda", cache=DEFAULT_CACHE, gpu_name=None):
    """Tuned configuration for this batch shape on this GPU, or None (entries
    from before a parameter existed get that parameter's default)."""
    try:
        with open(cache) as f:
            entries = json.load(f)
    except (OSError, ValueError):
        return None
    e = entries.get(signature(host_batch, k, tol, gpu_name or _gpu_name(device)))
    return dict(DEFAULTS, **e["config"]) if e else None


def _time_solve(db, k, tol, cfg, repeats):
    import torch
    db.set_shift(cfg["shift_ev"])
    kw = solve_kwargs(cfg, tol)
    db.solve(k, **kw)                     # warm (workspace, graphs)
    torch.cuda.synchronize()
    best = None
    for _ in range(repeats):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        out = db.solve(k, **kw)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    converged = int(out[4]["converged_dots"]) == db.host.n_dots
    return best, converged


def search(timer, space=None, start=None, verbose=False):
    """Coordinate descent: ``timer(cfg) -> (ms, converged)``; returns (best
    config, best ms, trace).  Parameters are visited in ORDER; a candidate
    replaces the best only if it converged and is faster."""
    space = space or SPACE
    best = dict(start or DEFAULTS)
    best_ms, ok = timer(best)
    trace = [{"config": dict(best), "ms": best_ms, "converged": ok}]
    seen = {tuple(sorted(best.items()))}
    if not ok:
        best_ms = float("inf")
    for name in ORDER:
        for value in space.get(name, []):
            cand = dict(best)
            cand[name] = value
            key = tuple(sorted(cand.items()))
            if key in seen:           # timed already (e.g. the value best started from)
                continue
            seen.add(key)
            ms, ok = timer(cand)
            trace.append({"config": dict(cand), "ms": ms, "converged": ok})
            if verbose:
                print(f"  {name}={value}: {ms:.1f} ms{'' if ok else ' (not converged)'}", flush=True)
            if ok and ms < best_ms:
                best, best_ms = cand, ms
    return best, best_ms, trace


def tune(host_batch, k: int = 8, tol: float = 1e-9, device="cuda", space=None, repeats=2,
         cache=DEFAULT_CACHE, verbose=False, timer=None, gpu_name=None):
    """Coordinate-descent search; returns (config, trace) and updates the
    cache.  ``timer`` replaces the GPU timing (tests)."""
    if timer is None:
        from .batch import DeviceBatch
        db = DeviceBatch(host_batch, device)
        db.upload(non_blocking=False)
        db.assemble()

        def timer(cfg):
            return _time_solve(db, k, tol, cfg, repeats)
    gpu = gpu_name or _gpu_name(device)
    best, best_ms, trace = search(timer, space, verbose=verbose)
    entry = {"config": best, "ms": best_ms, "gpu": gpu, "k": k, "tol": tol,
             "n_dots": host_batch.n_dots, "rows": int(host_batch.n), "nnz": int(host_batch.nnz),
             "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()), "trace": trace}
    entries = {}
    try:
        with open(cache) as f:
            entries = json.load(f)
    except (OSError, ValueError):
        pass
    entries[signature(host_batch, k, tol, gpu)] = entry
    os.makedirs(os.path.dirname(os.path.abspath(cache)), exist_ok=True)
    with open(cache, "w") as f:
        json.dump(entries, f, indent=1)
    return best, trace


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--dots", type=int, default=256)
    ap.add_argument("--k", type=int, default=8)
    ap.add_argument("--tol", type=float, default=1e-9)
    ap.add_argument("--repeats", type=int, default=2)
    ap.add_argument("--cache", default=str(DEFAULT_CACHE))
    args = ap.parse_args()
    from . import workloads as W
    from .batch import HostBatch
    hb = HostBatch(W.sweep_batch(args.dots))
    best, trace = tune(hb, args.k, args.tol, repeats=args.repeats, cache=args.cache,
                       verbose=True)
    print(json.dumps({"best": best, "ms": min(t["ms"] for t in trace if t["converged"])}))


if __name__ == "__main__":
    main()
