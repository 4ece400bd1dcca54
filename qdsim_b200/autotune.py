"""Autotuner for the batched eigensolve.

Picks, for one batch of dots, the LOBPCG block size, the DST preconditioner
shift and the FP32 -> FP64 hand-over of the mixed mode (FP32 target and
stagnation window) by timing solves of the batch itself on the GPU.  The
search is coordinate descent over a small candidate set (one parameter at a
time, the others fixed at the best values found so far); a configuration only
counts if every dot converges.  Results are cached in a JSON file keyed by the
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
DEFAULTS = {"block": 12, "shift_ev": 0.02, "stag_window": 12, "tol32": 1e-7}
SPACE = {
    "shift_ev": [0.01, 0.02, 0.04],
    "block": [12, 16],
    "stag_window": [8, 12, 20],
    "tol32": [3e-8, 1e-7, 3e-7],
}


def signature(host_batch, k: int, tol: float, gpu_name: str) -> str:
    h = hashlib.sha1()
    h.update(np.asarray(host_batch.rows_per_dot, np.int64).tobytes())
    h.update(np.asarray(host_batch.nnz_per_dot, np.int64).tobytes())
    h.update(f"{host_batch.order}|{k}|{tol:.3e}|{gpu_name}".encode())
    return h.hexdigest()[:16]


def _gpu_name(device) -> str:
    import torch
    return torch.cuda.get_device_name(device)


def load(host_batch, k: int, tol: float, device="cuda", cache=DEFAULT_CACHE):
    """Tuned configuration for this batch shape on this GPU, or None."""
    try:
        with open(cache) as f:
            entries = json.load(f)
    except (OSError, ValueError):
        return None
    e = entries.get(signature(host_batch, k, tol, _gpu_name(device)))
    return dict(e["config"]) if e else None


def _time_solve(db, k, tol, cfg, repeats):
    import torch
    db.set_shift(cfg["shift_ev"])
    kw = dict(b=cfg["block"], precision="mixed", tol=tol, max_iter=4000,
              tol32=cfg["tol32"], stag_window=cfg["stag_window"])
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


def tune(host_batch, k: int = 8, tol: float = 1e-9, device="cuda", space=None, repeats=2,
         cache=DEFAULT_CACHE, verbose=False):
    """Coordinate-descent search; returns (config, trace) and updates the cache."""
    from .batch import DeviceBatch
    space = space or SPACE
    db = DeviceBatch(host_batch, device)
    db.upload(non_blocking=False)
    db.assemble()
    best = dict(DEFAULTS)
    best_ms, ok = _time_solve(db, k, tol, best, repeats)
    trace = [{"config": dict(best), "ms": best_ms, "converged": ok}]
    if not ok:
        best_ms = float("inf")
    for name in ("shift_ev", "block", "stag_window", "tol32"):
        for value in space[name]:
            if value == best[name]:
                continue
            cand = dict(best)
            cand[name] = value
            ms, ok = _time_solve(db, k, tol, cand, repeats)
            trace.append({"config": dict(cand), "ms": ms, "converged": ok})
            if verbose:
                print(f"  {name}={value}: {ms:.1f} ms{'' if ok else ' (not converged)'}", flush=True)
            if ok and ms < best_ms:
                best, best_ms = cand, ms
    entry = {"config": best, "ms": best_ms, "gpu": _gpu_name(device), "k": k, "tol": tol,
             "n_dots": host_batch.n_dots, "rows": int(host_batch.n), "nnz": int(host_batch.nnz),
             "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()), "trace": trace}
    entries = {}
    try:
        with open(cache) as f:
            entries = json.load(f)
    except (OSError, ValueError):
        pass
    entries[signature(host_batch, k, tol, _gpu_name(device))] = entry
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
