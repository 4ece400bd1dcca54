"""The autotuner's search and cache logic on the CPU, with a stand-in for the
GPU timing: coordinate descent finds the fastest converged configuration of
a known cost surface, never picks a configuration that did not converge,
writes the cache entry keyed by batch shape and GPU, and reads it back with
defaults for parameters an older entry lacks."""
import json

import numpy as np


def _batch():
    from qdsim_b200 import workloads as W
    from qdsim_b200.batch import HostBatch
    return HostBatch([W.sweep_dot(i, nx=40 + 8 * i) for i in range(3)])


def test_search_finds_fastest_converged_configuration():
    from qdsim_b200 import autotune as AT
    best_target = {"chunk_rows": 2048, "shift_ev": 0.04, "block": 12, "stag_window": 8,
                   "tol32": 3e-7}
    calls = []

    def timer(cfg):
        calls.append(dict(cfg))
        ms = 100.0 + sum(0.0 if cfg[k] == v else 10.0 for k, v in best_target.items())
        if cfg["block"] == 16:          # pretend the wider block misses the target
            return ms - 50.0, False
        return ms, True

    best, best_ms, trace = AT.search(timer)
    assert best == best_target and best_ms == 100.0
    assert all(t["converged"] or t["config"]["block"] == 16 for t in trace)
    assert len(calls) == 1 + sum(len(v) - 1 for v in AT.SPACE.values())


def test_tune_writes_and_load_reads_the_cache(tmp_path):
    from qdsim_b200 import autotune as AT
    hb = _batch()
    cache = tmp_path / "tuned.json"

    def timer(cfg):
        return 50.0 - (cfg["chunk_rows"] == 512) * 5.0, True

    best, trace = AT.tune(hb, k=8, tol=1e-9, cache=cache, timer=timer, gpu_name="GPU-A")
    assert best["chunk_rows"] == 512
    assert AT.load(hb, 8, 1e-9, cache=cache, gpu_name="GPU-A") == best
    assert AT.load(hb, 8, 1e-9, cache=cache, gpu_name="GPU-B") is None       # per GPU
    assert AT.load(hb, 4, 1e-9, cache=cache, gpu_name="GPU-A") is None       # per k
    # an entry written before chunk_rows existed reads back with its default
    entries = json.loads(cache.read_text())
    key = next(iter(entries))
    del entries[key]["config"]["chunk_rows"]
    cache.write_text(json.dumps(entries))
    cfg = AT.load(hb, 8, 1e-9, cache=cache, gpu_name="GPU-A")
    assert cfg["chunk_rows"] == AT.DEFAULTS["chunk_rows"]
    kw = AT.solve_kwargs(cfg, 1e-9)
    assert kw["chunk_rows"] == 1024 and kw["b"] == cfg["block"]


def test_chunk_rows_sets_the_workspace_partials():
    """Fewer rows per chunk means more chunks and more per-chunk partial sums
    in the workspace; values outside [256, 8192] or not multiples of 64 fall
    back to 1024."""
    import ctypes as C
    from qdsim_b200 import _native as N
    L = N.lib()

    def ws(chunk):
        opts = np.zeros(1, dtype=N.LOBPCG_OPTS_DTYPE)
        opts["chunk_rows"] = chunk
        out = C.c_size_t()
        assert L.qd_lobpcg_workspace_size(4, 400000, 4000000, 12, 1, None, N.ptr(opts),
                                          C.byref(out)) == N.QD_OK
        return out.value

    assert ws(256) > ws(1024) > ws(4096)
    assert ws(1000) == ws(1024) == ws(0) == ws(16384)
