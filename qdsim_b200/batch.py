"""Batches of independent dots packed as one disjoint-union mesh.

The union's reduced DOFs are numbered dot by dot, so its CSR pattern is block
diagonal: one assembly launch fills every dot's H and M, and one batched
LOBPCG call solves them all.  Per-shape CSR patterns (and assembly plans) are
built once on the host and replicated with offsets.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _native as N
from .eigen import DSTPreconditioner, EigResult, Workspace, lobpcg_packed
from .fem import build_pattern, dof_map_for, stream_ptr

_SHAPE_CACHE: dict = {}


def _shape_pattern(mesh, dirichlet=True):
    key = (mesh.shape_key(), dirichlet)
    if key not in _SHAPE_CACHE:
        dm, n = dof_map_for(mesh, dirichlet)
        _SHAPE_CACHE[key] = (dm, n, build_pattern(mesh.elems, dm, n, mesh.num_nodes))
    return _SHAPE_CACHE[key]


class HostBatch:
    """Host (numpy) arrays of the union mesh, its pattern and coefficients."""

    def __init__(self, dots, dirichlet=True, precondition=True):
        if not dots:
            raise ValueError("empty batch")
        order = dots[0].mesh.order
        if any(d.mesh.order != order for d in dots):
            raise ValueError("all dots in a batch must share the element order")
        self.order = order
        self.n_dots = len(dots)
        nodes, elems, dmaps, cs, Vs = [], [], [], [], []
        rowptr, col, adjptr, adj, cptr, contrib, slotcnt = [], [], [], [], [], [], []
        node_off = elem_off = row_off = nnz_off = adj_off = con_off = 0
        self.row_off = [0]
        self.nnz_per_dot = []
        self.rows_per_dot = []
        for d in dots:
            m = d.mesh
            dm, n, P = _shape_pattern(m, dirichlet)
            nodes.append(m.nodes)
            elems.append(m.elems + node_off)
            dmaps.append(np.where(dm >= 0, dm + row_off, -1))
            cs.append(np.asarray(d.c, np.float64))
            Vs.append(np.asarray(d.V, np.float64))
            rowptr.append(P.rowptr[:-1] + nnz_off)
            col.append(P.col + row_off)
            adjptr.append(P.adjptr[:-1] + adj_off)
            adj.append(P.adj + (elem_off << 4))
            cptr.append(P.cptr[:-1] + con_off)
            contrib.append(P.contrib)
            slotcnt.append(P.slotcnt)
            node_off += m.num_nodes
            elem_off += m.num_elements
            row_off += n
            nnz_off += P.nnz
            adj_off += P.adj.size
            con_off += P.contrib.size
            self.row_off.append(row_off)
            self.nnz_per_dot.append(P.nnz)
            self.rows_per_dot.append(n)
        if nnz_off >= 2**31 or con_off >= 2**31 or elem_off >= 2**27:
            raise ValueError("batch too large for the int32 CSR / plan indices")
        i32 = lambda parts, last: np.ascontiguousarray(  # noqa: E731
            np.concatenate(parts + [np.array([last], np.int64)]).astype(np.int32))
        self.arrays = {
            "nodes": np.ascontiguousarray(np.concatenate(nodes).astype(np.float64)),
            "elems": np.ascontiguousarray(np.concatenate(elems).astype(np.int32)),
            "c": np.ascontiguousarray(np.concatenate(cs)),
            "V": np.ascontiguousarray(np.concatenate(Vs)),
            "rowptr": i32(rowptr, nnz_off),
            "col": np.ascontiguousarray(np.concatenate(col).astype(np.int32)),
            "adjptr": i32(adjptr, adj_off),
            "adj": np.ascontiguousarray(np.concatenate(adj).astype(np.int32)),
            "cptr": i32(cptr, con_off),
            "contrib": np.ascontiguousarray(np.concatenate(contrib)),
            "slotcnt": np.ascontiguousarray(np.concatenate(slotcnt)),
        }
        self.dof_map = np.concatenate(dmaps).astype(np.int32)
        self.num_nodes = node_off
        self.num_elems = elem_off
        self.n = row_off
        self.nnz = nnz_off
        self.row_off = np.asarray(self.row_off, dtype=np.int32)
        self._prec_src = [(d.mesh, d.c, d.V) for d in dots] if (precondition and dirichlet) else None
        self.prec_specs = self.prec_specs_for(None)

    def prec_specs_for(self, shift_ev):
        """Per-dot DST preconditioner specs with the given shift (eV; None:
        the default), or None for a batch without preconditioning."""
        if self._prec_src is None:
            return None
        return [DSTPreconditioner.spec_for(m, c, V, shift_ev) for m, c, V in self._prec_src]

    def pin(self):
        """Page-locked copies of the input arrays (for timed host->device copies)."""
        return {k: torch.from_numpy(v).pin_memory() for k, v in self.arrays.items()}

    def input_bytes(self) -> int:
        return int(sum(v.nbytes for v in self.arrays.values()))


class DeviceBatch:
    """Device-resident union mesh; ``assemble`` + ``solve`` are the hot path."""

    def __init__(self, host: HostBatch, device="cuda"):
        self.host = host
        self.device = torch.device(device)
        self.d = {k: torch.empty(v.shape, dtype=torch.from_numpy(v[:0]).dtype, device=self.device)
                  for k, v in host.arrays.items()}
        self.H = torch.empty(host.nnz, dtype=torch.float64, device=self.device)
        self.M = torch.empty(host.nnz, dtype=torch.float64, device=self.device)
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.ws = Workspace(self.device)
        self.precond = (DSTPreconditioner(host.prec_specs, self.device)
                        if host.prec_specs is not None else None)

    def set_shift(self, shift_ev):
        """Rebuild the DST preconditioner with another shift (eV)."""
        specs = self.host.prec_specs_for(shift_ev)
        self.precond = DSTPreconditioner(specs, self.device) if specs is not None else None

    def upload(self, pinned=None, non_blocking=True):
        src = pinned if pinned is not None else {k: torch.from_numpy(v) for k, v in self.host.arrays.items()}
        for k, t in src.items():
            self.d[k].copy_(t, non_blocking=non_blocking)

    def assemble(self, stream=None):
        h, d = self.host, self.d
        self.status.zero_()
        N.check(N.lib().qd_assemble(
            h.order, N.QD_ASM_FEM, h.num_nodes, h.num_elems, h.n, N.ptr(d["nodes"]),
            N.ptr(d["elems"]), N.ptr(d["c"]), N.ptr(d["V"]), None, N.ptr(d["rowptr"]),
            N.ptr(d["adjptr"]), N.ptr(d["adj"]), N.ptr(d["cptr"]), N.ptr(d["contrib"]),
            N.ptr(d["slotcnt"]), N.ptr(self.H), N.ptr(self.M), None, N.ptr(self.status),
            stream_ptr(stream)), "qd_assemble")

    def solve(self, k, **kw):
        h = self.host
        kw.setdefault("precond", self.precond)
        return lobpcg_packed(h.row_off, self.d["rowptr"], self.d["col"], self.H, self.M, k,
                             workspace=self.ws, **kw)

    def check_status(self):
        flag = int(self.status.item())
        if flag:
            raise N.QDError(N.QD_ERR_DEGENERATE, f"qd_assemble (flag {flag})")


class SweepPipeline:
    """Repeated assemble-and-solve of one batch shape with the host <-> device
    copies overlapped with the solves.

    Two device batches alternate.  While step s assembles and solves on the
    current stream, step s+1's inputs are copied up into the other batch and
    step s-1's eigenvalues and eigenvectors are copied down, both on a copy
    stream; every step still moves all of its inputs and results.  The solve
    call returns only when its step is done, so the other batch is free when
    its next upload is issued.
    """

    def __init__(self, host: HostBatch, device="cuda", shift_ev=None):
        self.device = torch.device(device)
        self.batches = [DeviceBatch(host, self.device), DeviceBatch(host, self.device)]
        if shift_ev is not None:
            for b in self.batches:
                b.set_shift(shift_ev)
        self.copy = torch.cuda.Stream(device=self.device)

    def run(self, steps, k, inputs, out_E, out_X, **solve_kw):
        """``inputs(s)``: dict of pinned host arrays of step s (``HostBatch.pin``);
        ``out_E(s)``, ``out_X(s)``: pinned host tensors receiving step s's E
        ([n_dots, k]) and X ([n_rows, k]).  Returns the last step's solver info."""
        comp = torch.cuda.current_stream(self.device)
        ready = [torch.cuda.Event(), torch.cuda.Event()]
        with torch.cuda.stream(self.copy):
            self.batches[0].upload(inputs(0), non_blocking=True)
            ready[0].record(self.copy)
        info = None
        for s in range(steps):
            i = s % 2
            if s + 1 < steps:
                with torch.cuda.stream(self.copy):
                    self.batches[1 - i].upload(inputs(s + 1), non_blocking=True)
                    ready[1 - i].record(self.copy)
            comp.wait_event(ready[i])
            db = self.batches[i]
            db.assemble()
            # the same batch every step: the set-up reads nothing back and
            # copies no unchanged table, so that no small copy of the solver
            # queues behind this pipeline's own large ones
            E, X, _, _, info, _ = db.solve(k, setup_cached=True, **solve_kw)
            done = torch.cuda.Event()
            done.record(comp)
            self.copy.wait_event(done)
            with torch.cuda.stream(self.copy):
                out_E(s).copy_(E, non_blocking=True)
                out_X(s).copy_(X, non_blocking=True)
            E.record_stream(self.copy)
            X.record_stream(self.copy)
        comp.wait_stream(self.copy)
        return info


# ---------------------------------------------------------------------------
# Sharding a fixed set of dots (or bias points) over ranks
# ---------------------------------------------------------------------------

# CSR nonzeros per row of the P1 / P2 / P3 stiffness pattern on the structured
# mesh (the average over a 60 x 30-cell mesh), the cost model's row weight
_NNZ_PER_ROW = {1: 6.8, 2: 11.3, 3: 16.8}


def dot_cost(dot) -> float:
    """Predicted solve cost of a dot: its stiffness nonzeros.  With the DST
    preconditioner the LOBPCG iteration count hardly depends on the grid, so
    nonzeros x iterations is proportional to the nonzeros."""
    m = dot.mesh
    return float(m.num_nodes) * _NNZ_PER_ROW[int(m.order)]


def partition_by_cost(costs, parts: int):
    """Longest-processing-time-first split of items with ``costs`` into
    ``parts`` groups: items in decreasing cost (ties by index), each to the
    group with the least load so far (the lowest-numbered on ties).  The
    heaviest group is within 4/3 of the best possible split.  Returns one
    sorted index array per group; every rank computes the same split."""
    costs = np.asarray(costs, dtype=np.float64).reshape(-1)
    if parts < 1:
        raise ValueError("parts must be at least 1")
    if not np.all(np.isfinite(costs)) or (costs < 0).any():
        raise ValueError("costs must be finite and non-negative")
    order = np.argsort(-costs, kind="stable")
    load = np.zeros(parts)
    groups = [[] for _ in range(parts)]
    for i in order:
        g = int(np.argmin(load))
        groups[g].append(int(i))
        load[g] += costs[i]
    return [np.array(sorted(g), dtype=np.int64) for g in groups]


def shard_dots(dots, rank: int, world: int):
    """(indices, dots) of this rank's share of ``dots``, split by
    ``partition_by_cost`` on ``dot_cost``; the shards are disjoint and cover
    every dot, and no data moves between ranks during the solves."""
    if not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    idx = partition_by_cost([dot_cost(d) for d in dots], world)[rank]
    return idx, [dots[i] for i in idx]


def gather_by_index(local, indices, n_items: int, group=None):
    """Reassemble per-item host results from every rank's shard: ``local``
    holds this rank's rows for ``indices``; the rows of all ranks are
    all-gathered (small host objects over the process group) and returned in
    item order, shape (n_items, ...).  Without an initialised process group
    the local rows are returned in item order."""
    local = np.asarray(local)
    indices = np.asarray(indices, dtype=np.int64)
    if local.shape[0] != indices.size:
        raise ValueError("one row of results per index")
    import torch.distributed as dist
    parts = [(indices, local)]
    if dist.is_available() and dist.is_initialized():
        parts = [None] * dist.get_world_size(group)
        dist.all_gather_object(parts, (indices, local), group=group)
    out = None
    seen = np.zeros(n_items, dtype=bool)
    for idx, rows in parts:
        rows = np.asarray(rows)
        if out is None:
            out = np.zeros((n_items,) + rows.shape[1:], dtype=rows.dtype)
        if seen[idx].any():
            raise ValueError("an item appears in more than one shard")
        out[idx] = rows
        seen[idx] = True
    if not seen.all():
        raise ValueError("the shards do not cover every item")
    return out


def solve_dots(dots, k, device="cuda", **kw) -> EigResult:
    """Assemble and solve a list of ``workloads.Dot`` on the GPU."""
    hb = HostBatch(dots)
    db = DeviceBatch(hb, device)
    db.upload(non_blocking=False)
    db.assemble()
    db.check_status()
    E, X, R, it, info, st = db.solve(k, **kw)
    ro = hb.row_off
    return EigResult(E.cpu().numpy(), [X[ro[i]:ro[i + 1]] for i in range(hb.n_dots)],
                     R.cpu().numpy(), it.cpu().numpy(), info, st)
