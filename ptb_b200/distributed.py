"""The submatrix method over ranks: one process per GPU, torch.distributed.

sm_stupid_simple (source/sm.f90:34-409) solves independent submatrices that
couple only through the chemical-potential bisection: every step needs the
electron count summed over all submatrices (source/sm.f90:322-340).  Here each
rank plans the whole system (grouping, pattern scan: cheap and identical on
every rank), prepares a size-balanced share of the submatrices on its own
device, and every rank runs the same bisection with one all-reduce of the
partial electron count per step.  The owned columns of P are disjoint between
ranks, so one all-reduce (sum) of the packed P assembles the result.

Errors are collective: each all-reduce also carries one status word per rank
(0, or the failing rank's PTBGPU_E* code; -1 for a host exception).  A rank
whose plan or prepare phase fails still joins the first bisection all-reduce,
one whose finish phase fails joins the all-reduce of P, and after that
collective every rank raises.  No rank is left waiting in a collective that a
failed peer will never join.

The per-rank device work goes through the C-ABI phases (ptbgpu_sm_plan /
_prepare / _nel / _finish); anything with the same four methods can stand in
for it (the tests drive the protocol with the CPU oracle on gloo ranks).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .api import EINVAL, EITER, Context, Options, PtbGpuError

# REAL(4) literals of the reference's stop test, source/sm.f90:191-192
TOL_MU = float(np.float32(1e-3))
TOL_NEL = float(np.float32(1e-5))


def assign_submatrices(dims, nranks: int) -> list:
    """Size-balanced assignment: submatrices in decreasing dim^3 (ties: lower
    index) go to the rank with the least accumulated dim^3 (ties: lower rank).
    Deterministic, so every rank computes the same assignment.  Returns one
    sorted list of 0-based submatrix indices per rank."""
    dims = [int(d) for d in dims]
    order = sorted(range(len(dims)), key=lambda k: (-dims[k], k))
    loads = [0.0] * nranks
    out = [[] for _ in range(nranks)]
    for k in order:
        r = min(range(nranks), key=lambda q: (loads[q], q))
        out[r].append(k)
        loads[r] += float(dims[k]) ** 3
    return [sorted(v) for v in out]


def mu_bisect(nel_fn, nelref: float, mua: float = -10.0, mub: float = 10.0, maxiter: int = 100):
    """Chemical-potential bisection of source/sm.f90:191-383: mu = (a + b)/2,
    stop when |a - b| < 1e-3 or |nel - nelref| < 1e-5 (REAL(4) literals), then
    one final evaluation at the same mu; nel > nelref moves b.  Returns
    (mu, nel, [(mu, nel) per step], converged)."""
    finaliter = False
    mu = nel = 0.0
    trace = []
    for _ in range(maxiter):
        mu = 0.5 * (mua + mub)
        nel = nel_fn(mu)
        if finaliter:
            break
        trace.append((mu, nel))
        if abs(mua - mub) < TOL_MU or abs(nel - nelref) < TOL_NEL:
            finaliter = True
        if not finaliter:
            if nel > nelref:
                mub = mu
            else:
                mua = mu
    return mu, nel, trace, finaliter


class DeviceShard:
    """One rank's share of the step on its device, through the C-ABI phases."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def plan(self, ndim, Hvec, Svec, n, xyz, aoat, columns, mode, partition, opts):
        return self.ctx.sm_plan(ndim, Hvec, Svec, n, xyz, aoat, columns, mode, partition, opts)

    def prepare(self, ids):
        return self.ctx.sm_prepare(ids)

    def nel(self, mu: float) -> float:
        return self.ctx.sm_nel(mu)

    def finish(self, ndim: int, mu: float) -> np.ndarray:
        return self.ctx.sm_finish(ndim, mu)


def _status_code(err) -> int:
    if err is None:
        return 0
    return int(err.code) if isinstance(err, PtbGpuError) else -1


def _raise_failures(status, err, phase: str):
    """Raises on every rank when any rank's status word is set: the failing rank
    re-raises its own error, the others a PtbGpuError naming the first failing
    rank and its code (EINVAL for a host exception)."""
    failed = [(r, int(c)) for r, c in enumerate(status) if c != 0]
    if not failed:
        return
    if err is not None:
        raise err
    r, c = failed[0]
    raise PtbGpuError(c if c > 0 else EINVAL, f"rank {r} failed in the {phase} phase (status {c})")


@dataclass
class ShardInfo:
    mu: float
    nel: float
    nsm: int
    local: list
    dims: np.ndarray
    trace: list = field(default_factory=list)


def sm_stupid_simple_sharded(shard, ndim: int, nelref: int, Hvec: np.ndarray, Svec: np.ndarray, n: int,
                             xyz: np.ndarray, aoat: np.ndarray, submatrix_columns: int, submatrix_mode: int,
                             partition=None, opts: Options | None = None, group=None):
    """sm_stupid_simple over the ranks of `group` (all ranks call it with the
    same arguments; without an initialised process group it runs alone).
    Returns (packed P, ShardInfo) on every rank."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
    rank = dist.get_rank(group) if world > 1 else 0
    dims, ids, err = np.zeros(0, dtype=np.int64), [], None
    try:
        dims = np.asarray(shard.plan(ndim, Hvec, Svec, n, xyz, aoat, submatrix_columns, submatrix_mode, partition,
                                     opts or Options()))
        ids = assign_submatrices(dims, world)[rank]
        shard.prepare(ids)
    except Exception as e:   # noqa: BLE001 -- reported to the peers, then re-raised
        if world == 1:
            raise
        err = e
    dev = torch.device("cpu")
    if world > 1 and dist.get_backend(group) == "nccl":
        dev = torch.device("cuda", torch.cuda.current_device())
    phase = ["plan, prepare or first bisection step"]

    def nel_total(mu: float) -> float:
        nonlocal err
        if world == 1:
            return shard.nel(mu)
        v = 0.0
        if err is None:
            try:
                v = shard.nel(mu)
            except Exception as e:   # noqa: BLE001
                err = e
        t = torch.zeros(1 + world, dtype=torch.float64, device=dev)
        t[0] = v
        t[1 + rank] = _status_code(err)
        dist.all_reduce(t, group=group)
        h = t.cpu().tolist()
        _raise_failures(h[1:], err, phase[0])
        phase[0] = "bisection"   # later failures happen in a bisection step
        return h[0]

    mu, nel, trace, ok = mu_bisect(nel_total, float(nelref))
    if not ok:
        raise PtbGpuError(EITER, "chemical potential bisection did not converge")
    if world == 1:
        return shard.finish(ndim, mu), ShardInfo(mu, nel, int(dims.shape[0]), ids, dims, trace)
    npk = ndim * (ndim + 1) // 2
    P = np.zeros(npk)
    try:
        P = shard.finish(ndim, mu)
    except Exception as e:   # noqa: BLE001
        err = e
    t = torch.zeros(npk + world, dtype=torch.float64, device=dev)
    if err is None:
        t[:npk] = torch.from_numpy(np.ascontiguousarray(P, dtype=np.float64)).to(dev)
    t[npk + rank] = _status_code(err)
    dist.all_reduce(t, group=group)
    h = t.cpu().numpy()
    _raise_failures(h[npk:], err, "finish")
    return h[:npk].copy(), ShardInfo(mu, nel, int(dims.shape[0]), ids, dims, trace)
