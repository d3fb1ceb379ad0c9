"""The submatrix method over ranks (ptb_b200.distributed) on CPU gloo ranks,
with the oracle standing in for each rank's device share: the size-balanced
assignment, the bisection with one all-reduce per step and the assembly of P
must reproduce the one-process oracle."""
import os
import socket
import tempfile

import numpy as np
import pytest

from oracle import ptb_oracle as O
from ptb_b200 import Options, synth
from ptb_b200.distributed import assign_submatrices, mu_bisect, sm_stupid_simple_sharded
from shard_oracle import OracleShard

FILTER = 1e-4


def _system():
    return synth.alkane(6, seed=2)


def test_assignment_covers_and_balances():
    rng = np.random.default_rng(3)
    dims = rng.integers(20, 600, size=57)
    for nr in (1, 2, 3, 8):
        parts = assign_submatrices(dims, nr)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(dims)))
        loads = [sum(float(dims[k]) ** 3 for k in p) for p in parts]
        assert max(loads) - min(loads) <= float(max(dims)) ** 3
        assert parts == assign_submatrices(dims, nr)


def test_lattice_batch_split_over_ranks():
    """The 256-system lattice batch on N ranks (bench.py --workload lattice256
    --gpus N): every system on exactly one rank, loads within one largest
    system's ndim^3 of each other, and the split the same on every rank."""
    ndims = []
    for i in range(256):   # the sizes of synth.lattice_instance without building H and S
        rng = np.random.default_rng(11 * 1000003 + i)
        nat = int(rng.integers(20, 401))
        sym, _ = synth.lattice_geometry(nat, 11 * 7777 + i)
        ndims.append(sum(synth.AO_PER_ELEMENT[s] for s in sym))
    assert min(ndims) == 166 and max(ndims) == 3064
    for nr in (2, 4, 8):
        parts = assign_submatrices(ndims, nr)
        assert sorted(k for p in parts for k in p) == list(range(256))
        loads = [sum(float(ndims[k]) ** 3 for k in p) for p in parts]
        assert max(loads) - min(loads) <= float(max(ndims)) ** 3
        assert max(loads) <= 1.05 * sum(loads) / nr
        assert parts == assign_submatrices(list(ndims), nr)


@pytest.mark.parametrize("columns", [1, 2])
def test_single_process_matches_oracle(columns):
    s = _system()
    n = s.ndim
    o = Options(filter=FILTER)
    P, info = sm_stupid_simple_sharded(OracleShard(), n, s.nel, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat, columns, 2,
                                       opts=o)
    ref = O.sm_stupid_simple(n, s.nel, O.filter_matrix_sym(s.Hvec, FILTER), O.filter_matrix_sym(s.Svec, FILTER),
                             s.nat, s.xyz, s.aoat, columns, 2)
    assert info.mu == ref.mu
    assert np.max(np.abs(P - ref.Pvec)) < 1e-13


def test_bisection_restates_the_reference():
    """mu_bisect on a monotone staircase: the reference's stop rule and final pass."""
    levels = np.linspace(-1.0, 1.0, 41)
    nel_fn = lambda mu: 2.0 * float(np.sum(levels < mu)) + float(np.sum(levels == mu))
    mu, nel, trace, ok = mu_bisect(nel_fn, 40.0)
    assert ok and abs(nel - 40.0) < 1e-5 and len(trace) >= 1


def _worker(rank, world, port, out, columns):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        s = _system()
        P, info = sm_stupid_simple_sharded(OracleShard(), s.ndim, s.nel, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat,
                                           columns, 2, opts=Options(filter=FILTER))
        np.save(os.path.join(out, f"P{rank}.npy"), P)
        np.save(os.path.join(out, f"ids{rank}.npy"), np.asarray(info.local, dtype=np.int64))
        np.save(os.path.join(out, f"mu{rank}.npy"), np.array([info.mu]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_oracle():
    columns = 1   # one submatrix per column: the most submatrices to split
    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")   # the two ranks share the host cores
    with tempfile.TemporaryDirectory() as out:
        mp.spawn(_worker, args=(2, port, out, columns), nprocs=2, join=True)
        P0, P1 = np.load(os.path.join(out, "P0.npy")), np.load(os.path.join(out, "P1.npy"))
        ids0, ids1 = np.load(os.path.join(out, "ids0.npy")), np.load(os.path.join(out, "ids1.npy"))
        mu0, mu1 = np.load(os.path.join(out, "mu0.npy")), np.load(os.path.join(out, "mu1.npy"))
    s = _system()
    ref = O.sm_stupid_simple(s.ndim, s.nel, O.filter_matrix_sym(s.Hvec, FILTER), O.filter_matrix_sym(s.Svec, FILTER),
                             s.nat, s.xyz, s.aoat, columns, 2)
    assert len(ids0) > 0 and len(ids1) > 0 and not set(ids0) & set(ids1)
    assert np.array_equal(P0, P1) and mu0[0] == mu1[0]
    assert np.max(np.abs(P0 - ref.Pvec)) < 1e-12


class _FailingShard(OracleShard):
    """The oracle shard with a planted failure on one rank (host-side error
    injection: the failing phase raises the library's exception type)."""

    def __init__(self, rank, fail_rank, where):
        self.rank, self.fail_rank, self.where, self.calls = rank, fail_rank, where, 0

    def _maybe_fail(self, where):
        if self.rank == self.fail_rank and self.where == where:
            from ptb_b200.api import ENOTSPD, PtbGpuError
            raise PtbGpuError(ENOTSPD, f"planted failure in {where}")

    def prepare(self, ids):
        self._maybe_fail("prepare")
        return super().prepare(ids)

    def nel(self, mu):
        self.calls += 1
        if self.calls == 3:
            self._maybe_fail("nel")
        return super().nel(mu)

    def finish(self, ndim, mu):
        self._maybe_fail("finish")
        return super().finish(ndim, mu)


def _failing_worker(rank, world, port, out, where):
    import datetime

    import torch.distributed as dist
    from ptb_b200.api import PtbGpuError
    # a short timeout: a rank left waiting in a collective ends the test with an error, not a hang
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        s = _system()
        try:
            sm_stupid_simple_sharded(_FailingShard(rank, 1, where), s.ndim, s.nel, s.Hvec, s.Svec, s.nat, s.xyz,
                                     s.aoat, 1, 2, opts=Options(filter=FILTER))
            msg = "no error"
        except PtbGpuError as e:
            msg = f"{e.code}|{e}"
        with open(os.path.join(out, f"r{rank}.txt"), "w") as f:
            f.write(msg)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("where", ["prepare", "nel", "finish"])
def test_a_failing_rank_fails_every_rank(where):
    """A failure on rank 1 in any phase reaches rank 0 through the protocol's own
    all-reduces: rank 1 raises its own error, rank 0 a PtbGpuError with the same
    code naming rank 1, and neither waits for the process-group timeout."""
    import time

    import torch.multiprocessing as mp
    from ptb_b200.api import ENOTSPD
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    t0 = time.perf_counter()
    with tempfile.TemporaryDirectory() as out:
        mp.spawn(_failing_worker, args=(2, port, out, where), nprocs=2, join=True)
        r0 = open(os.path.join(out, "r0.txt")).read()
        r1 = open(os.path.join(out, "r1.txt")).read()
    assert time.perf_counter() - t0 < 50.0
    assert r1.startswith(f"{ENOTSPD}|") and "planted failure" in r1
    assert r0.startswith(f"{ENOTSPD}|") and "rank 1 failed" in r0


def test_a_rank_with_an_empty_share():
    """The full-matrix grouping has one submatrix: on two ranks one of them prepares
    nothing, still takes every collective step, and both return the oracle's P."""
    import torch.multiprocessing as mp
    columns = 3
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    with tempfile.TemporaryDirectory() as out:
        mp.spawn(_worker, args=(2, port, out, columns), nprocs=2, join=True)
        P0, P1 = np.load(os.path.join(out, "P0.npy")), np.load(os.path.join(out, "P1.npy"))
        ids = [np.load(os.path.join(out, f"ids{r}.npy")) for r in (0, 1)]
    s = _system()
    ref = O.sm_stupid_simple(s.ndim, s.nel, O.filter_matrix_sym(s.Hvec, FILTER), O.filter_matrix_sym(s.Svec, FILTER),
                             s.nat, s.xyz, s.aoat, columns, 2)
    assert sorted(len(x) for x in ids) == [0, 1]
    assert np.array_equal(P0, P1)
    assert np.max(np.abs(P0 - ref.Pvec)) < 1e-12
