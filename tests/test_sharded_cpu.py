"""Host-side logic of the sector-sharded matvec, without a GPU.

* The partition: contiguous sector ranges covering every sector once, each
  rank within total/world + (largest sector cost) of the even share, empty
  ranges for ranks past the sector count.
* The distributed Lanczos on gloo ranks (world sizes 2 and 3, processes
  started with spawn, rendezvous on 127.0.0.1) against numpy's dense
  eigensolver.  The operator is a random Hermitian matrix split into
  "sectors" of uneven sizes; each rank's stand-in matvec computes only the
  rows of its own sectors and writes NaN everywhere else, so a rank that
  used another rank's output, or an all-gather that left a gap, would end
  in NaN.  Lowest eigenvalue within 1e-10 relative, residual of the
  gathered eigenvector below 1e-8, every rank on the same eigenvalue and
  matvec count."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from chainamps_b200.sharded import ShardLayout, ShardedOperator, lanczos_lowest, partition_sectors


def test_partition_covers_and_balances():
    rng = np.random.default_rng(5)
    for trial in range(200):
        n = int(rng.integers(1, 60))
        world = int(rng.integers(1, 9))
        costs = rng.exponential(1.0, n) * (rng.random(n) < 0.9)
        ranges = partition_sectors(costs, world)
        assert len(ranges) == world
        assert ranges[0][0] == 0 and ranges[-1][1] == n
        for (a0, a1), (b0, b1) in zip(ranges, ranges[1:]):
            assert a1 == b0 and a0 <= a1
        loads = [costs[a:b].sum() for a, b in ranges]
        assert max(loads) <= costs.sum() / world + costs.max() + 1e-12, (costs, ranges)


def test_partition_more_ranks_than_sectors():
    ranges = partition_sectors([1.0, 2.0], 5)
    assert sum(b - a for a, b in ranges) == 2
    assert sum(1 for a, b in ranges if b > a) <= 2


def test_layout_spans_are_contiguous_slices():
    offsets = [0, 10, 10, 45, 60, 100]
    lay = [ShardLayout(offsets, [1, 0, 3, 1, 4], 3, r) for r in range(3)]
    spans = lay[0].spans
    assert spans[0][0] == 0 and spans[-1][1] == 100
    for (a0, a1), (b0, b1) in zip(spans, spans[1:]):
        assert a1 == b0
    for r, L in enumerate(lay):
        assert (L.lo, L.hi) == spans[r]
        assert L.owned.sum() == L.m1 - L.m0
        assert L.width == max(h - l for l, h in spans)


N = 230
OFFSETS = [0, 17, 17, 60, 61, 120, 171, 200, 230]


def _hermitian():
    rng = np.random.default_rng(7)
    A = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
    return (A + A.conj().T) / 2


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.set_num_threads(1)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        H = torch.as_tensor(_hermitian())
        costs = np.diff(OFFSETS).astype(float) ** 2
        layout = ShardLayout(OFFSETS, costs, world, rank)

        def apply_full(xin, yout):
            y = H @ torch.complex(xin[0], xin[1])
            yout.fill_(float("nan"))
            yout[0, layout.lo:layout.hi] = y.real[layout.lo:layout.hi]
            yout[1, layout.lo:layout.hi] = y.imag[layout.lo:layout.hi]

        op = ShardedOperator(layout, apply_full, "cpu")
        g = np.random.default_rng(99).standard_normal((2, N))
        x0 = torch.as_tensor(g[:, layout.lo:layout.hi]).contiguous()
        theta, x, mv, conv = lanczos_lowest(op, x0, None, tol=1e-12, krylov_dim=20, max_restarts=60)
        full = op.gather(x).clone()
        xv = torch.complex(full[0], full[1])
        res = float(torch.linalg.norm(H @ xv - theta * xv))
        q.put((rank, theta, mv, conv, res))
    except Exception as e:  # reported to the parent
        q.put((rank, repr(e), None, None, None))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_distributed_lanczos_on_gloo_ranks(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = np.linalg.eigvalsh(_hermitian())[0]
    thetas = set()
    for rank, theta, mv, conv, res in out:
        assert isinstance(theta, float), theta
        assert conv
        assert abs(theta - want) <= 1e-10 * abs(want), (theta, want)
        assert res <= 1e-8, res
        thetas.add((theta, mv))
    assert len(thetas) == 1  # every rank took the same steps
