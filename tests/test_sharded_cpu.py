"""Host-side logic of the sector-sharded matvec, without a GPU.

* The partition: contiguous sector ranges covering every sector once, each
  rank within total/world + (largest sector cost) of the even share, empty
  ranges for ranks past the sector count.
* The windows: each rank's input window packs exactly the sectors it reads,
  its output window is its owned slice, and the exchange plan moves every
  read sector from its owner.
* The distributed Lanczos on gloo ranks (world sizes 2 and 3, processes
  started with spawn, rendezvous on 127.0.0.1) against numpy's dense
  eigensolver.  The operator is a random Hermitian matrix, block-sparse
  between "sectors" of uneven sizes (sector m' couples to m' - 1, m', m' + 1,
  as a charge shift of one would); each rank's stand-in matvec reads only its
  input window and writes only its owned slice.  No rank holds a whole
  vector: each rank's window and slice are shorter than the vector.  Lowest
  eigenvalue within 1e-10 relative, residual of the gathered eigenvector
  below 1e-8, every rank on the same eigenvalue and matvec count, and the
  eigenvector after HED's post-processing (phase of the largest entry, drop,
  FixComplexPrecision) equal to numpy's post-processed eigenvector (1e-8)."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from chainamps_b200.sharded import (ShardLayout, ShardedOperator, gather_needs, lanczos_lowest, partition_sectors,
                                    postprocess)


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
NSEC = len(OFFSETS) - 1


def _hermitian():
    """Random Hermitian matrix, non-zero only between sectors at most one apart."""
    rng = np.random.default_rng(7)
    A = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
    sec = np.searchsorted(OFFSETS, np.arange(N), side="right") - 1
    A[np.abs(sec[:, None] - sec[None, :]) > 1] = 0.0
    return (A + A.conj().T) / 2


def _needs(layout_ranges):
    """(world, NSEC): the sectors each rank's owned outputs read."""
    size = np.diff(OFFSETS)
    out = np.zeros((len(layout_ranges), NSEC), bool)
    for q, (a, b) in enumerate(layout_ranges):
        for mp_ in range(a, b):
            if size[mp_] == 0:
                continue
            for m in (mp_ - 1, mp_, mp_ + 1):
                if 0 <= m < NSEC and size[m] > 0:
                    out[q, m] = True
    return out


def test_windows_and_exchange_plan():
    costs = np.diff(OFFSETS).astype(float) ** 2
    size = np.diff(OFFSETS)
    for world in (2, 3, 4):
        lays = [ShardLayout(OFFSETS, costs, world, r) for r in range(world)]
        needs = _needs(lays[0].ranges)
        for L in lays:
            L.set_needs(needs)
        for r, L in enumerate(lays):
            read = [m for m in range(NSEC) if needs[r, m]]
            assert L.in_len == sum(size[m] for m in read)
            assert all(L.in_base[m] >= 0 for m in read)
            assert all(L.in_base[m] < 0 for m in range(NSEC) if not needs[r, m])
            assert L.out_len == L.n_local
            for m in range(L.m0, L.m1):
                assert L.out_base[m] == OFFSETS[m] - L.lo
            # what rank r receives from p is what p sends to r
            for p, Lp in enumerate(lays):
                assert L.recv_counts[p] == Lp.send_counts[r]
        # simulated exchange: every window holds the right entries
        x = np.arange(N, dtype=np.float64)
        for r, L in enumerate(lays):
            got = np.concatenate([x[Lp.lo:Lp.hi][Lp.send_idx[r]] for Lp in lays])
            want = np.concatenate([x[OFFSETS[m]:OFFSETS[m + 1]] for m in range(NSEC) if needs[r, m]])
            np.testing.assert_array_equal(got, want)


def _reference_postprocess(v):
    k = int(np.argmax(np.abs(v)))
    v = v * (abs(v[k]) / v[k])
    keep = np.abs(v) > np.finfo(float).eps * np.abs(v).max()
    out = np.zeros_like(v)
    out[keep] = v[keep]
    return out


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.set_num_threads(1)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        H = _hermitian()
        costs = np.diff(OFFSETS).astype(float) ** 2
        layout = ShardLayout(OFFSETS, costs, world, rank)
        mine = _needs(layout.ranges)[rank]
        layout.set_needs(gather_needs(mine))
        size = np.diff(OFFSETS)

        def apply_window(xin, yout):
            # only the window's sectors and the owned outputs are touched
            yout.fill_(float("nan"))
            xw = xin[0].numpy() + 1j * xin[1].numpy()
            for mp_ in range(layout.m0, layout.m1):
                if size[mp_] == 0:
                    continue
                acc = np.zeros(size[mp_], complex)
                for m in (mp_ - 1, mp_, mp_ + 1):
                    if 0 <= m < NSEC and size[m] > 0:
                        b = layout.in_base[m]
                        acc += H[OFFSETS[mp_]:OFFSETS[mp_ + 1], OFFSETS[m]:OFFSETS[m + 1]] @ xw[b:b + size[m]]
                o = layout.out_base[mp_]
                yout[0, o:o + size[mp_]] = torch.as_tensor(acc.real)
                yout[1, o:o + size[mp_]] = torch.as_tensor(acc.imag)

        op = ShardedOperator(layout, apply_window, "cpu")
        g = np.random.default_rng(99).standard_normal((2, N))
        x0 = torch.as_tensor(g[:, layout.lo:layout.hi]).contiguous()
        theta, x, mv, conv = lanczos_lowest(op, x0, None, tol=1e-12, krylov_dim=20, max_restarts=60)
        xp = postprocess(x)
        # gathered only for the check
        parts = [torch.zeros(2, layout.width, dtype=torch.float64) for _ in range(world)]
        pad = torch.zeros(2, layout.width, dtype=torch.float64)
        pad[:, :layout.n_local] = xp
        dist.all_gather(parts, pad)
        full = torch.cat([parts[r][:, :h - l] for r, (l, h) in enumerate(layout.spans)], dim=1)
        xv = full[0].numpy() + 1j * full[1].numpy()
        res = float(np.linalg.norm(H @ xv - theta * xv))
        q.put((rank, theta, mv, conv, res, layout.in_len, layout.n_local, xv))
    except Exception as e:  # reported to the parent
        q.put((rank, repr(e), None, None, None, None, None, None))
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
    w, V = np.linalg.eigh(_hermitian())
    want = _reference_postprocess(V[:, 0])
    thetas = set()
    for rank, theta, mv, conv, res, in_len, n_local, xv in out:
        assert isinstance(theta, float), theta
        assert conv
        assert abs(theta - w[0]) <= 1e-10 * abs(w[0]), (theta, w[0])
        assert res <= 1e-8, res
        assert in_len < N and n_local < N  # no rank holds a whole vector
        assert np.max(np.abs(xv - want)) <= 1e-8
        thetas.add((theta, mv))
    assert len(thetas) == 1  # every rank took the same steps
