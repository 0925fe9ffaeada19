"""The finite-sweep schedule (no GPU): the device driver's fDMRG.run, the
oracle's run_fdmrg and the oracle's excited-state run make the same moves,
in the same order, and record rows at the same steps as the reference's
FiniteDMRG::run (fDMRG_routines.cpp:19-66) and ExcitedStateFiniteDMRG::run
(:198-242), restated here with C++ loop semantics.  Moves are faked: only
the window position is tracked."""
import numpy as np
import pytest


def reference_moves(nvertices, sweeps):
    """[(direction, records_row)] of the reference's sweeps from the centre:
    for (r = right_size(); r > 0; --r) move right;
    for (l = left_size(); l > 0; --l) move left, row if left == right;
    for (r = right_size(); r > left_size(); --r) move right, row if
    left == right (the condition reads the left size as it grows)."""
    left = right = nvertices // 2 - 1
    out = []
    for _ in range(sweeps):
        r = right
        while r > 0:
            left, right = left + 1, right - 1
            out.append((+1, False))
            r -= 1
        l = left
        while l > 0:
            left, right = left - 1, right + 1
            out.append((-1, left == right))
            l -= 1
        r = right
        while r > left:
            left, right = left + 1, right - 1
            out.append((+1, left == right))
            r -= 1
    return out


@pytest.mark.parametrize("nvertices,sweeps", [(10, 2), (16, 3), (4, 1), (20, 1)])
def test_reference_schedule_ends_at_the_centre(nvertices, sweeps):
    moves = reference_moves(nvertices, sweeps)
    pos = nvertices // 2 - 1 + sum(d for d, _ in moves)
    assert pos == nvertices // 2 - 1
    assert sum(rec for _, rec in moves) == 2 * sweeps


@pytest.mark.parametrize("nvertices,sweeps", [(10, 2), (16, 3), (4, 1), (20, 1)])
def test_device_driver_schedule(nvertices, sweeps):
    from chainamps_b200.capi import fDMRG

    class Fake(fDMRG):
        def __init__(self, n):
            self.nvertices = n
            self.size = 0
            self.nl = 0
            self.log = []

        def grow(self, chi=0, max_trunc=0.0):
            self.size += 2
            self.nl = self.size // 2 - 1
            return ("grow", self.size)

        def position(self):
            return self.nl, self.size

        def move(self, direction, chi=0, max_trunc=0.0):
            self.nl += direction
            self.log.append(direction)
            return ("move", len(self.log))

        def close(self):
            pass

    run = Fake(nvertices)
    rows = run.run(sweeps, 8, 1e-16)
    ref = reference_moves(nvertices, sweeps)
    assert run.log == [d for d, _ in ref]
    recorded = [("move", i + 1) for i, (_, rec) in enumerate(ref) if rec]
    assert rows == [("grow", 2 * (k + 1)) for k in range(nvertices // 2)] + recorded


class FakeSuperBlock:
    """The part of the oracle's SuperBlock the schedule touches."""

    def __init__(self, *a, **k):
        self.size, self.nleft, self.log = 0, 0, []

    @property
    def nright(self):
        return self.size - self.nleft - 2

    def grow(self, chi=0, trunc=0.0):
        self.size += 2
        self.nleft = self.size // 2 - 1
        return ("grow", self.size)

    def finish_growth(self):
        pass

    def move_right(self, chi=0, trunc=0.0):
        self.nleft += 1
        self.log.append(+1)
        return ("move", len(self.log))

    def move_left(self, chi=0, trunc=0.0):
        self.nleft -= 1
        self.log.append(-1)
        return ("move", len(self.log))


@pytest.mark.parametrize("nvertices,sweeps", [(10, 2), (16, 3), (20, 1)])
def test_oracle_schedule(monkeypatch, nvertices, sweeps):
    from oracle import dmrg as od
    monkeypatch.setattr(od, "SuperBlock", FakeSuperBlock)
    sb, rows = od.run_fdmrg(None, nvertices, sweeps, 8)
    ref = reference_moves(nvertices, sweeps)
    assert sb.log == [d for d, _ in ref]
    recorded = [("move", i + 1) for i, (_, rec) in enumerate(ref) if rec]
    assert rows == [("grow", 2 * (k + 1)) for k in range(nvertices // 2)] + recorded


@pytest.mark.parametrize("nvertices,sweeps", [(10, 2), (16, 1)])
def test_oracle_excited_schedule(nvertices, sweeps):
    from oracle.excited import ExcitedSuperBlock

    class Fake(ExcitedSuperBlock):
        def __init__(self, n):
            self.size, self.nleft, self.log = n, n // 2 - 1, []

        def init(self, chi=0, trunc=0.0):
            return ("init",)

        move_right = FakeSuperBlock.move_right
        move_left = FakeSuperBlock.move_left

    ex = Fake(nvertices)
    rows = ex.run(sweeps, 8)
    ref = reference_moves(nvertices, sweeps)
    assert ex.log == [d for d, _ in ref]
    assert rows == [("init",)] + [("move", i + 1) for i, (_, rec) in enumerate(ref) if rec]
