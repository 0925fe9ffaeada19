"""Measured tile shapes (cmps_heff_autotune) on the GPU: tuning every grouped
GEMM plan of a handle -- the folded FP64 plans of the spin ladder, the
canonical FP64 plans of an Ising chain vertex, and the same plans in FP32
under split precision -- leaves the matvec within 1e-14 (FP64) of the
untuned one, reports the plans it timed, and a second handle of the same
operator takes every choice from the cache."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from chainamps_b200 import Context
    c = Context(0)
    yield c
    c.close()


def _ising_envs():
    """The 12-site, 64-state chain vertex: canonical order in FP64, and the
    FP32 canonical operator in split precision."""
    from tests.helpers import ising_mpo, to_tensor
    from tests.test_heff_gpu import make_envs
    H = ising_mpo(12, 64)
    L, R = make_envs(H, 5, 30, 28)
    return H.rules, to_tensor(L), to_tensor(H), to_tensor(R)


@pytest.mark.parametrize("case", ["ladder_fp64", "ising_fp64", "ising_fp32"])
def test_autotune_keeps_the_matvec(ctx, case):
    from chainamps_b200 import TwoVertexComponents, CMPS_FP64, CMPS_SPLIT_TF32, models
    if case == "ladder_fp64":
        wl = models.ladder_workload(96, 3)
        args = (wl["rules"], wl["L"], wl["Wt"], wl["R"])
        prec = CMPS_FP64
    else:
        args = _ising_envs()
        prec = CMPS_FP64 if case == "ising_fp64" else CMPS_SPLIT_TF32
    h0 = TwoVertexComponents(ctx, *args, precision=prec)
    x = np.random.default_rng(1).standard_normal(h0.n) + 1j * np.random.default_rng(2).standard_normal(h0.n)
    want = h0.multiply(x)
    h1 = TwoVertexComponents(ctx, *args, precision=prec)
    s1 = h1.autotune()
    assert s1["tuned"] + s1["cached"] >= 2
    got = h1.multiply(x)
    tol = 1e-14 if prec == CMPS_FP64 else 1e-5
    assert np.max(np.abs(got - want)) <= tol * np.max(np.abs(want))
    h2 = TwoVertexComponents(ctx, *args, precision=prec)
    s2 = h2.autotune()
    assert s2["tuned"] == 0 and s2["cached"] == s1["tuned"] + s1["cached"]
