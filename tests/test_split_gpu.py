"""GPU parity of the split-precision form (3-term TF32 on tcgen05, FP32
accumulation) against the oracle, through the C ABI.

Tolerances, stated: the split-TF32 matvec agrees with the FP64 oracle to
2e-5 relative (max-norm over the output, relative to its largest entry) at
the unit-test sizes, and at the chi = 512 benchmark size to 3e-4 max-norm
and 1e-4 rms (measured on B200: 4.8e-5 / 3.4e-5 with 3.5-wide charge
sectors, 1.2e-4 / 8.5e-5 with 1.2-wide ones, whose K is ~3x longer): each
product keeps ~22 mantissa bits, but sums are accumulated in FP32 over K of
up to ~4e4 terms, so the error grows with K.
Ground-state energies, which the solver takes from an FP64 Rayleigh
quotient of the split-precision eigenvector, agree with the FP64 solver to
1e-9 relative, the accuracy the mixed-precision form is held to."""
import numpy as np
import pytest

from oracle import dmrg as od
from tests.helpers import to_tensor, model_zoo
from tests.test_heff_gpu import make_envs, CHI, grown

pytestmark = pytest.mark.gpu

ZOO = model_zoo()
SPLIT_RTOL = 2e-5
SCALE_RTOL = 3e-4


@pytest.fixture(scope="module")
def ctx():
    from chainamps_b200 import Context
    c = Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("name", sorted(ZOO))
def test_split_matvec_matches_oracle(ctx, name):
    from chainamps_b200 import TwoVertexComponents, CMPS_SPLIT_TF32
    H = ZOO[name]
    L, R = make_envs(H, 7, *CHI[name])
    ref = od.TwoVertexComponents(L, H, R)
    gpu = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R), precision=CMPS_SPLIT_TF32)
    rng = np.random.default_rng(11)
    for _ in range(2):
        x = rng.standard_normal(gpu.n) + 1j * rng.standard_normal(gpu.n)
        want = ref.matvec(x)
        got = gpu.multiply(x)
        err = np.max(np.abs(got - want)) / np.max(np.abs(want))
        assert err <= SPLIT_RTOL, err


def test_split_matvec_larger_sectors(ctx):
    """Sectors wider than one 128-row tile and K longer than one stage ring."""
    from chainamps_b200 import TwoVertexComponents, CMPS_SPLIT_TF32, CMPS_FP64
    from tests.helpers import random_bond, random_left_block, random_right_block
    H = ZOO["xxz"]
    rng = np.random.default_rng(12)
    pool = [(0,), (1,), (2,)]           # three sectors of ~100-150 elements each
    bq = H.indices[1].charges
    L = random_left_block(rng, H.rules, random_bond(rng, 300, pool), bq)
    R = random_right_block(rng, H.rules, random_bond(rng, 260, pool), bq)
    g64 = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R), precision=CMPS_FP64)
    g32 = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R), precision=CMPS_SPLIT_TF32)
    rng = np.random.default_rng(2)
    x = rng.standard_normal(g64.n) + 1j * rng.standard_normal(g64.n)
    a, b = g64.multiply(x), g32.multiply(x)
    assert np.max(np.abs(a - b)) / np.max(np.abs(a)) <= SPLIT_RTOL


@pytest.mark.parametrize("name,steps,chi", [("xxz", 6, 24), ("tfim", 3, 20)])
def test_split_ground_state_energy(ctx, name, steps, chi):
    from chainamps_b200 import TwoVertexComponents, CMPS_SPLIT_TF32, CMPS_FP64
    H = ZOO[name]
    sb = grown(H, steps, chi)
    L = od.make_left_block(sb.left_blocks[sb.nleft], H, sb.dec.U)
    R = od.make_right_block(sb.right_blocks[sb.nleft], H, sb.dec.Vd)
    g64 = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R), precision=CMPS_FP64)
    e64, v64, _ = g64.HED(tol=1e-12, krylov_dim=32)
    g32 = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R), precision=CMPS_SPLIT_TF32)
    e32, v32, _ = g32.HED(tol=1e-12, krylov_dim=32)
    assert abs(e32 - e64) <= 1e-9 * abs(e64), (e32, e64)
    assert abs(abs(np.vdot(v64, v32)) - 1.0) <= 1e-6


@pytest.mark.parametrize("width", [3.5, 1.2])
def test_split_matvec_at_benchmark_scale(ctx, width):
    """chi = 512 ladder workload; width 1.2 gives charge sectors above 128
    states (several N tiles per task in both stages)."""
    from chainamps_b200 import TwoVertexComponents, CMPS_SPLIT_TF32, CMPS_FP64, models
    rules, ch, W, bq = models.ladder_model(4, 1.0, 0.5)
    used_l = sorted({int(b) for b in np.nonzero(np.any(W != 0, axis=(0, 2, 3)))[0]})
    used_r = sorted({int(b) for b in np.nonzero(np.any(W != 0, axis=(0, 1, 2)))[0]})
    bond = models.gaussian_bond(512, step=2, width=width)
    rng = np.random.default_rng(5)
    L = models.random_environment(rng, rules, bond, bq, used_l, right=False)
    R = models.random_environment(rng, rules, bond, bq, used_r, right=True)
    Wt = models.mpo_tensor(ch, W, bq)
    g64 = TwoVertexComponents(ctx, rules, L, Wt, R, precision=CMPS_FP64)
    x = rng.standard_normal(g64.n) + 1j * rng.standard_normal(g64.n)
    a = g64.multiply(x)
    del g64
    g32 = TwoVertexComponents(ctx, rules, L, Wt, R, precision=CMPS_SPLIT_TF32)
    b = g32.multiply(x)
    err = np.max(np.abs(a - b)) / np.max(np.abs(a))
    assert err <= SCALE_RTOL, err
    rms = np.sqrt(np.mean(np.abs(a - b) ** 2)) / np.sqrt(np.mean(np.abs(a) ** 2))
    assert rms <= 1e-4, rms
