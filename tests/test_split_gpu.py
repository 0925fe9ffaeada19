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


@pytest.mark.parametrize("width,seed", [(3.5, 20261203), (1.2, 5)])
def test_matvecs_at_benchmark_scale_against_the_oracle(ctx, width, seed):
    """chi = 512 ladder workload, checked against the oracle's block port at
    its own size.  (3.5, 20261203) is exactly the benchmark's workload;
    width 1.2 gives charge sectors above 128 states (several N tiles per task
    in both split stages).  FP64 within 1e-12 (max-norm, relative); split-TF32
    within SCALE_RTOL (max-norm) and 1e-4 (rms)."""
    from chainamps_b200 import TwoVertexComponents, CMPS_SPLIT_TF32, CMPS_FP64, models
    from oracle import blocks as ob
    wl = models.ladder_workload(512, seed=seed, width=width)
    chi, D = wl["bond"].shape[0], wl["bq"].shape[0]
    bh = ob.BlockHeff(wl["rules"], wl["ch"], wl["bond"], wl["bond"], wl["bq"], wl["W"],
                      ob.env_matrices(chi, D, wl["L"].colptr, wl["L"].rowind, wl["L"].values),
                      ob.env_matrices(chi, D, wl["R"].colptr, wl["R"].rowind, wl["R"].values))
    rng = np.random.default_rng(seed + 1)
    x = rng.standard_normal(bh.n) + 1j * rng.standard_normal(bh.n)
    want = bh.matvec(x)
    scale = np.max(np.abs(want))
    g64 = TwoVertexComponents(ctx, wl["rules"], wl["L"], wl["Wt"], wl["R"], precision=CMPS_FP64)
    assert g64.n == bh.n
    np.testing.assert_array_equal(g64.allowed_indices, bh.allowed)
    a = g64.multiply(x)
    del g64
    assert np.max(np.abs(a - want)) <= 1e-12 * scale
    g32 = TwoVertexComponents(ctx, wl["rules"], wl["L"], wl["Wt"], wl["R"], precision=CMPS_SPLIT_TF32)
    b = g32.multiply(x)
    del g32
    err = np.max(np.abs(b - want)) / scale
    assert err <= SCALE_RTOL, err
    rms = np.sqrt(np.mean(np.abs(b - want) ** 2)) / np.sqrt(np.mean(np.abs(want) ** 2))
    assert rms <= 1e-4, rms
