"""GPU parity of the split-BF16 form (3-term BF16 on tcgen05: hi.hi +
hi.mid + mid.hi per real product, FP32 accumulation) against the oracle,
through the C ABI.

Each operand keeps 16 significant bits (hi + mid, relative error <= 2^-16)
and the mid.mid product is dropped, so a product carries about 1e-5 relative
error where split-TF32 carries 2e-7; FP32 accumulation adds the same as in
the TF32 form.  Tolerances, stated: the matvec agrees with the FP64 oracle to
2e-4 relative (max-norm over the output, relative to its largest entry) at
unit-test sizes, and at the chi = 512 benchmark size to 1e-3 max-norm and
3e-4 rms.  Ground-state energies of the mixed solver (FP64 Rayleigh
quotients, FP64 refinement cycles) agree with the FP64 solver to 1e-9
relative, the accuracy the mixed-precision form is held to; so do the
energies of a mixed-precision iDMRG run.  Windowed shards reassemble the
unsharded split-BF16 matvec bit for bit."""
import numpy as np
import pytest

from oracle import dmrg as od
from tests.helpers import to_tensor, model_zoo
from tests.test_heff_gpu import make_envs, CHI, grown

pytestmark = pytest.mark.gpu

ZOO = model_zoo()
BF16_RTOL = 2e-4


@pytest.fixture(scope="module")
def ctx():
    from chainamps_b200 import Context
    c = Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("name", sorted(ZOO))
def test_bf16_matvec_matches_oracle(ctx, name):
    from chainamps_b200 import TwoVertexComponents, CMPS_SPLIT_BF16
    H = ZOO[name]
    L, R = make_envs(H, 7, *CHI[name])
    ref = od.TwoVertexComponents(L, H, R)
    gpu = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R), precision=CMPS_SPLIT_BF16)
    rng = np.random.default_rng(11)
    for _ in range(2):
        x = rng.standard_normal(gpu.n) + 1j * rng.standard_normal(gpu.n)
        want = ref.matvec(x)
        got = gpu.multiply(x)
        err = np.max(np.abs(got - want)) / np.max(np.abs(want))
        assert err <= BF16_RTOL, err


def test_bf16_matvec_larger_sectors(ctx):
    """Sectors wider than one 128-row tile and K longer than one stage ring."""
    from chainamps_b200 import TwoVertexComponents, CMPS_SPLIT_BF16, CMPS_FP64
    from tests.helpers import random_bond, random_left_block, random_right_block
    H = ZOO["xxz"]
    rng = np.random.default_rng(12)
    pool = [(0,), (1,), (2,)]
    bq = H.indices[1].charges
    L = random_left_block(rng, H.rules, random_bond(rng, 300, pool), bq)
    R = random_right_block(rng, H.rules, random_bond(rng, 260, pool), bq)
    g64 = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R), precision=CMPS_FP64)
    g16 = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R), precision=CMPS_SPLIT_BF16)
    rng = np.random.default_rng(2)
    x = rng.standard_normal(g64.n) + 1j * rng.standard_normal(g64.n)
    a, b = g64.multiply(x), g16.multiply(x)
    assert np.max(np.abs(a - b)) / np.max(np.abs(a)) <= BF16_RTOL


@pytest.mark.parametrize("name,steps,chi", [("xxz", 6, 24), ("tfim", 3, 20), ("ladder4", 2, 16)])
def test_bf16_ground_state_energy(ctx, name, steps, chi):
    from chainamps_b200 import TwoVertexComponents, CMPS_SPLIT_BF16, CMPS_FP64
    H = ZOO[name]
    sb = grown(H, steps, chi)
    L = od.make_left_block(sb.left_blocks[sb.nleft], H, sb.dec.U)
    R = od.make_right_block(sb.right_blocks[sb.nleft], H, sb.dec.Vd)
    g64 = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R), precision=CMPS_FP64)
    e64, v64, _ = g64.HED(tol=1e-12, krylov_dim=32)
    g16 = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R), precision=CMPS_SPLIT_BF16)
    e16, v16, _ = g16.HED(tol=1e-12, krylov_dim=32)
    assert abs(e16 - e64) <= 1e-9 * abs(e64), (e16, e64)
    assert abs(abs(np.vdot(v64, v16)) - 1.0) <= 1e-6


def test_bf16_idmrg_energies(ctx):
    """Mixed-precision iDMRG (split-BF16 matvecs) on the XXZ chain, 10 steps
    at chi = 32: every energy within 1e-9 relative of the FP64 run."""
    from chainamps_b200 import iDMRG, CMPS_FP64, CMPS_SPLIT_BF16
    H = ZOO["xxz"]
    e = {}
    for prec in (CMPS_FP64, CMPS_SPLIT_BF16):
        run = iDMRG(ctx, H.rules, to_tensor(H), precision=prec, tol=1e-12, krylov_dim=32)
        e[prec] = np.array([run.grow(32, 1e-16)["energy"] for _ in range(10)])
        run.close()
    rel = np.abs(e[CMPS_SPLIT_BF16] - e[CMPS_FP64]) / np.abs(e[CMPS_FP64])
    assert rel.max() <= 1e-9, rel


def test_bf16_matvec_at_benchmark_scale_against_the_oracle(ctx):
    """The chi = 512 benchmark workload against the oracle's block port at
    its own size: split-BF16 within 1e-3 (max-norm) and 3e-4 (rms)."""
    from chainamps_b200 import TwoVertexComponents, CMPS_SPLIT_BF16, models
    from oracle import blocks as ob
    wl = models.ladder_workload(512, seed=20261203, width=3.5)
    chi, D = wl["bond"].shape[0], wl["bq"].shape[0]
    bh = ob.BlockHeff(wl["rules"], wl["ch"], wl["bond"], wl["bond"], wl["bq"], wl["W"],
                      ob.env_matrices(chi, D, wl["L"].colptr, wl["L"].rowind, wl["L"].values),
                      ob.env_matrices(chi, D, wl["R"].colptr, wl["R"].rowind, wl["R"].values))
    rng = np.random.default_rng(20261204)
    x = rng.standard_normal(bh.n) + 1j * rng.standard_normal(bh.n)
    want = bh.matvec(x)
    g16 = TwoVertexComponents(ctx, wl["rules"], wl["L"], wl["Wt"], wl["R"], precision=CMPS_SPLIT_BF16)
    b = g16.multiply(x)
    del g16
    err = np.max(np.abs(b - want)) / np.max(np.abs(want))
    rms = np.sqrt(np.mean(np.abs(b - want) ** 2)) / np.sqrt(np.mean(np.abs(want) ** 2))
    print(f"split-BF16 at chi=512: max-norm {err:.3g}, rms {rms:.3g}")
    assert err <= 1e-3, err
    assert rms <= 3e-4, rms


def test_bf16_windowed_shards(ctx):
    from chainamps_b200 import CMPS_SPLIT_BF16
    from tests.test_sharded_gpu import ladder, _windowed_halves
    import torch
    rules, L, W, R = ladder(96)
    got, want, _, _ = _windowed_halves(ctx, rules, L, W, R, CMPS_SPLIT_BF16)
    assert torch.equal(got, want)
