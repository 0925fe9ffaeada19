"""The sector-sharded matvec on the GPU, through the C ABI.

* Two handles of the same H_eff (4-leg ladder MPO, d = 16, seeded synthetic
  environments with a Gaussian sector profile at chi = 96) own the two
  halves of a balanced two-way partition of the output sectors; together
  their owned outputs equal the unsharded theta-layout matvec: bit for bit
  in FP64 and in split-TF32 (each output element is produced by the same
  tiles either way).
* A handle that owns only part of the sectors refuses the ARPACK-order
  apply and the eigensolver, and owns everything again after
  set_owned(all): its ARPACK-order apply is unchanged.
* The sharded Lanczos on one rank (no process group) finds the energy of the
  device eigensolver to 1e-10 relative on a physical (Hermitian) H_eff."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from chainamps_b200 import Context
    c = Context(0)
    yield c
    c.close()


def ladder(chi, seed=3):
    from chainamps_b200 import models
    rules, ch, W, bq = models.ladder_model(4, 1.0, 0.5)
    used_l = sorted({int(b) for b in np.nonzero(np.any(W != 0, axis=(0, 2, 3)))[0]})
    used_r = sorted({int(b) for b in np.nonzero(np.any(W != 0, axis=(0, 1, 2)))[0]})
    bond = models.gaussian_bond(chi, step=2, width=3.5)
    rng = np.random.default_rng(seed)
    L = models.random_environment(rng, rules, bond, bq, used_l, right=False)
    R = models.random_environment(rng, rules, bond, bq, used_r, right=True)
    return rules, L, models.mpo_tensor(ch, W, bq), R


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_two_shards_reassemble_the_matvec(ctx, precision):
    from chainamps_b200 import TwoVertexComponents, CMPS_FP64, CMPS_SPLIT_TF32
    from chainamps_b200.sharded import ShardLayout, torch_stream_handle
    prec = CMPS_FP64 if precision == "fp64" else CMPS_SPLIT_TF32
    rules, L, W, R = ladder(96)
    full = TwoVertexComponents(ctx, rules, L, W, R, precision=prec)
    off, fl = full.sector_table()
    assert off[0] == 0 and np.all(np.diff(off) >= 0) and fl.sum() > 0
    total = int(off[-1])
    x = torch.randn(2, total, dtype=torch.float64, device="cuda")
    want = torch.zeros_like(x)
    full.multiply_theta_device(x.data_ptr(), want.data_ptr(), torch_stream_handle())
    got = torch.full_like(x, float("nan"))
    for rank in range(2):
        lay = ShardLayout(off, fl, 2, rank)
        assert 0 < lay.owned.sum() < lay.owned.size
        h = TwoVertexComponents(ctx, rules, L, W, R, precision=prec)
        h.set_owned(lay.owned)
        y = torch.full_like(x, float("nan"))
        h.multiply_theta_device(x.data_ptr(), y.data_ptr(), torch_stream_handle())
        torch.cuda.synchronize()
        h.status()
        got[:, lay.lo:lay.hi] = y[:, lay.lo:lay.hi]
        h.close()
    assert not torch.isnan(got).any()
    assert torch.equal(got, want)


def test_partial_handle_refuses_whole_vector_entry_points(ctx):
    from chainamps_b200 import TwoVertexComponents, CmpsError
    from chainamps_b200.sharded import ShardLayout
    rules, L, W, R = ladder(48)
    h = TwoVertexComponents(ctx, rules, L, W, R)
    x = np.random.default_rng(1).standard_normal(h.n) + 0j
    before = h.multiply(x)
    off, fl = h.sector_table()
    h.set_owned(ShardLayout(off, fl, 2, 0).owned)
    with pytest.raises(CmpsError):
        h.multiply(x)
    with pytest.raises(CmpsError):
        h.HED(tol=1e-10)
    h.set_owned(np.ones(off.size - 1, bool))
    np.testing.assert_array_equal(h.multiply(x), before)


def test_sharded_lanczos_single_rank_matches_device_solver(ctx):
    """Physical environments (oracle iDMRG on the XXZ chain, 6 steps at
    chi = 24) make H_eff Hermitian, as the solver needs."""
    from chainamps_b200 import TwoVertexComponents
    from chainamps_b200.sharded import ShardedTwoVertex
    from oracle import dmrg as od
    from tests.helpers import model_zoo, to_tensor
    H = model_zoo()["xxz"]
    sb = od.SuperBlock(H)
    for _ in range(6):
        sb.grow(24, 1e-16)
    L = od.make_left_block(sb.left_blocks[sb.nleft], H, sb.dec.U)
    R = od.make_right_block(sb.right_blocks[sb.nleft], H, sb.dec.Vd)
    h = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R))
    e_dev, _, _ = h.HED(tol=1e-12, krylov_dim=32, want_vector=False)
    sh = ShardedTwoVertex(h)
    assert sh.layout.n_local == sh.layout.total
    e, x, mv, conv = sh.lowest(tol=1e-12, krylov_dim=32, max_restarts=80)
    assert conv, (e, mv)
    assert abs(e - e_dev) <= 1e-10 * abs(e_dev), (e, e_dev)
