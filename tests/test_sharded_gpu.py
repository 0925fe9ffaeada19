"""The sector-sharded matvec on the GPU, through the C ABI.

* Two handles of the same H_eff (4-leg ladder MPO, d = 16, seeded synthetic
  environments with a Gaussian sector profile at chi = 96) own the two
  halves of a balanced two-way partition of the output sectors; together
  their owned outputs equal the unsharded theta-layout matvec: bit for bit
  in FP64 and in split-TF32 (each output element is produced by the same
  tiles either way).
* The same with vector windows: each handle reads a packed window of only
  the input sectors its owned outputs read and writes only its owned slice,
  both shorter than the vector; FP64, split-TF32 and the canonical order
  (coupled Ising vertex) reassemble the unsharded matvec bit for bit.
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


def _windowed_halves(ctx, rules, L, W, R, prec, order=None):
    from chainamps_b200 import TwoVertexComponents
    from chainamps_b200.sharded import ShardLayout, torch_stream_handle
    full = TwoVertexComponents(ctx, rules, L, W, R, precision=prec)
    if order is not None:
        full.set_order(order)
    off, fl = full.sector_table()
    total = int(off[-1])
    x = torch.randn(2, total, dtype=torch.float64, device="cuda")
    want = torch.zeros_like(x)
    full.multiply_theta_device(x.data_ptr(), want.data_ptr(), torch_stream_handle())
    torch.cuda.synchronize()
    lays = [ShardLayout(off, fl, 2, r) for r in range(2)]
    hs = []
    for lay in lays:
        h = TwoVertexComponents(ctx, rules, L, W, R, precision=prec)
        if order is not None:
            h.set_order(order)
        h.set_owned(lay.owned)
        hs.append(h)
    needs = np.stack([h.input_sectors() for h in hs])
    got = torch.full_like(x, float("nan"))
    for lay, h in zip(lays, hs):
        lay.set_needs(needs)
        assert lay.out_len < total
        h.set_windows(lay.in_base, lay.in_len, lay.out_base, lay.out_len)
        idx = np.concatenate([np.arange(off[m], off[m + 1]) for m in range(off.size - 1) if lay.in_base[m] >= 0])
        xw = x[:, torch.as_tensor(idx, device="cuda")].contiguous()
        assert xw.shape[1] == lay.in_len
        y = torch.full((2, lay.out_len), float("nan"), dtype=torch.float64, device="cuda")
        h.multiply_theta_device(xw.data_ptr(), y.data_ptr(), torch_stream_handle())
        torch.cuda.synchronize()
        h.status()
        got[:, lay.lo:lay.hi] = y
        h.close()
    assert not torch.isnan(got).any()
    return got, want, lays, total


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_windowed_shards_reassemble_the_matvec(ctx, precision):
    from chainamps_b200 import CMPS_FP64, CMPS_SPLIT_TF32
    rules, L, W, R = ladder(96)
    got, want, lays, total = _windowed_halves(ctx, rules, L, W, R,
                                              CMPS_FP64 if precision == "fp64" else CMPS_SPLIT_TF32)
    assert torch.equal(got, want)
    # total-Sz sectors couple to their neighbours only: each input window
    # leaves out the far sectors
    assert all(lay.in_len < total for lay in lays)


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_windowed_shards_canonical_order(ctx, precision):
    """The coupled-Ising vertex (canonical order; in split precision the FP32
    canonical operator) with windows."""
    from chainamps_b200 import CMPS_FP64, CMPS_SPLIT_TF32
    from tests.helpers import ising_mpo, to_tensor, charge_pool_for, random_bond, random_left_block, \
        random_right_block
    H = ising_mpo(8, 16)
    rng = np.random.default_rng(4)
    pool = charge_pool_for(H)
    bq = H.indices[1].charges
    Lb = random_left_block(rng, H.rules, random_bond(rng, 20, pool), bq)
    Rb = random_right_block(rng, H.rules, random_bond(rng, 18, pool), bq)
    # (two Z2 sectors, each output reading both: the input window is the
    # whole vector, the output window half of it)
    got, want, _, _ = _windowed_halves(ctx, H.rules, to_tensor(Lb), to_tensor(H), to_tensor(Rb),
                                       CMPS_FP64 if precision == "fp64" else CMPS_SPLIT_TF32)
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
    # HED's post-processing: the largest entry real positive, as the device
    # eigensolver leaves its vector (overlap 1 within the solver tolerance)
    e2, vec, _ = h.HED(tol=1e-12, krylov_dim=32)
    xa = torch.empty(2 * h.n, dtype=torch.float64, device="cuda")
    from chainamps_b200.sharded import torch_stream_handle
    h.theta_to_arpack_device(x.contiguous().data_ptr(), xa.data_ptr(), torch_stream_handle())
    torch.cuda.synchronize()
    xv = xa.cpu().numpy()
    xv = xv[0::2] + 1j * xv[1::2]
    k = int(np.argmax(np.abs(xv)))
    assert abs(xv[k].imag) == 0.0 and xv[k].real > 0
    assert abs(abs(np.vdot(vec, xv)) - 1.0) <= 1e-8
