"""The FP64 H_eff matvec in the canonical contraction order (L . theta, W on
sigma1, W on sigma2, . R; canonical.cu) against the oracle, through the C
ABI.  It is the same operator as the reference's folded LeftPart . V .
RightPart (DMRG_routines.cpp:898-945), so every case must agree with the
dense oracle and with the device's folded order within 1e-12 (max-norm,
relative); sector structure exact.  The automatic choice takes the canonical
order for the 64-state chain vertex (dense sigma^x_i within parity classes)
and the folded order for the spin ladder."""
import numpy as np
import pytest

from oracle import dmrg as od, canonical as oc
from tests.helpers import to_tensor, model_zoo, ising_mpo
from tests.test_heff_gpu import make_envs, CHI

pytestmark = pytest.mark.gpu

ZOO = model_zoo()


@pytest.fixture(scope="module")
def ctx():
    from chainamps_b200 import Context
    c = Context(0)
    yield c
    c.close()


def _cases():
    out = {k: (ZOO[k], CHI[k]) for k in sorted(ZOO)}
    out["ising8"] = (ising_mpo(4, 8), (10, 12))
    return out


CASES = _cases()


@pytest.mark.parametrize("name", sorted(CASES))
def test_canonical_matvec_matches_oracle_and_folded(ctx, name):
    from chainamps_b200 import TwoVertexComponents, CMPS_ORDER_CANONICAL, CMPS_ORDER_FOLDED
    H, (cl, cr) = CASES[name]
    L, R = make_envs(H, 7, cl, cr)
    ref = od.TwoVertexComponents(L, H, R)
    g = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R))
    np.testing.assert_array_equal(g.allowed_indices, ref.allowed)
    rng = np.random.default_rng(3)
    xs = [rng.standard_normal(g.n) + 1j * rng.standard_normal(g.n) for _ in range(2)]
    g.set_order(CMPS_ORDER_FOLDED)
    assert g.order()[0] == CMPS_ORDER_FOLDED
    folded = [g.multiply(x) for x in xs]
    g.set_order(CMPS_ORDER_CANONICAL)
    active, f_fold, f_can = g.order()
    assert active == CMPS_ORDER_CANONICAL and f_fold > 0 and f_can > 0
    for x, f in zip(xs, folded):
        want = ref.matvec(x)
        got = g.multiply(x)
        scale = np.max(np.abs(want))
        assert np.max(np.abs(got - want)) <= 1e-12 * scale
        assert np.max(np.abs(got - f)) <= 1e-12 * scale
    # the canonical plans execute the oracle's count of the same order, plus a
    # margin: their W2 and R tasks span whole row spaces, and class rows that
    # no W1 term reaches are zeros the oracle never forms (7% on the tiny XXZ
    # window, under 1% on the others)
    can = oc.from_mpx(H, L, R)
    assert can.flops() * (1 - 1e-12) <= f_can <= 1.25 * can.flops(), (f_can, can.flops())
    assert g.flops()[1] == f_can


def test_auto_order_per_vertex(ctx):
    """The 12-site chain cut to 64 states takes the canonical order and
    matches the canonical oracle; the 4-leg ladder keeps the folded order."""
    from chainamps_b200 import TwoVertexComponents, CMPS_ORDER_CANONICAL, CMPS_ORDER_FOLDED, models
    H = ising_mpo(12, 64)
    L, R = make_envs(H, 5, 14, 12)
    g = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R))
    active, f_fold, f_can = g.order()
    assert active == CMPS_ORDER_CANONICAL and f_can <= 0.5 * f_fold, (f_fold, f_can)
    ref = oc.from_mpx(H, L, R)
    np.testing.assert_array_equal(g.allowed_indices, ref.allowed)
    rng = np.random.default_rng(9)
    x = rng.standard_normal(g.n) + 1j * rng.standard_normal(g.n)
    want = ref.matvec(x)
    assert np.max(np.abs(g.multiply(x) - want)) <= 1e-12 * np.max(np.abs(want))
    del g
    wl = models.ladder_workload(48, seed=3)
    h = TwoVertexComponents(ctx, wl["rules"], wl["L"], wl["Wt"], wl["R"])
    assert h.order()[0] == CMPS_ORDER_FOLDED


def test_canonical_ground_state(ctx):
    """HED on the canonical-order operator: energy within 1e-10 of the
    oracle's, overlap 1 within 1e-8."""
    from chainamps_b200 import TwoVertexComponents, CMPS_ORDER_CANONICAL
    H = ising_mpo(4, 8)
    Lb = od.make_dummy_left_block(H, np.zeros(1, np.int64))
    Rb = od.make_dummy_right_block(H, np.zeros(1, np.int64))
    sb = od.SuperBlock(H, tol=1e-13)
    for _ in range(3):
        sb.grow(10, 1e-16)
    L = od.make_left_block(sb.left_blocks[sb.nleft], H, sb.dec.U)
    R = od.make_right_block(sb.right_blocks[sb.nleft], H, sb.dec.Vd)
    ref = od.TwoVertexComponents(L, H, R)
    e_ref, v_ref = ref.hed(tol=1e-14)
    g = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R))
    g.set_order(CMPS_ORDER_CANONICAL)
    e, v, _ = g.HED(tol=1e-12, krylov_dim=32)
    assert abs(e - e_ref) <= 1e-10 * abs(e_ref), (e, e_ref)
    assert abs(abs(np.vdot(v_ref[ref.allowed], v)) - 1.0) <= 1e-8
    del Lb, Rb


def test_canonical_sharded_halves(ctx):
    """Two handles owning complementary output sectors reassemble the whole
    canonical-order matvec bit for bit (theta layout)."""
    import torch
    from chainamps_b200 import TwoVertexComponents, CMPS_ORDER_CANONICAL
    H = ising_mpo(4, 8)
    L, R = make_envs(H, 12, 12, 11)
    full = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R))
    full.set_order(CMPS_ORDER_CANONICAL)
    off, fl = full.sector_table()
    nsec = len(fl)
    assert nsec >= 2
    n = int(off[-1])
    x = torch.randn(2, n, dtype=torch.float64, device="cuda")
    want = torch.empty_like(x)
    full.multiply_theta_device(x.data_ptr(), want.data_ptr(), None)
    torch.cuda.synchronize()
    got = torch.zeros_like(x)
    for part in (np.arange(nsec) < nsec // 2, np.arange(nsec) >= nsec // 2):
        h = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R))
        h.set_order(CMPS_ORDER_CANONICAL)
        h.set_owned(part.astype(np.uint8))
        y = torch.full_like(x, float("nan"))
        h.multiply_theta_device(x.data_ptr(), y.data_ptr(), None)
        torch.cuda.synchronize()
        for s in np.nonzero(part)[0]:
            got[:, off[s]:off[s + 1]] = y[:, off[s]:off[s + 1]]
        del h
    assert torch.equal(got, want)


def test_split_precision_runs_the_canonical_order_in_fp32(ctx):
    """For the 64-state chain vertex the split-precision operator is the
    canonical order in FP32 (its flops are a small fraction of the folded
    order's), accurate to FP32 accumulation: within 2e-5 of the oracle
    (max-norm, relative).  The ladder keeps the folded order on tcgen05."""
    from chainamps_b200 import TwoVertexComponents, CMPS_SPLIT_TF32, models
    H = ising_mpo(12, 64)
    L, R = make_envs(H, 5, 30, 28)
    g = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R), precision=CMPS_SPLIT_TF32)
    _, f_fold, f_can = g.order()
    assert g.flops()[1] == f_can and f_can <= 0.25 * f_fold
    ref = oc.from_mpx(H, L, R)
    rng = np.random.default_rng(4)
    for _ in range(2):
        x = rng.standard_normal(g.n) + 1j * rng.standard_normal(g.n)
        want = ref.matvec(x)
        err = np.max(np.abs(g.multiply(x) - want)) / np.max(np.abs(want))
        assert err <= 2e-5, err
    del g
    wl = models.ladder_workload(48, seed=3)
    h = TwoVertexComponents(ctx, wl["rules"], wl["L"], wl["Wt"], wl["R"], precision=CMPS_SPLIT_TF32)
    _, f_fold, f_can = h.order()
    assert h.flops()[1] == f_fold


def test_mixed_ground_state_on_the_fp32_canonical_operator(ctx):
    """The mixed-precision eigensolver (FP32 canonical matvecs, FP64 Rayleigh
    quotients) reaches the FP64 solver's energy within 1e-9 on a grown
    coupled-Ising window."""
    from chainamps_b200 import TwoVertexComponents, CMPS_SPLIT_TF32, CMPS_FP64
    H = ising_mpo(4, 8)
    sb = od.SuperBlock(H, tol=1e-13)
    for _ in range(4):
        sb.grow(16, 1e-16)
    L = od.make_left_block(sb.left_blocks[sb.nleft], H, sb.dec.U)
    R = od.make_right_block(sb.right_blocks[sb.nleft], H, sb.dec.Vd)
    e = {}
    for name, prec in (("fp64", CMPS_FP64), ("mixed", CMPS_SPLIT_TF32)):
        g = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R), precision=prec)
        e[name], v, _ = g.HED(tol=1e-12, krylov_dim=32)
        del g
    assert abs(e["mixed"] - e["fp64"]) <= 1e-9 * abs(e["fp64"]), e


def test_fp32_canonical_sharded_halves(ctx):
    """Two split-precision handles owning complementary output sectors
    reassemble the whole FP32 canonical matvec bit for bit."""
    import torch
    from chainamps_b200 import TwoVertexComponents, CMPS_SPLIT_TF32
    H = ising_mpo(12, 64)
    L, R = make_envs(H, 12, 30, 28)
    full = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R), precision=CMPS_SPLIT_TF32)
    assert full.flops()[1] == full.order()[2]  # the FP32 canonical operator
    off, fl = full.sector_table()
    nsec = len(fl)
    assert nsec >= 2
    n = int(off[-1])
    x = torch.randn(2, n, dtype=torch.float64, device="cuda")
    want = torch.empty_like(x)
    full.multiply_theta_device(x.data_ptr(), want.data_ptr(), None)
    torch.cuda.synchronize()
    got = torch.zeros_like(x)
    for part in (np.arange(nsec) < nsec // 2, np.arange(nsec) >= nsec // 2):
        h = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R), precision=CMPS_SPLIT_TF32)
        h.set_owned(part.astype(np.uint8))
        y = torch.full_like(x, float("nan"))
        h.multiply_theta_device(x.data_ptr(), y.data_ptr(), None)
        torch.cuda.synchronize()
        for s in np.nonzero(part)[0]:
            got[:, off[s]:off[s + 1]] = y[:, off[s]:off[s + 1]]
        del h
    assert torch.equal(got, want)
