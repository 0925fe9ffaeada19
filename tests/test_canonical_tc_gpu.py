"""The split-BF16 H_eff matvec in the canonical contraction order on the
tcgen05 tensor cores (canonical_tc.cu: stages R, W2, W1, L as four
persistent split GEMMs, intermediates in BF16 planes), through the C ABI.

* Every model of the zoo (one, two and no charges; classes of 1 to 8
  states, so the padding of every contracted index is exercised) and a
  64-state chain window, with the canonical order requested: the form in use
  is the tcgen05 one and the matvec agrees with the canonical-order oracle
  (oracle/canonical.py) within 2e-4 of the largest entry.
* The benchmarked chain vertex (12 sites cut to 64 states, D = 26) takes this
  form by itself under split BF16 and agrees with the device's FP64 matvec
  within 1e-4 (the FP64 matvec is checked against the oracle elsewhere).
* The mixed-precision ground state on a grown chain's environments agrees
  with the FP64 one and the oracle's within 1e-10 relative (FP64
  refinement cycles).
* A sharded handle and split TF32 run the FP32 canonical form instead."""
import numpy as np
import pytest

from oracle import canonical as oc
from tests.helpers import to_tensor, model_zoo, ising_mpo
from tests.test_heff_gpu import make_envs, CHI

pytestmark = pytest.mark.gpu

ZOO = model_zoo()
TOL = 2e-4


@pytest.fixture(scope="module")
def ctx():
    from chainamps_b200 import Context
    c = Context(0)
    yield c
    c.close()


def _cases():
    out = {k: (ZOO[k], CHI[k]) for k in sorted(ZOO)}
    out["ising8"] = (ising_mpo(4, 8), (10, 12))
    out["ising64"] = (ising_mpo(12, 64), (14, 12))
    return out


CASES = _cases()


def _handle(ctx, H, L, R, precision):
    from chainamps_b200 import TwoVertexComponents
    return TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R), precision=precision)


@pytest.mark.parametrize("name", sorted(CASES))
def test_tc_canonical_matches_oracle(ctx, name):
    from chainamps_b200 import CMPS_SPLIT_BF16, CMPS_ORDER_CANONICAL, CMPS_FORM_CANONICAL_TC
    H, (cl, cr) = CASES[name]
    L, R = make_envs(H, 7, cl, cr)
    ref = oc.from_mpx(H, L, R)
    g = _handle(ctx, H, L, R, CMPS_SPLIT_BF16)
    g.set_order(CMPS_ORDER_CANONICAL)
    assert g.split_form() == CMPS_FORM_CANONICAL_TC
    np.testing.assert_array_equal(g.allowed_indices, ref.allowed)
    rng = np.random.default_rng(5)
    for _ in range(2):
        x = rng.standard_normal(g.n) + 1j * rng.standard_normal(g.n)
        want = ref.matvec(x)
        got = g.multiply(x)
        scale = np.max(np.abs(want))
        err = np.max(np.abs(got - want)) / scale
        assert err <= TOL, (name, err)
        # not an FP64 result passed through: the BF16 rounding shows
        assert err > 1e-12, (name, err)
    g.status()


def test_tc_canonical_is_chosen_for_the_chain_vertex(ctx):
    from chainamps_b200 import (CMPS_FP64, CMPS_SPLIT_BF16, CMPS_SPLIT_TF32, CMPS_ORDER_CANONICAL,
                                CMPS_FORM_CANONICAL_TC, CMPS_FORM_CANONICAL_FP32, CMPS_FORM_NONE)
    H = ising_mpo(12, 64)
    L, R = make_envs(H, 5, 30, 28)
    f = _handle(ctx, H, L, R, CMPS_FP64)
    assert f.order()[0] == CMPS_ORDER_CANONICAL and f.split_form() == CMPS_FORM_NONE
    b = _handle(ctx, H, L, R, CMPS_SPLIT_BF16)
    assert b.split_form() == CMPS_FORM_CANONICAL_TC
    t = _handle(ctx, H, L, R, CMPS_SPLIT_TF32)
    assert t.split_form() == CMPS_FORM_CANONICAL_FP32
    rng = np.random.default_rng(17)
    for _ in range(3):
        x = rng.standard_normal(b.n) + 1j * rng.standard_normal(b.n)
        want = f.multiply(x)
        scale = np.max(np.abs(want))
        assert np.max(np.abs(b.multiply(x) - want)) <= 1e-4 * scale
        assert np.max(np.abs(t.multiply(x) - want)) <= 1e-5 * scale
    # linear, and zero in zero out
    x = rng.standard_normal(b.n) + 1j * rng.standard_normal(b.n)
    assert np.max(np.abs(b.multiply(np.zeros_like(x)))) == 0.0
    b.status()


def test_tc_canonical_ground_state(ctx):
    """HED on a grown chain's environments (Hermitian H_eff) with the
    operator in the tcgen05 canonical form: the mixed eigensolver's energy
    within 1e-10 of the FP64 one and of the oracle's, overlap 1 within
    1e-8."""
    from oracle import dmrg as od
    from chainamps_b200 import CMPS_FP64, CMPS_SPLIT_BF16, CMPS_ORDER_CANONICAL, CMPS_FORM_CANONICAL_TC
    H = ising_mpo(4, 8)
    sb = od.SuperBlock(H, tol=1e-13)
    for _ in range(3):
        sb.grow(10, 1e-16)
    L = od.make_left_block(sb.left_blocks[sb.nleft], H, sb.dec.U)
    R = od.make_right_block(sb.right_blocks[sb.nleft], H, sb.dec.Vd)
    e_ref, _ = od.TwoVertexComponents(L, H, R).hed(tol=1e-14)
    f = _handle(ctx, H, L, R, CMPS_FP64)
    e64, v64, _ = f.HED(tol=1e-12, krylov_dim=32)
    b = _handle(ctx, H, L, R, CMPS_SPLIT_BF16)
    b.set_order(CMPS_ORDER_CANONICAL)
    assert b.split_form() == CMPS_FORM_CANONICAL_TC
    e, v, _ = b.HED(tol=1e-12, krylov_dim=32)
    assert abs(e - e64) <= 1e-10 * abs(e64), (e, e64)
    assert abs(e - e_ref) <= 1e-10 * abs(e_ref), (e, e_ref)
    assert abs(abs(np.vdot(v64, v)) - 1.0) <= 1e-8


def test_sharded_handle_keeps_the_fp32_form(ctx):
    from chainamps_b200 import CMPS_SPLIT_BF16, CMPS_ORDER_CANONICAL, CMPS_FORM_CANONICAL_FP32, CMPS_FORM_CANONICAL_TC
    H = ising_mpo(4, 8)
    L, R = make_envs(H, 12, 12, 11)
    h = _handle(ctx, H, L, R, CMPS_SPLIT_BF16)
    h.set_order(CMPS_ORDER_CANONICAL)
    assert h.split_form() == CMPS_FORM_CANONICAL_TC
    off, fl = h.sector_table()
    part = (np.arange(len(fl)) < len(fl) // 2).astype(np.uint8)
    h.set_owned(part)
    assert h.split_form() == CMPS_FORM_CANONICAL_FP32
