"""Excited-state projectors in H_eff (ProjectorTensors, DMRG_routines.cpp:
947-973) through the C ABI.

* The matvec with projector tensors P_p and weights w_p differs from the
  plain one by exactly sum_p w_p (P_p . x) conj(P_p) (P . x without
  conjugation): 1e-13 of the output's scale, in FP64 and in split-TF32 (the
  term itself is added in FP64 to the same split output).
* Projecting out the ground state g of a physical H_eff (oracle iDMRG on
  the XXZ chain, 6 steps at chi = 24) with P = conj(g) and weight 50 moves
  it above the spectrum: the device eigensolver, FP64 and mixed precision,
  then finds the next level, the second-lowest eigenvalue of the oracle's
  H_eff from scipy's eigsh (1e-10 relative).
* The adjoint (dE/dlambda) ignores the projectors."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from chainamps_b200 import Context
    c = Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def physical():
    from oracle import dmrg as od
    from tests.helpers import model_zoo, to_tensor
    H = model_zoo()["xxz"]
    sb = od.SuperBlock(H)
    for _ in range(6):
        sb.grow(24, 1e-16)
    L = od.make_left_block(sb.left_blocks[sb.nleft], H, sb.dec.U)
    R = od.make_right_block(sb.right_blocks[sb.nleft], H, sb.dec.Vd)
    return H, od.TwoVertexComponents(L, H, R), (to_tensor(L), to_tensor(H), to_tensor(R))


@pytest.mark.parametrize("precision", ["fp64", "split"])
def test_projector_term_is_the_rank_one_update(ctx, physical, precision):
    from chainamps_b200 import TwoVertexComponents, CMPS_FP64, CMPS_SPLIT_TF32
    H, ref, (L, W, R) = physical
    prec = CMPS_FP64 if precision == "fp64" else CMPS_SPLIT_TF32
    h = TwoVertexComponents(ctx, H.rules, L, W, R, precision=prec)
    rng = np.random.default_rng(2)
    x = rng.standard_normal(h.n) + 1j * rng.standard_normal(h.n)
    P = rng.standard_normal((2, h.n)) + 1j * rng.standard_normal((2, h.n))
    w = np.array([2.5, 0.7])
    y0 = h.multiply(x)
    h.set_projectors(P, w)
    y1 = h.multiply(x)
    want = sum(w[p] * (P[p] @ x) * P[p].conj() for p in range(2))
    scale = max(np.max(np.abs(y0)), np.max(np.abs(want)))
    assert np.max(np.abs((y1 - y0) - want)) <= 1e-13 * scale
    h.set_projectors([], [])
    np.testing.assert_array_equal(h.multiply(x), y0)
    h.close()


def test_projected_ground_state_gives_the_next_level(ctx, physical):
    from scipy.sparse.linalg import LinearOperator, eigsh
    from chainamps_b200 import TwoVertexComponents, CMPS_FP64, CMPS_SPLIT_TF32
    H, ref, (L, W, R) = physical
    n = ref.allowed.size
    op = LinearOperator((n, n), matvec=lambda v: ref.matvec(np.asarray(v).ravel()), dtype=np.complex128)
    ev = np.sort(eigsh(op, k=2, which="SA", tol=1e-14, v0=np.ones(n))[0])
    for prec in (CMPS_FP64, CMPS_SPLIT_TF32):
        h = TwoVertexComponents(ctx, H.rules, L, W, R, precision=CMPS_FP64)
        e0, g, _ = h.HED(tol=1e-12, krylov_dim=32)
        assert abs(e0 - ev[0]) <= 1e-10 * abs(ev[0])
        h.set_projectors([g.conj()], [50.0])
        h.set_precision(prec)
        e1, _, _ = h.HED(tol=1e-12, krylov_dim=32)
        assert abs(e1 - ev[1]) <= 1e-10 * abs(ev[1]), (prec, e1, ev)
        h.close()


def test_adjoint_ignores_projectors(ctx):
    from chainamps_b200 import TwoVertexComponents, models
    rules, ch, W0, bq = models.xxz_model(1.0, 0.7, 0.0)
    dW = 0.5 * (models.xxz_model(1.0, 1.7, 0.0)[2] - models.xxz_model(1.0, -0.3, 0.0)[2])
    used_l = sorted({int(b) for b in np.nonzero(np.any(W0 != 0, axis=(0, 2, 3)))[0]})
    used_r = sorted({int(b) for b in np.nonzero(np.any(W0 != 0, axis=(0, 1, 2)))[0]})
    rng = np.random.default_rng(5)
    bond = models.gaussian_bond(20, step=2, width=3.0)
    L = models.random_environment(rng, rules, bond, bq, used_l, right=False)
    R = models.random_environment(rng, rules, bond, bq, used_r, right=True)
    h = TwoVertexComponents(ctx, rules, L, models.mpo_tensor(ch, W0, bq), R)
    x = rng.standard_normal(h.n) + 1j * rng.standard_normal(h.n)
    h.set_theta(x)
    g0 = h.adjoint(models.mpo_tensor(ch, dW, bq))
    h.set_projectors([x], [3.0])
    g1 = h.adjoint(models.mpo_tensor(ch, dW, bq))
    assert g1 == g0
