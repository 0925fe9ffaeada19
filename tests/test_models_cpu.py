"""The product's MPO builder (reference-layout MakeGeneralHMPO, used by the
benchmark workloads) equals the oracle's restatement exactly, and the
synthetic environments obey the reference's charge rule."""
import numpy as np

from chainamps_b200 import models as pm
from oracle import model as om
from oracle.mpx import q_add, q_eq


def _dense(t):
    M = np.zeros((t.rows, t.cols), np.complex128)
    cols = np.repeat(np.arange(t.cols), np.diff(t.colptr))
    M[t.rowind, cols] = t.values
    return M


def test_xxz_mpo_matches_oracle():
    rules, ch, W, bq = pm.xxz_model(1.0, 0.7, 0.3)
    v = om.spin_half_vertex()
    H = om.make_general_hmpo(v, om.xxz_couplings(1.0, 0.7, 0.3))
    assert W.shape == H.data.shape
    np.testing.assert_array_equal(W, H.data)
    np.testing.assert_array_equal(bq, H.indices[1].charges)


def test_ladder_mpo_matches_oracle():
    rules, ch, W, bq = pm.ladder_model(4, 1.0, 0.5)
    v = om.ladder_vertex(4, 0.5)
    H = om.make_general_hmpo(v, om.ladder_couplings(4, 1.0))
    assert W.shape == (16, 110, 16, 110)  # 2 + 12 couplings x 9 charge differences
    np.testing.assert_array_equal(W, H.data)
    np.testing.assert_array_equal(bq, H.indices[1].charges)
    np.testing.assert_array_equal(ch, v.charges)
    t = pm.mpo_tensor(ch, W, bq)
    M = _dense(t)
    np.testing.assert_array_equal(M, H.matrix())


def test_synthetic_environment_charge_rule():
    rules, ch, W, bq = pm.ladder_model(4, 1.0, 0.5)
    bond = pm.gaussian_bond(64)
    assert bond.shape == (64, 1)
    rng = np.random.default_rng(0)
    L = pm.random_environment(rng, rules, bond, bq, [0, 5, 109], right=False)
    M = _dense(L)  # rows a', cols b + D a
    D = bq.shape[0]
    r, c = np.nonzero(M)
    b, a = c % D, c // D
    assert set(np.unique(b)) <= {0, 5, 109}
    assert np.all(q_eq(bond[r], q_add(bq[b], bond[a], rules)))
