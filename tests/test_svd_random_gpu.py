"""GPU parity of the charge-block SVD's randomized route (sectors much larger
than the bond dimension) against the oracle's dense block SVD, through the
C ABI.  The wavefunctions have a prescribed spectrum: a random charge-
conserving theta re-weighted to singular values exp(-k / decay) in global
order, so the truncation point and the tail below it are known.

Tolerances: kept counts per sector exact; values within
1e-13 + 200 eps s_0^2 / s_j (the error class of a Gram-matrix eigenvalue,
which the randomized route's last step shares with the Gram route); the
truncated wavefunction within 1e-10 (max-norm); the discarded weight within
1e-12.  A weight cut below the cap is settled by the leading triplets and
the weight outside the range.  Where they do not settle the truncation (a
flat spectrum, or a weight cut within 1 % of a partial weight), the route
must step aside and the result must still match."""
import numpy as np
import pytest

from oracle import dmrg as od
from oracle.mpx import from_matrix
from tests.helpers import to_tensor, model_zoo, random_bond, random_left_block, random_right_block

pytestmark = pytest.mark.gpu

EPS = np.finfo(float).eps


@pytest.fixture(scope="module")
def case():
    from chainamps_b200 import Context, TwoVertexComponents
    ctx = Context(0)
    H = model_zoo()["xxz"]
    rng = np.random.default_rng(33)
    pool = [(0,), (1,), (2,)]
    bq = H.indices[1].charges
    L = random_left_block(rng, H.rules, random_bond(rng, 320, pool), bq)
    R = random_right_block(rng, H.rules, random_bond(rng, 300, pool), bq)
    ref = od.TwoVertexComponents(L, H, R)
    gpu = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R))
    x = rng.standard_normal(gpu.n) + 1j * rng.standard_normal(gpu.n)
    full = np.zeros(ref.length, complex)
    full[ref.allowed] = x / np.linalg.norm(x)
    flat = full.reshape((ref.vrows, ref.vcols), order="F")
    yield H, ref, gpu, flat
    ctx.close()


def spectrum(H, ref, flat, decay):
    """The prescribed values exp(-k / decay), normalised, one per value of `flat`."""
    d0 = od.block_svd(from_matrix(H.rules, ref.indices, 2, flat), 0, 0.0)
    s = np.exp(-np.arange(len(d0.values)) / decay)
    return d0, s / np.linalg.norm(s)


def decaying(H, ref, flat, decay):
    """The same singular vectors as `flat`, values exp(-k / decay) normalised."""
    d0, s = spectrum(H, ref, flat, decay)
    return d0.U.matrix() @ np.diag(s) @ d0.Vd.matrix()


def check(H, ref, gpu, M, chi, max_trunc):
    dref = od.block_svd(from_matrix(H.rules, ref.indices, 2, M), chi, max_trunc)
    gpu.set_theta(M.reshape(-1, order="F")[ref.allowed])
    s = gpu.SVD(chi, max_trunc)
    routes = s.routes()
    assert s.kept == len(dref.values)
    out = s.copy(ref.vrows, ref.vcols)
    s0 = dref.values[0]
    tol = 1e-13 + 200 * EPS * s0 * s0 / dref.values
    assert np.all(np.abs(out["values"] - dref.values) <= tol)
    keys, cnt = np.unique(out["charges"], axis=0, return_counts=True)
    rkeys, rcnt = np.unique(dref.U.indices[2].charges, axis=0, return_counts=True)
    np.testing.assert_array_equal(keys, rkeys)
    np.testing.assert_array_equal(cnt, rcnt)
    ucp, uri, uv = out["u"]
    U = np.zeros((ref.vrows, s.kept), complex)
    for c in range(s.kept):
        U[uri[ucp[c]:ucp[c + 1]], c] = uv[ucp[c]:ucp[c + 1]]
    vcp, vri, vv = out["vd"]
    Vd = np.zeros((s.kept, ref.vcols), complex)
    for c in range(ref.vcols):
        Vd[vri[vcp[c]:vcp[c + 1]], c] = vv[vcp[c]:vcp[c + 1]]
    rec = U @ np.diag(out["values"]) @ Vd
    rec_ref = dref.U.matrix() @ np.diag(dref.values) @ dref.Vd.matrix()
    assert np.max(np.abs(rec - rec_ref)) <= 1e-10
    assert abs(s.discarded - dref.truncation) <= 1e-12
    return routes


@pytest.mark.parametrize("decay,chi", [(10.0, 40), (10.0, 80), (30.0, 80)])
def test_randomized_route_matches_oracle(case, decay, chi):
    """One sector (about 214 x 200) is large enough for the randomized route
    at these bond dimensions; the cap decides the kept count."""
    H, ref, gpu, flat = case
    routes = check(H, ref, gpu, decaying(H, ref, flat, decay), chi, 1e-16)
    assert routes["randomized"] == 1


def test_randomized_route_steps_aside_for_a_flat_spectrum(case):
    """A random wavefunction: the weight outside any 92-column range is far
    above the cut, so the sector is redone by the Gram route."""
    H, ref, gpu, flat = case
    routes = check(H, ref, gpu, flat, 60, 1e-16)
    assert routes["randomized"] == 0


def test_randomized_route_settles_a_weight_cut(case):
    """max_trunc = 1e-3 cuts below the cap (35 values kept of at most 80):
    the rule's loop over the computed values, with the weight outside the
    range standing for the values left out, stops inside them, on partial
    weights 1.11 and 0.91 times the threshold."""
    H, ref, gpu, flat = case
    routes = check(H, ref, gpu, decaying(H, ref, flat, 10.0), 80, 1e-3)
    assert routes["randomized"] == 1


def test_randomized_route_steps_aside_near_the_weight_threshold(case):
    """A threshold 0.5 % below the partial weight of the last kept value:
    the cut is not left to the randomized route's rounding."""
    H, ref, gpu, flat = case
    _, s = spectrum(H, ref, flat, 10.0)
    tail = np.cumsum((s * s)[::-1])[::-1]  # tail[i] = sum_{j >= i} s_j^2
    assert tail[34] >= 1e-3 > tail[35]      # the previous test's cut: 35 kept
    routes = check(H, ref, gpu, decaying(H, ref, flat, 10.0), 80, tail[34] / 1.005)
    assert routes["randomized"] == 0
