"""GPU parity of the effective-Hamiltonian matvec, the Krylov ground state,
the charge-block SVD and the environment updates against the oracle, all
through the C ABI.  Tolerances: FP64 results within 1e-12 relative of the
oracle (max-norm), energies within 1e-10 relative; sector structure and kept
counts exact."""
import numpy as np
import pytest

from oracle import dmrg as od
from oracle.mpx import from_matrix, contract, q_eq
from tests.helpers import (to_tensor, model_zoo, random_bond, random_left_block, random_right_block,
                           charge_pool_for, block_to_mpx)

pytestmark = pytest.mark.gpu

ZOO = model_zoo()
CHI = {"xxz": (23, 17), "ladder4": (9, 7), "tfim": (11, 13), "nocharge": (12, 9), "twocharge": (10, 8)}


@pytest.fixture(scope="module")
def ctx():
    from chainamps_b200 import Context
    c = Context(0)
    yield c
    c.close()


def make_envs(H, seed, chi_l, chi_r):
    rng = np.random.default_rng(seed)
    pool = charge_pool_for(H)
    bq = H.indices[1].charges
    bl = random_bond(rng, chi_l, pool)
    br = random_bond(rng, chi_r, pool)
    return random_left_block(rng, H.rules, bl, bq), random_right_block(rng, H.rules, br, bq)


@pytest.mark.parametrize("name", sorted(ZOO))
def test_matvec_matches_oracle(ctx, name):
    from chainamps_b200 import TwoVertexComponents
    H = ZOO[name]
    L, R = make_envs(H, 7, *CHI[name])
    ref = od.TwoVertexComponents(L, H, R)
    gpu = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R))
    assert gpu.n == ref.allowed.size
    assert gpu.full_length == ref.length
    np.testing.assert_array_equal(gpu.allowed_indices, ref.allowed)
    rng = np.random.default_rng(11)
    for _ in range(3):
        x = rng.standard_normal(gpu.n) + 1j * rng.standard_normal(gpu.n)
        want = ref.matvec(x)
        got = gpu.multiply(x)
        scale = np.max(np.abs(want))
        assert np.max(np.abs(got - want)) <= 1e-12 * scale
    can, exe = gpu.flops()
    assert can > 0 and exe > 0


def test_matvec_linear_and_empty_vector(ctx):
    from chainamps_b200 import TwoVertexComponents
    H = ZOO["xxz"]
    L, R = make_envs(H, 3, 31, 29)
    gpu = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R))
    rng = np.random.default_rng(5)
    x = rng.standard_normal(gpu.n) + 1j * rng.standard_normal(gpu.n)
    y = rng.standard_normal(gpu.n) + 1j * rng.standard_normal(gpu.n)
    a, b = 0.3 - 1.1j, 2.0 + 0.5j
    lhs = gpu.multiply(a * x + b * y)
    rhs = a * gpu.multiply(x) + b * gpu.multiply(y)
    assert np.max(np.abs(lhs - rhs)) <= 1e-12 * np.max(np.abs(rhs))
    assert np.all(gpu.multiply(np.zeros(gpu.n, complex)) == 0)


def test_charge_violation_is_rejected(ctx):
    from chainamps_b200 import TwoVertexComponents, CmpsError
    H = ZOO["xxz"]
    L, R = make_envs(H, 3, 8, 8)
    bad = L.copy()
    # put a value on a charge-forbidden entry
    m = bad.data.reshape(8, H.indices[1].size, 8)
    ok = np.abs(m) > 0
    i = np.argwhere(~ok)[0]
    m[tuple(i)] = 1.0
    with pytest.raises(CmpsError) as e:
        TwoVertexComponents(ctx, H.rules, to_tensor(bad), to_tensor(H), to_tensor(R))
    assert e.value.code == 2


def grown(H, steps, chi, target=None):
    sb = od.SuperBlock(H, target)
    for _ in range(steps):
        sb.grow(chi, 1e-16)
    return sb


@pytest.mark.parametrize("name,steps,chi", [("xxz", 6, 24), ("ladder4", 2, 16), ("tfim", 3, 20)])
def test_ground_state_svd_and_blocks(ctx, name, steps, chi):
    """Physical environments from an oracle iDMRG run; the GPU solves the
    next step and its factors/blocks are compared with the oracle's."""
    from chainamps_b200 import TwoVertexComponents
    H = ZOO[name]
    sb = grown(H, steps, chi)
    L = od.make_left_block(sb.left_blocks[sb.nleft], H, sb.dec.U)
    R = od.make_right_block(sb.right_blocks[sb.nleft], H, sb.dec.Vd)
    ref = od.TwoVertexComponents(L, H, R)
    e_ref, full_ref = ref.hed(tol=1e-14)
    gpu = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R))
    e, vec, nmv = gpu.HED(tol=1e-12, krylov_dim=32)
    assert abs(e - e_ref) <= 1e-10 * abs(e_ref)
    ov = abs(np.vdot(full_ref[ref.allowed], vec))
    assert abs(ov - 1.0) <= 1e-8
    # SVD of the oracle's wavefunction through the GPU: same kept structure
    gpu.set_theta(full_ref[ref.allowed])
    theta = from_matrix(H.rules, ref.indices, 2, full_ref.reshape((ref.vrows, ref.vcols), order="F"))
    dref = od.block_svd(theta, chi, 1e-16)
    s = gpu.SVD(chi, 1e-16)
    assert s.kept == len(dref.values)
    out = s.copy(ref.vrows, ref.vcols)
    np.testing.assert_allclose(out["values"], dref.values, rtol=1e-12, atol=1e-15)
    # kept states per charge sector: exact
    def per_sector(ch):
        keys, cnt = np.unique(ch, axis=0, return_counts=True)
        return {tuple(k): int(c) for k, c in zip(keys, cnt)}
    assert per_sector(out["charges"]) == per_sector(dref.U.indices[2].charges)
    assert abs(s.discarded - dref.truncation) <= 1e-14
    # reconstructed truncated wavefunction
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
    assert np.max(np.abs(rec - rec_ref)) <= 1e-11
    # environment updates with the GPU's own factors, checked by the oracle
    from oracle.mpx import Index, MPX
    Umpx = from_matrix(H.rules, list(theta.indices[:2]) + [Index(False, False, out["charges"])], 2, U)
    Vmpx = from_matrix(H.rules, [Index(True, False, out["charges"])] + list(theta.indices[2:]), 1, Vd)
    Lnew_ref = od.make_left_block(L, H, Umpx)
    Rnew_ref = od.make_right_block(R, H, Vmpx)
    bl = gpu.make_left_block(s)
    br = gpu.make_right_block(s)
    D = H.indices[1].size
    ch, csc = bl.to_csc()
    np.testing.assert_array_equal(ch, out["charges"])
    Lg = block_to_mpx(H.rules, ch, csc, D, H.indices[1].charges, right=False)
    ch, csc = br.to_csc()
    Rg = block_to_mpx(H.rules, ch, csc, D, H.indices[1].charges, right=True)
    sl = np.max(np.abs(Lnew_ref.data))
    assert np.max(np.abs(Lg.data.reshape(-1) - Lnew_ref.data.reshape(-1))) <= 1e-12 * sl
    sr = np.max(np.abs(Rnew_ref.data))
    assert np.max(np.abs(Rg.data.reshape(-1) - Rnew_ref.data.reshape(-1))) <= 1e-12 * sr


def test_svd_large_sectors(ctx):
    """Sectors of >= 192 rows and columns take the Gram-matrix route when
    the bond-dimension cap decides the kept count; values, per-sector kept
    counts and the truncated wavefunction must match the oracle's SVD."""
    from chainamps_b200 import TwoVertexComponents
    from tests.helpers import random_bond, random_left_block, random_right_block
    H = ZOO["xxz"]
    rng = np.random.default_rng(21)
    pool = [(0,), (1,), (2,)]
    bq = H.indices[1].charges
    L = random_left_block(rng, H.rules, random_bond(rng, 320, pool), bq)
    R = random_right_block(rng, H.rules, random_bond(rng, 300, pool), bq)
    ref = od.TwoVertexComponents(L, H, R)
    gpu = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R))
    x = rng.standard_normal(gpu.n) + 1j * rng.standard_normal(gpu.n)
    x /= np.linalg.norm(x)
    full = np.zeros(ref.length, complex)
    full[ref.allowed] = x
    theta = from_matrix(H.rules, ref.indices, 2, full.reshape((ref.vrows, ref.vcols), order="F"))
    for chi in (150, 400):
        dref = od.block_svd(theta, chi, 1e-16)
        gpu.set_theta(x)
        s = gpu.SVD(chi, 1e-16)
        assert s.kept == len(dref.values)
        out = s.copy(ref.vrows, ref.vcols)
        np.testing.assert_allclose(out["values"], dref.values, rtol=1e-10, atol=1e-14)
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
