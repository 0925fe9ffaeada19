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


def _kron_ising(sites, g):
    """Dense Kronecker-product construction of the periodic TFIM chain."""
    sx, sy, sz = pm.pauli()
    eye = np.eye(2)

    def op(o, j):
        m = np.array([[1.0]], np.complex128)
        for k in range(sites):
            m = np.kron(m, o if k == j else eye)
        return m
    H = np.zeros((2 ** sites, 2 ** sites), np.complex128)
    for j in range(sites):
        H -= op(sx, j) @ op(sx, (j + 1) % sites) + g * op(sz, j)
    return H, [op(sx, j) for j in range(sites)]


def test_ising_chain_vertex_against_dense_construction():
    """Kept spectrum, parity labels and the coupled two-chain spectrum agree
    with a dense Kronecker construction (basis-independent checks)."""
    sites, g, keep, jp = 5, 1.2, 12, 0.3
    ch, ops, H, dH, gap = pm.ising_chain_vertex(sites, g, keep)
    Hd, xs = _kron_ising(sites, g)
    w = np.linalg.eigvalsh(Hd)
    np.testing.assert_allclose(np.sort(np.diag(H).real), w[:keep], atol=1e-12)
    assert np.allclose(H, np.diag(np.diag(H)))
    assert gap == w[keep] - w[keep - 1] or abs(gap - (w[keep] - w[keep - 1])) < 1e-12
    for o in ops.values():                     # sigma^x flips the Z2 parity
        for p in (0, 1):
            sel = ch[:, 0] == p
            assert np.allclose(o[np.ix_(sel, sel)], 0)
    # two chains coupled by jp sum_i X_i X_i, restricted to the kept states:
    # same spectrum as projecting the dense operators onto the dense kept space
    wv, V = np.linalg.eigh(Hd)
    P = V[:, :keep]
    Xk = [P.conj().T @ x @ P for x in xs]
    E = np.diag(wv[:keep])
    I = np.eye(keep)
    ref = np.kron(E, I) + np.kron(I, E) + jp * sum(np.kron(x, x) for x in Xk)
    mine = np.kron(H, I) + np.kron(I, H) + jp * sum(np.kron(ops[f"X{j}"], ops[f"X{j}"]) for j in range(sites))
    np.testing.assert_allclose(np.linalg.eigvalsh(mine), np.linalg.eigvalsh(ref), atol=1e-10)
    # the field derivative in the fixed basis
    ch2, ops2, H2, dH2, _ = pm.ising_chain_vertex(sites, g + 0.5, keep, g_basis=g)
    np.testing.assert_allclose(H2, H + 0.5 * dH, atol=1e-12)


def test_coupled_ising_mpo_matches_oracle():
    """Product MPO builder on the coupled-chain vertex equals the oracle's
    MakeGeneralHMPO fed with the same vertex (D = 2 + 12 couplings x 2 = 26
    for 12-site chains)."""
    rules, ch, W, bq = pm.coupled_ising_model(4, 1.2, 8, 0.05)
    ch_, ops, H, _, _ = pm.ising_chain_vertex(4, 1.2, 8)
    v = om.Vertex((2,), ch, ops, H)
    Ho = om.make_general_hmpo(v, [om.Coupling(f"J{i}", f"X{i}", f"X{i}", 0.05) for i in range(4)])
    np.testing.assert_array_equal(W, Ho.data)
    np.testing.assert_array_equal(bq, Ho.indices[1].charges)
    assert pm.coupled_ising_model(12, 1.2, 64, 0.05)[2].shape == (64, 26, 64, 26)


def test_benchmark_workload_through_the_oracle_block_port():
    """The benchmark's synthetic ladder workload, read by the oracle's block
    port from the CSC storage (``env_matrices``, as the CPU baseline and the
    GPU parity test at chi = 512 read it), gives the dense oracle's matvec
    (``TwoVertexComponents`` on the same tensors) at a size the dense
    restatement holds."""
    from oracle import blocks as ob, dmrg as od
    from oracle.mpx import from_csc, Index

    wl = pm.ladder_workload(24, seed=11, width=1.5)
    D = wl["bq"].shape[0]
    chi = wl["bond"].shape[0]
    bh = ob.BlockHeff(wl["rules"], wl["ch"], wl["bond"], wl["bond"], wl["bq"], wl["W"],
                      ob.env_matrices(chi, D, wl["L"].colptr, wl["L"].rowind, wl["L"].values),
                      ob.env_matrices(chi, D, wl["R"].colptr, wl["R"].rowind, wl["R"].values))

    def mpx(t):
        idx = [Index(i.inward, i.physical, np.asarray(i.charges, np.int64)) for i in t.indices]
        return from_csc(wl["rules"], idx, t.nrow, t.rows, t.cols, t.colptr, t.rowind, t.values)
    ref = od.TwoVertexComponents(mpx(wl["L"]), mpx(wl["Wt"]), mpx(wl["R"]))
    np.testing.assert_array_equal(bh.allowed, ref.allowed)
    x = np.random.default_rng(2).standard_normal(bh.n) + 1j * np.random.default_rng(3).standard_normal(bh.n)
    a, b = bh.matvec(x), ref.matvec(x)
    assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b))


def test_ising_workload_charge_rule():
    """The synthetic coupled-Ising workload (the bench's ``ising_matvec``):
    a Z2 bond of two equal sectors, and environment entries only where the
    reference's charge rule allows them, on the MPO slots the MPO uses."""
    wl = pm.ising_workload(12)
    bond, bq = wl["bond"], wl["bq"]
    assert bond.shape == (12, 1) and np.sum(bond == 0) == 6 and np.sum(bond == 1) == 6
    assert wl["W"].shape == (64, 26, 64, 26)
    D = bq.shape[0]
    used_l = set(np.nonzero(np.any(wl["W"] != 0, axis=(0, 2, 3)))[0])
    M = _dense(wl["L"])  # rows a', cols b + D a
    r, c = np.nonzero(M)
    b, a = c % D, c // D
    assert r.size > 0 and set(np.unique(b)) <= used_l
    assert np.all(q_eq(bond[r], q_add(bq[b], bond[a], wl["rules"])))
