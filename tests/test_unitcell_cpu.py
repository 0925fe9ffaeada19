"""The oracle's iDMRG unit cell (Orthogonalise + iTwoVertexEnergy), pinned
on the CPU.

The reference has no example output for this path that a converged solver
reproduces (its one iDMRG example runs ARPACK at tol 0.1 on a built-in
vertex generator), so it is pinned by physics and by its own invariants, on
the spin-1/2 Heisenberg chain (Pauli couplings, Jxy = Jz = 1) grown to
chi = 24 (14 steps):
* the orthogonalised cell is left canonical and Lambda_0'^2 is its right
  fixed point (1e-12): the regauging is consistent;
* the energy per vertex is within 1e-3 of the exact infinite-chain value
  1 - 4 ln 2 (Bethe ansatz), the error of chi = 24;
* random complex phases on the singular vectors (u_k e^{i phi_k},
  e^{-i phi_k} v_k^dag; the SVD's gauge freedom) change neither the energy
  nor the entropy (1e-12): bra and ket sides are paired correctly;
* the energy through the transfer matrix's fixed points, without
  regauging (the device's route), equals the regauged cell's (1e-12)."""
import numpy as np
import pytest

from oracle import dmrg as od, model as om, unitcell as ou

BETHE = 1.0 - 4.0 * np.log(2.0)


@pytest.fixture(scope="module")
def grown():
    H = om.make_general_hmpo(om.spin_half_vertex(), om.xxz_couplings(1.0, 1.0, 0.0))
    sb = od.SuperBlock(H, tol=1e-12)
    for _ in range(14):
        sb.grow(24, 1e-16)
    return H, sb


def fixed_point_energy(cell, W):
    """Energy per vertex from the unregauged cell: <O> = Tr[T_O(l) r] /
    (eta Tr[l r]) with the dominant left / right fixed points l, r."""
    A0, A1 = cell["A0"], cell["A1"]
    chi = A0.shape[1]
    M = ou.cell_matrices(A0, A1)
    eta, l = ou.dominant(lambda x: ou.left_map(M, x), chi)
    _, r = ou.dominant(lambda x: ou.right_map(M, x), chi)
    eta = eta.real
    H1, row, col = ou.mpo_parts(np.asarray(W))
    I = np.eye(A0.shape[0])

    def T(O1, O2, env):
        return np.einsum("ik,jl,ijab,ac,klcd->bd", O1, O2, M.conj(), env, M)
    norm = np.trace(l @ r)
    e = np.trace(T(H1, I, l) @ r) + np.trace(T(I, H1, l) @ r)
    e += sum(np.trace(T(R, C, l) @ r) for R, C in zip(row, col))
    e2 = sum(np.trace(T(C, I, T(I, R, l)) @ r) for R, C in zip(row, col)) / eta
    return float((0.5 * (e + e2) / (eta * norm)).real)


def test_orthogonalised_cell_is_canonical_and_near_bethe(grown):
    H, sb = grown
    o = ou.orthogonalise(ou.unit_cell(sb.dec, sb.prev_lambda))
    M = ou.cell_matrices(o["A0"], o["A1"])
    lam2 = np.diag(o["lambdas"][0] ** 2)
    left = np.einsum("ijab,ijac->bc", M.conj(), M)
    np.testing.assert_allclose(left, np.eye(left.shape[0]), atol=1e-12)
    right = np.einsum("ijab,bc,ijdc->ad", M, lam2, M.conj())
    np.testing.assert_allclose(right, lam2, atol=1e-12)
    assert abs(np.sum(o["lambdas"][0] ** 2) - 1.0) <= 1e-14
    e = ou.itwo_vertex_energy(H.data, o)
    assert abs(e.imag) <= 1e-12
    assert abs(e.real - BETHE) <= 1e-3, (e, BETHE)
    assert e.real > BETHE - 1e-12            # variational: above the exact value


def test_energy_and_entropy_ignore_svd_phases(grown):
    H, sb = grown
    ref = ou.measure(sb.dec, sb.prev_lambda, H.data)
    dec = sb.dec
    k = len(dec.values)
    ph = np.exp(1j * np.random.default_rng(11).uniform(0, 2 * np.pi, k))
    U = dec.U.copy()
    U.data = U.data * ph[None, None, :]
    Vd = dec.Vd.copy()
    Vd.data = Vd.data * ph.conj()[:, None, None]
    rot = od.Decomposition(U, dec.values, Vd, dec.truncation)
    got = ou.measure(rot, sb.prev_lambda, H.data)
    assert abs(got["energy"] - ref["energy"]) <= 1e-12
    assert abs(got["entropy"] - ref["entropy"]) <= 1e-12


def test_fixed_point_route_equals_regauged_cell(grown):
    H, sb = grown
    cell = ou.unit_cell(sb.dec, sb.prev_lambda)
    e_regauged = ou.itwo_vertex_energy(H.data, ou.orthogonalise(cell)).real
    assert abs(fixed_point_energy(cell, H.data) - e_regauged) <= 1e-12
