"""Test helpers: reference-layout tensors for the C ABI, built from the
oracle's dense tensors, and synthetic charge-structured environments."""
import numpy as np

from oracle.mpx import MPX, Index, dummy_index, q_add, q_eq, to_csc, from_csc, from_matrix
from oracle import model as om


def to_tensor(A: MPX, drop=0.0):
    """oracle MPX -> chainamps_b200.MPXTensor (the reference's storage)."""
    from chainamps_b200.capi import MPXTensor, MPXIndexSpec
    rows, cols, cp, ri, vals = to_csc(A, drop)
    idx = [MPXIndexSpec(ix.inward, ix.physical, np.asarray(ix.charges, np.int64)) for ix in A.indices]
    return MPXTensor(idx, A.nrow, rows, cols, cp, ri, vals)


def block_to_mpx(rules, charges, csc, D, bq, right):
    """Exported device block (rows a', cols b + D*a) -> oracle 6-index MPX in
    the layout MakeLeftBlock / MakeRightBlock produce."""
    nq = len(rules)
    chi = charges.shape[0]
    cp, ri, v = csc
    z = np.zeros(nq, np.int64)
    if not right:
        idx = [dummy_index(False, z, nq), Index(True, False, charges), dummy_index(True, z, nq),
               Index(False, False, bq), dummy_index(True, z, nq), Index(False, False, charges)]
        nrow = 3
    else:
        idx = [Index(False, False, charges), dummy_index(True, z, nq), Index(True, False, bq),
               dummy_index(False, z, nq), Index(True, False, charges), dummy_index(False, z, nq)]
        nrow = 2
    M = np.zeros((chi, D * chi), np.complex128)
    for c in range(D * chi):
        for p in range(cp[c], cp[c + 1]):
            M[ri[p], c] += v[p]
    # matrix rows a', cols (b, a) -> tensor; both layouts share this matrix up to dummies
    T = M.reshape(chi, D, chi, order="F")
    if not right:
        data = T.reshape(1, chi, 1, D, 1, chi)
    else:
        data = T.reshape(chi, 1, D, 1, chi, 1)
    return MPX(tuple(rules), idx, nrow, np.ascontiguousarray(data))


def random_bond(rng, chi, charge_pool, weights=None):
    p = None if weights is None else np.asarray(weights, float) / np.sum(weights)
    pick = rng.choice(len(charge_pool), size=chi, p=p)
    return np.asarray([charge_pool[i] for i in pick], np.int64).reshape(chi, -1)


def random_left_block(rng, rules, bond, bq, hermitian_scale=1.0):
    """Random L with the charge rule q(a') = q(b) + q(a) (MakeLeftBlock layout)."""
    nq = len(rules)
    chi, D = bond.shape[0], bq.shape[0]
    z = np.zeros(nq, np.int64)
    ok = q_eq(bond[:, None, None, :], q_add(bq[None, :, None, :], bond[None, None, :, :], rules))
    vals = (rng.standard_normal((chi, D, chi)) + 1j * rng.standard_normal((chi, D, chi))) * ok
    idx = [dummy_index(False, z, nq), Index(True, False, bond), dummy_index(True, z, nq),
           Index(False, False, bq), dummy_index(True, z, nq), Index(False, False, bond)]
    return MPX(tuple(rules), idx, 3, np.ascontiguousarray(vals.reshape(1, chi, 1, D, 1, chi)))


def random_right_block(rng, rules, bond, bq):
    nq = len(rules)
    chi, D = bond.shape[0], bq.shape[0]
    z = np.zeros(nq, np.int64)
    ok = q_eq(bond[:, None, None, :], q_add(bq[None, :, None, :], bond[None, None, :, :], rules))
    vals = (rng.standard_normal((chi, D, chi)) + 1j * rng.standard_normal((chi, D, chi))) * ok
    idx = [Index(False, False, bond), dummy_index(True, z, nq), Index(True, False, bq),
           dummy_index(False, z, nq), Index(True, False, bond), dummy_index(False, z, nq)]
    return MPX(tuple(rules), idx, 2, np.ascontiguousarray(vals.reshape(chi, 1, D, 1, chi, 1)))


def tfim_chain_vertex(sites=4, g=1.2, keep=None):
    """Periodic transverse-field Ising chain H = -sum XX - g sum Z, exactly
    diagonalised, kept states labelled by Z2 parity; sigma^x_i operators in
    the eigenbasis (parity odd).  Rules (2,)."""
    sx, sy, sz = om.pauli()
    dim = 2 ** sites
    eye = np.eye(2)

    def op(o, j):
        m = np.array([[1.0]], np.complex128)
        for k in range(sites):
            m = np.kron(m, o if k == j else eye)
        return m
    H = np.zeros((dim, dim), np.complex128)
    for j in range(sites):
        H -= op(sx, j) @ op(sx, (j + 1) % sites) + g * op(sz, j)
    P = np.eye(1)
    for _ in range(sites):
        P = np.kron(P, sz)
    evals, evecs = [], []
    for par in (1, -1):
        sel = np.nonzero(np.isclose(np.diag(P).real, par))[0]
        w, v = np.linalg.eigh(H[np.ix_(sel, sel)])
        for k in range(len(w)):
            vec = np.zeros(dim, np.complex128)
            vec[sel] = v[:, k]
            i = int(np.argmax(np.abs(vec)))
            vec *= np.sign(vec[i].real) if vec[i].real != 0 else 1
            evals.append(w[k])
            evecs.append((vec, 0 if par == 1 else 1))
    order = np.argsort(evals, kind="stable")
    if keep is None:
        keep = dim
    order = order[:keep]
    V = np.stack([evecs[i][0] for i in order], axis=1)
    ch = np.asarray([[evecs[i][1]] for i in order], np.int64)
    ops = {f"X{j}": V.conj().T @ op(sx, j) @ V for j in range(sites)}
    Hd = np.diag(np.asarray(evals)[order]).astype(np.complex128)
    return om.Vertex((2,), ch, ops, Hd)


def model_zoo():
    """Small MPOs covering the charge kinds: Z (XXZ, ladder), Z2 with dense
    chain-basis operators (TFIM chains), none (Z_1), and two charges."""
    out = {}
    v = om.spin_half_vertex()
    out["xxz"] = om.make_general_hmpo(v, om.xxz_couplings(1.0, 1.0, 0.0))
    v4 = om.ladder_vertex(4, 0.5)
    out["ladder4"] = om.make_general_hmpo(v4, om.ladder_couplings(4, 1.0))
    vt = tfim_chain_vertex(4, 1.2, keep=10)
    out["tfim"] = om.make_general_hmpo(vt, [om.Coupling(f"J{j}", f"X{j}", f"X{j}", 0.05) for j in range(4)])
    v1 = om.spin_half_vertex(sz_charges=False)
    out["nocharge"] = om.make_general_hmpo(v1, om.xxz_couplings(1.0, 0.5, 0.3))
    # two charges: Sz (Z) and a Z_3 label on a 3-state vertex
    ch = np.array([[1, 0], [-1, 1], [1, 2]], np.int64)
    sx = np.zeros((3, 3), np.complex128)
    sx[0, 1] = sx[1, 0] = 1.0
    sz = np.diag([1.0, -1.0, 1.0]).astype(np.complex128)
    vq = om.Vertex((0, 3), ch, {"A": sx, "Z": sz}, np.diag([0.0, 0.1, 0.2]).astype(np.complex128))
    out["twocharge"] = om.make_general_hmpo(vq, [om.Coupling("J", "A", "A", 1.0), om.Coupling("K", "Z", "Z", 0.5)])
    return out


def charge_pool_for(H):
    """Bond charges that connect to the vertex charges."""
    rules = H.rules
    sig = H.indices[0].charges
    pool = {tuple(int(x) for x in q_add(a, b, rules)) for a in sig for b in sig}
    pool |= {tuple(int(x) for x in s) for s in sig}
    pool.add(tuple([0] * len(rules)))
    return sorted(pool)


def ising_mpo(sites=4, keep=8, g=1.2, j_perp=0.05):
    """Oracle MPO of coupled transverse-field Ising chains: each vertex a
    periodic chain of `sites` sites cut to its `keep` lowest states (Z2
    parity), J_perp sum_i X_i X_i between vertices (MakeGeneralHMPO layout)."""
    from chainamps_b200 import models
    ch, ops, Hv, _, _ = models.ising_chain_vertex(sites, g, keep)
    return om.make_general_hmpo(om.Vertex((2,), ch, ops, Hv),
                                [om.Coupling(f"J{i}", f"X{i}", f"X{i}", j_perp) for i in range(sites)])
