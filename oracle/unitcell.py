"""CPU restatement of the iDMRG unit cell, its orthogonalisation and the
energy per vertex.  Test infrastructure (the oracle): only tests use it.

Dense numpy on the small bonds of the tests, following the reference's steps:

* unit_cell(dec, prev_lambda) -- UnitCell(MPSDecomposition, PreviousLambda)
  (UnitCell.hpp:42-47): A0[s1] = U[s1], A1[s2] = diag(s) V^dagger[s2]
  diag(1/lambda_prev); Lambdas = [lambda_prev, s].  The cell's right bond a2
  is the left bond a0 of the next cell, element by element.
* orthogonalise(cell) -- Orthogonalise(UnitCell) (measurement.cpp:180-246):
  the dominant left and right eigenvectors of the cell's transfer matrix
  (TransferMatrixComponents::LeftED / RightED, measurement.cpp:456-575,
  LeftComponentsMultiply / RightComponentsMultiply :582-625), made Hermitian;
  SqrtDR of each (MPX_matrix.cpp:829-911: eigenvalues with |w| <= 100 eps
  max|w| dropped, mixed signs a failure); the SVD of X Y, rescaled to unit
  square sum, gives the new boundary values; the cell is regauged as
  A0' = U'^dag X A0 / sqrt(eta_L), A1' = A1 X^-1 U'.
* itwo_vertex_energy(W, ortho) -- iTwoVertexEnergy(ColX, RowX, H1, UnitCell)
  (measurement.cpp:371-397) with H1 = W[D-1, 0], ColX = W[1..D-2, 0],
  RowX = W[D-1, 1..D-2] (:371-376): half the sum of the on-vertex terms of
  both sites, the bond inside the cell (TwoVertexMeasurement, :317-322) and
  the bond to the next cell, each a trace against Lambda_0'^2.

Conventions.  The left map is L(l) = sum_s M_s^dag l M_s with l[bra, ket];
the right map R(r) = sum_s M_s r M_s^dag with r[ket, bra] (M_s = A0[s1]
A1[s2]).  The eigenvector phase that ARPACK leaves free is fixed so that
the trace is real and positive before the Hermitian part is taken (the
reference adds the vector to its conjugate transpose as returned).
"""
import numpy as np

EPS = np.finfo(float).eps


def unit_cell(dec, prev_lambda):
    """Dense cell tensors A0 (d, chi0, chi1), A1 (d, chi1, chi0) and the
    values [lambda_prev, s] from a growth step's decomposition."""
    U = np.asarray(dec.U.data)          # (d, chi0, k) [s1, a0, a1]
    Vd = np.asarray(dec.Vd.data)        # (k, d, chi2) [a1, s2, a2]
    s = np.asarray(dec.values, float)
    lp = np.asarray(prev_lambda, float)
    if U.shape[1] != Vd.shape[2] or U.shape[1] != lp.size:
        raise ValueError("the cell's end bonds differ: no unit cell")
    A0 = np.ascontiguousarray(U)
    inv = np.where(lp != 0.0, 1.0 / np.where(lp != 0.0, lp, 1.0), 0.0)
    A1 = np.ascontiguousarray(np.transpose(s[:, None, None] * Vd * inv[None, None, :], (1, 0, 2)))
    return dict(A0=A0, A1=A1, lambdas=[lp.copy(), s.copy()])


def cell_matrices(A0, A1):
    """M[s1, s2] = A0[s1] A1[s2]: (d, d, chi, chi)."""
    return np.einsum("iab,jbc->ijac", A0, A1)


def left_map(M, l):
    return np.einsum("ijab,ac,ijcd->bd", M.conj(), l, M)


def right_map(M, r):
    return np.einsum("ijab,bd,ijcd->ac", M, r, M.conj())


def dominant(apply, chi):
    """Largest-magnitude eigenpair of a map on chi x chi matrices: the dense
    transfer matrix for chi^2 <= 1000 (the reference's SPARSE_THRESHOLD,
    sparse_interface.hpp:16), ARPACK (scipy) "LM" on the map above it."""
    n = chi * chi
    if n <= 1000:
        T = np.zeros((n, n), np.complex128)
        for k in range(n):
            e = np.zeros(n, np.complex128)
            e[k] = 1.0
            T[:, k] = apply(e.reshape(chi, chi)).reshape(n)
        w, v = np.linalg.eig(T)
        i = int(np.argmax(np.abs(w)))
        ev, vec = w[i], v[:, i]
    else:
        from scipy.sparse.linalg import LinearOperator, eigs
        op = LinearOperator((n, n), matvec=lambda x: apply(np.asarray(x).reshape(chi, chi)).reshape(n),
                            dtype=np.complex128)
        w, v = eigs(op, k=1, which="LM", tol=1e-14, v0=np.ones(n, np.complex128))
        ev, vec = w[0], v[:, 0]
    V = vec.reshape(chi, chi)
    tr = np.trace(V)
    V = V * (np.conj(tr) / abs(tr))
    return ev, 0.5 * (V + V.conj().T)


def sqrt_dr(M):
    """SqrtDR: M = R^dag D R; returns (sqrt|D| kept, R kept) or None."""
    w, E = np.linalg.eigh(M)
    tol = np.max(np.abs(w)) * 100.0 * EPS
    keep = np.abs(w) > tol
    neg = int(np.sum(w[keep] < 0.0))
    if neg != 0 and neg != int(np.sum(keep)):
        return None
    return np.sqrt(np.abs(w[keep])), E[:, keep].conj().T


def orthogonalise(cell):
    A0, A1 = cell["A0"], cell["A1"]
    chi = A0.shape[1]
    M = cell_matrices(A0, A1)
    eta_l, l = dominant(lambda x: left_map(M, x), chi)
    eta_r, r = dominant(lambda x: right_map(M, x), chi)
    for eta in (eta_l, eta_r):   # IMAGTOL = 100 eps (measurement.cpp:12,187,212), with room for the solver
        if abs(eta.imag) >= 1e-10 * abs(eta.real):
            raise RuntimeError("dominant eigenvalue has a non-negligible imaginary part")
    dl = sqrt_dr(l)
    dr = sqrt_dr(r)
    if dl is None or dr is None:
        raise RuntimeError("SqrtDR failure")
    rl, Rl = dl
    rr, Rr = dr
    X = rl[:, None] * Rl                       # l = X^dag X  (X: k_L x ket)
    Xinv = Rl.conj().T / rl[None, :]           # X Xinv = 1
    Y = Rr.conj().T * rr[None, :]              # r = Y Y^dag  (Y: ket x k_R)
    Up, lam, Wh = np.linalg.svd(X @ Y, full_matrices=False)
    lam = lam / np.sqrt(np.sum(lam ** 2))
    A0n = np.einsum("kn,ka,sab->snb", Up.conj(), X, A0) / np.sqrt(eta_l.real)
    A1n = np.einsum("sab,bk,kn->san", A1, Xinv, Up)
    return dict(A0=A0n, A1=A1n, lambdas=[lam, cell["lambdas"][1]], eta_left=eta_l, eta_right=eta_r,
                X=X, Y=Y)


def mpo_parts(W):
    """H1, RowX[k], ColX[k] (k = 1..D-2) from W (d, D, d, D) [s', bl, s, br]."""
    D = W.shape[1]
    H1 = W[:, D - 1, :, 0]
    row = [W[:, D - 1, :, k] for k in range(1, D - 1)]
    col = [W[:, k, :, 0] for k in range(1, D - 1)]
    return H1, row, col


def itwo_vertex_energy(W, ortho):
    """Energy per vertex of the orthogonalised cell (left canonical, right
    boundary Lambda_0'^2)."""
    A0, A1 = ortho["A0"], ortho["A1"]
    lam2 = np.diag(ortho["lambdas"][0] ** 2)
    H1, row, col = mpo_parts(np.asarray(W))
    M = cell_matrices(A0, A1)                        # (s1, s2, a, b)
    d = A0.shape[0]
    I = np.eye(d)

    def cell_op(O1, O2):
        # sum O1[s1',s1] O2[s2',s2] M[s1',s2']^dag M[s1,s2] -> (b', b), left index traced
        return np.einsum("ik,jl,ijab,klac->bc", O1, O2, M.conj(), M)

    local = np.trace(cell_op(H1, I) @ lam2) + np.trace(cell_op(I, H1) @ lam2)
    bond1 = sum(np.trace(cell_op(R, C) @ lam2) for R, C in zip(row, col))
    bond2 = 0.0
    for R, C in zip(row, col):
        E1 = cell_op(I, R)                            # first cell: RowX on site 1
        # second cell: ColX on site 0, environment E1 on its left
        E2 = np.einsum("ik,ijab,ac,kjcd->bd", C, M.conj(), E1, M)
        bond2 = bond2 + np.trace(E2 @ lam2)
    return complex(0.5 * (local + bond1 + bond2))


def entropy(values):
    v = np.asarray(values)
    v = v[v != 0.0]
    return float(-np.sum(v * v * np.log(v * v)))


def measure(dec, prev_lambda, W):
    """Orthogonalise + iTwoVertexEnergy of one growth step (iDMRG_DRV.cpp:71-77)."""
    o = orthogonalise(unit_cell(dec, prev_lambda))
    return dict(energy=itwo_vertex_energy(W, o).real, entropy=entropy(o["lambdas"][0]),
                chi=int(np.sum(o["lambdas"][0] > 0.0)), ortho=o)
