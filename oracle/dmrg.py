"""CPU oracle (test infrastructure only): the two-site DMRG hot path.

Restates, on dense numpy tensors, the reference's step logic
(andyjaj/chainamps):

* ``TwoVertexComponents`` -- LeftPart / RightPart formation and the
  charge-allowed entries of the two-site wavefunction, in ARPACK order
  (``DMRG_routines.cpp:779-833``);
* ``TwoVertexMPOMPSMultiply`` -- the H_eff matvec
  (``DMRG_routines.cpp:898-945``), computed as (LeftPart . V) . RightPart
  exactly as the reference contracts it;
* ``TwoVertexComponents::HED`` -- dense branch for n <= 1000, Krylov branch
  otherwise, then eigenvector phase fix, small-entry drop and
  ``FixComplexPrecision`` (``DMRG_routines.cpp:835-896``,
  ``sparse_interface.cpp:28-32``);
* ``MPX_matrix::SVD`` / ``SparseMatrix::SVD`` -- charge-block SVD with the
  reference's truncation rule (``MPX_matrix.cpp:157-192``,
  ``sparse_interface.cpp:1248-1406``);
* ``MakeLeftBlock`` / ``MakeRightBlock`` / ``MakeInitial*Block`` /
  ``MakeDummy*Block`` (``DMRG_routines.cpp:583-653``);
* ``MakePrediction`` / ``CheckConvergence`` (``DMRG_routines.cpp:693-776``);
* ``SuperBlock::initialise / grow_two_vertex / move_{right,left}_two_vertex``
  (``DMRG_routines.cpp:309-444``) and the sweep schedule of
  ``FiniteDMRG::run`` (``fDMRG_routines.cpp:19-66``), with environments kept
  in memory instead of ``.BLOCK`` files.

The eigensolver used for the Krylov branch is SciPy's ARPACK (``eigsh``)
with a tight tolerance, standing in for the reference's converged ARPACK run.
"""
from __future__ import annotations

import numpy as np

from .mpx import (EPS, Index, MPX, contract, reorder, remove_dummy, shift_num_rows,
                  move_dummy, from_matrix, diag_mpx, q_add, q_sub, q_eq, dummy_index)
from .model import left_open_bc, right_open_bc

SPARSE_THRESHOLD = 1000   # sparse_interface.hpp:16
DEGENERACY_REL = 1.0e-3   # sparse_interface.cpp:1373


# --------------------------------------------------------------------------
# environments
# --------------------------------------------------------------------------
def make_dummy_left_block(H: MPX, target) -> MPX:
    """MakeDummyLeftBlock (DMRG_routines.cpp:613-632)."""
    nq = H.nq
    z = np.zeros(nq, np.int64)
    D = H.indices[1].size
    idx = [dummy_index(False, z, nq), dummy_index(True, z, nq), dummy_index(True, z, nq),
           Index(False, False, H.indices[1].charges), dummy_index(True, z, nq), dummy_index(False, z, nq)]
    M = np.zeros((D, 1), np.complex128)
    M[D - 1, 0] = 1.0
    return from_matrix(H.rules, idx, 4, M)


def make_dummy_right_block(H: MPX, target) -> MPX:
    """MakeDummyRightBlock (DMRG_routines.cpp:634-653)."""
    nq = H.nq
    z = np.zeros(nq, np.int64)
    t = np.asarray(target, np.int64)
    D = H.indices[3].size
    idx = [dummy_index(False, t, nq), dummy_index(True, z, nq), Index(True, False, H.indices[3].charges),
           dummy_index(False, z, nq), dummy_index(True, t, nq), dummy_index(False, z, nq)]
    M = np.zeros((D, 1), np.complex128)
    M[0, 0] = 1.0
    return from_matrix(H.rules, idx, 3, M)


def make_initial_left_block(LeftH: MPX, A: MPX) -> MPX:
    """MakeInitialLeftBlock (DMRG_routines.cpp:583-587)."""
    return contract(A, True, contract(LeftH, False, A, False, [(2, 0)]), False, [(0, 0)])


def make_initial_right_block(RightH: MPX, B: MPX) -> MPX:
    """MakeInitialRightBlock (DMRG_routines.cpp:588-592)."""
    return contract(B, True, contract(RightH, False, B, False, [(2, 1)]), False, [(1, 0)])


def make_left_block(LB: MPX, H: MPX, A: MPX) -> MPX:
    """MakeLeftBlock (DMRG_routines.cpp:594-602): L' = A^dag (W (L A))."""
    x = contract(LB, False, A, False, [(5, 1)])
    x = contract(H, False, x, False, [(1, 3), (2, 5)])
    x = contract(A, True, x, False, [(0, 0), (1, 3)])
    return move_dummy(x, [2, 0, 3, 1, 4, 5])


def make_right_block(RB: MPX, H: MPX, B: MPX) -> MPX:
    """MakeRightBlock (DMRG_routines.cpp:603-611)."""
    x = contract(RB, False, B, False, [(4, 2)])
    x = contract(H, False, x, False, [(2, 6), (3, 2)])
    x = contract(B, True, x, False, [(1, 0), (2, 2)])
    return move_dummy(x, [0, 2, 1, 3, 5, 4])


# --------------------------------------------------------------------------
# H_eff
# --------------------------------------------------------------------------
class TwoVertexComponents:
    """TwoVertexComponents (DMRG_routines.cpp:779-833)."""

    def __init__(self, L: MPX, H: MPX, R: MPX):
        self.L, self.H, self.R = L, H, R
        self.rules = H.rules
        lp = contract(H, False, L, False, [(1, 3)])
        lp = remove_dummy(lp, [3, 5, 6])
        self.LeftPart = reorder(lp, False, [0, 3, 2, 1, 4], 3)
        rp = contract(H, False, R, False, [(3, 2)])
        rp = remove_dummy(rp, [4, 5, 7])
        self.RightPart = reorder(rp, False, [1, 2, 4, 0, 3], 3)
        sig = H.indices[2]
        self.indices = [sig.with_dir(True), L.indices[5].with_dir(True), sig.with_dir(True),
                        R.indices[4].with_dir(False)]
        s1, a0, s2, a2 = self.indices
        self.vrows = s1.size * a0.size
        self.vcols = s2.size * a2.size
        self.allowed, self.rows_and_cols = allowed_indices(self.rules, s1.charges, a0.charges,
                                                           s2.charges, a2.charges)

    @property
    def length(self):
        return self.vrows * self.vcols

    def matvec(self, x):
        """TwoVertexMPOMPSMultiply (DMRG_routines.cpp:898-945)."""
        v = np.zeros(self.vrows * self.vcols, np.complex128)
        v[self.allowed] = x
        V = from_matrix(self.rules, self.indices, 2, v.reshape((self.vrows, self.vcols), order="F"))
        M = shift_num_rows(contract(self.LeftPart, False, V, False, [(3, 0), (4, 1)]), 2)
        SM = contract(M, False, self.RightPart, False, [(2, 0), (3, 1), (4, 2)])
        return SM.matrix().reshape(-1, order="F")[self.allowed]

    def dense(self):
        n = self.allowed.size
        out = np.zeros((n, n), np.complex128)
        for j in range(n):
            e = np.zeros(n, np.complex128)
            e[j] = 1.0
            out[:, j] = self.matvec(e)
        return out

    def hed(self, guess_full=None, tol=1e-14):
        """TwoVertexComponents::HED (DMRG_routines.cpp:835-896), one eigenpair,
        smallest real part.  Returns (energy, full-length eigenvector)."""
        n = self.allowed.size
        if n <= SPARSE_THRESHOLD:
            Hd = self.dense()
            Hd = 0.5 * (Hd + Hd.conj().T)
            w, V = np.linalg.eigh(Hd)
            e = float(w[0])
            vec = V[:, 0]
            small = np.abs(vec) < EPS  # TranslateRows drop (sparse_interface.hpp:410-423)
            vec = phase_fix(vec)
            vec[small] = 0.0
        else:
            e, vec = lanczos_ground(self.matvec, n,
                                    None if guess_full is None else guess_full[self.allowed], tol=tol)
            vec = eigvec_postprocess(vec)
        full = np.zeros(self.length, np.complex128)
        full[self.allowed] = vec
        return e, full


def allowed_indices(rules, s1c, a0c, s2c, a2c):
    """The charge loop of TwoVertexComponents (DMRG_routines.cpp:808-824):
    a2 outermost, sigma1 innermost; rule sigma1 == a2 - sigma2 - a0."""
    d1, n0, d2, n2 = s1c.shape[0], a0c.shape[0], s2c.shape[0], a2c.shape[0]
    # target charge for each (a0, s2, a2) triple
    t = q_sub(q_sub(a2c[None, None, :, :], s2c[None, :, None, :], rules), a0c[:, None, None, :], rules)
    # compare with sigma1: ok[s1, a0, s2, a2]
    ok = q_eq(s1c[:, None, None, None, :], t[None, :, :, :, :])
    lin = np.nonzero(ok.reshape(-1, order="F"))[0].astype(np.int64)
    vrows = d1 * n0
    rc = np.stack([lin % vrows, lin // vrows], axis=1)
    return lin, rc


def phase_fix(vec):
    """Largest-|x| entry made real positive (DMRG_routines.cpp:873-884)."""
    k = int(np.argmax(np.abs(vec)))
    mx = vec[k]
    if abs(mx) == 0:
        return vec
    return vec * (abs(mx) / mx)


def fix_complex_precision(c):
    """FixComplexPrecision (sparse_interface.cpp:28-32), elementwise."""
    c = np.asarray(c, np.complex128).copy()
    re, im = c.real, c.imag
    with np.errstate(divide="ignore", invalid="ignore"):
        a = np.abs(im / re) < EPS
        b = np.abs(re / im) < EPS
    out = c.copy()
    out[a] = re[a]
    bb = b & ~a
    out[bb] = 1j * im[bb]
    return out


def eigvec_postprocess(vec):
    """Phase fix, drop |x| <= eps * max, FixComplexPrecision
    (DMRG_routines.cpp:870-889)."""
    vec = np.asarray(vec, np.complex128)
    mxabs = float(np.max(np.abs(vec)))
    v = phase_fix(vec)
    keep = np.abs(v) > EPS * mxabs
    out = np.zeros_like(v)
    out[keep] = fix_complex_precision(v[keep])
    return out


def lanczos_ground(mv, n, guess=None, tol=1e-14, maxit=2000, seed=1234):
    """Lowest eigenpair of a Hermitian operator: SciPy ARPACK (eigsh, SA)."""
    from scipy.sparse.linalg import LinearOperator, eigsh
    op = LinearOperator((n, n), matvec=lambda x: mv(np.asarray(x, np.complex128).ravel()), dtype=np.complex128)
    v0 = None
    if guess is not None and np.linalg.norm(guess) > 0:
        v0 = np.asarray(guess, np.complex128)
    else:
        rng = np.random.default_rng(seed)
        v0 = rng.standard_normal(n) + 0j
    ncv = min(n, 40)
    w, V = eigsh(op, k=1, which="SA", v0=v0, tol=tol, ncv=ncv, maxiter=maxit)
    return float(w[0]), V[:, 0]


# --------------------------------------------------------------------------
# SVD with truncation
# --------------------------------------------------------------------------
class Decomposition:
    def __init__(self, U, values, Vd, truncation):
        self.U = U          # LeftMatrix (row indices + new outgoing index)
        self.values = np.asarray(values, np.float64)
        self.Vd = Vd        # RightMatrix (new ingoing index + column indices)
        self.truncation = float(truncation)

    def square_rescale(self, s=1.0):
        """MPSDecomposition::SquareRescale (MPS_matrix.hpp:66-70)."""
        old = float(np.sum(self.values ** 2))
        if old <= 0.0:
            raise RuntimeError("square sum error")
        self.truncation = self.truncation / s
        self.values = self.values * np.sqrt(s / old)
        return self.values


def truncation_length(sorted_vals, D, max_trunc):
    """Kept count of SparseMatrix::SVD (sparse_interface.cpp:1346-1376)."""
    N = len(sorted_vals)
    length = D if (D > 0 and D < N) else N
    trunc_error = 0.0
    tl = N
    while trunc_error < max_trunc and tl > 0:
        trunc_error += sorted_vals[tl - 1] ** 2
        tl -= 1
    tl += 1
    if tl < length:
        length = tl
    while length < N and (sorted_vals[length - 1] - sorted_vals[length]) / sorted_vals[length - 1] < DEGENERACY_REL:
        length += 1
    return length


def block_svd(A: MPX, D=0, max_trunc=0.0):
    """MPX_matrix::SVD + SparseMatrix::SVD (MPX_matrix.cpp:157-192,
    sparse_interface.cpp:1248-1406).  Ties in the global sort are broken by
    first-seen order (the reference's std::sort leaves them unspecified)."""
    M = A.matrix()
    rows, cols = M.shape
    ucols, vcols, vals = [], [], []
    blocks_out = []
    for state, bcols in A.block_columns():
        sub = M[:, bcols]
        w = float(np.sum(np.abs(sub) ** 2))
        if w <= EPS * EPS:
            continue
        bcols = np.asarray(bcols)
        ne_c = bcols[np.any(sub != 0, axis=0)]
        sub = M[:, ne_c]
        ne_r = np.nonzero(np.any(sub != 0, axis=1))[0]
        blk = sub[ne_r, :]
        U, s, Vh = np.linalg.svd(blk, full_matrices=False)
        uthr = EPS / U.shape[0]
        vthr = EPS / Vh.shape[1]
        for k in range(s.size):
            uc = np.zeros(rows, np.complex128)
            u = U[:, k].copy()
            u[np.abs(u) <= uthr] = 0
            uc[ne_r] = u
            vc = np.zeros(cols, np.complex128)
            vv = Vh[k, :].copy()
            vv[np.abs(vv) <= vthr] = 0
            vc[ne_c] = vv
            ucols.append(uc)
            vcols.append(vc)
            vals.append(float(s[k]))
        blocks_out.append((state, ne_r, ne_c, s))
    if not vals:
        raise RuntimeError("no singular values")
    vals = np.asarray(vals)
    order = np.argsort(-vals, kind="stable")
    sv = vals[order]
    length = truncation_length(sv, D, max_trunc)
    keep = order[:length]
    discarded = float(np.sum(sv[length:] ** 2))
    Uk = np.stack([ucols[i] for i in keep], axis=1)
    Vk = np.stack([vcols[i] for i in keep], axis=0)  # rows of V^dagger
    rs = A.ingoing_row_states()
    newq = []
    for c in range(Uk.shape[1]):
        nz = np.nonzero(Uk[:, c])[0]
        if nz.size == 0:
            raise RuntimeError("Empty column! Malformed SVD")
        newq.append(rs[nz[0]])
    newq = np.asarray(newq, np.int64).reshape(len(newq), A.nq)
    li = list(A.indices[: A.nrow]) + [Index(False, False, newq)]
    ri = [Index(True, False, newq)] + list(A.indices[A.nrow:])
    Umpx = from_matrix(A.rules, li, A.nrow, Uk)
    Vmpx = from_matrix(A.rules, ri, 1, Vk)
    return Decomposition(Umpx, sv[:length], Vmpx, discarded)


def entropy(values):
    """entropy (sparse_interface.cpp:74-83)."""
    v = np.asarray(values)
    v = v[v != 0.0]
    return float(-np.sum(v * v * np.log(v * v)))


# --------------------------------------------------------------------------
# prediction and fidelity
# --------------------------------------------------------------------------
def make_prediction(dec: Decomposition, prev_lambda):
    """MakePrediction (DMRG_routines.cpp:693-707): returns (guess vector over
    the full two-vertex index space, auxiliary matrix)."""
    rules = dec.U.rules
    svals = diag_mpx(rules, dec.U.indices[2], dec.values)
    lamLB = reorder(contract(dec.U, False, svals, False, [(2, 0)]), False, [1, 0, 2], 1)
    alamR = reorder(contract(svals, False, dec.Vd, False, [(1, 0)]), False, [1, 0, 2], 2)
    rot = block_svd(alamR, 0, 0.0)
    aux = contract(diag_mpx(rules, rot.Vd.indices[0], rot.values), False, rot.Vd, False, [(1, 0)]).matrix()
    inv_prev = diag_mpx(rules, dec.Vd.indices[2], prev_lambda, inverse=True, rindex=dec.U.indices[1])
    g = contract(contract(alamR, False, inv_prev, False, [(2, 0)]), False, lamLB, False, [(2, 0)])
    return g.matrix().reshape(-1, order="F"), aux


def check_convergence(aux, prev_lambda):
    """CheckConvergence (DMRG_routines.cpp:769-771)."""
    s = np.linalg.svd(aux @ np.diag(np.asarray(prev_lambda, np.float64)), compute_uv=False)
    return 1.0 - float(np.sum(s))


def check_convergence_finite(guess, dec: Decomposition):
    """CheckConvergence(Prediction, MPSDecomposition) (DMRG_routines.cpp:773-776):
    1 - |Tr(G^dagger . U diag(s) V^dagger)|, G the prediction vector reshaped to
    rows (sigma1, a0) (column-major, ``reshape`` of sparse_interface.cpp:966-1003),
    U diag(s) V^dagger the new (rescaled) decomposition in the same layout."""
    us = contract(dec.U, False, diag_mpx(dec.U.rules, dec.U.indices[2], dec.values), False, [(2, 0)])
    M = contract(us, False, dec.Vd, False, [(2, 0)]).matrix()
    G = np.asarray(guess, np.complex128).reshape(M.shape, order="F")
    return 1.0 - abs(np.trace(G.conj().T @ M))


def make_r_finite_prediction(dec: Decomposition, B: MPX):
    """MakeRFinitePrediction (DMRG_routines.cpp:713-716)."""
    lam = diag_mpx(dec.U.rules, dec.U.indices[2], dec.values)
    x = reorder(contract(lam, False, dec.Vd, False, [(1, 0)]), False, [1, 0, 2], 2)
    return contract(x, False, B, False, [(2, 0)]).matrix().reshape(-1, order="F")


def make_l_finite_prediction(dec: Decomposition, A: MPX):
    """MakeLFinitePrediction (DMRG_routines.cpp:709-712)."""
    lam = diag_mpx(dec.U.rules, dec.U.indices[2], dec.values)
    x = contract(dec.U, False, lam, False, [(2, 0)])
    return contract(A, False, x, False, [(2, 1)]).matrix().reshape(-1, order="F")


def right_shape(B: MPX) -> MPX:
    """MPS_matrix::right_shape (MPS_matrix.cpp:126-136): (a_in, sigma, a_out), 1 row index."""
    if (not B.indices[0].physical) and B.indices[1].physical:
        return B
    return reorder(B, False, [1, 0, 2], 1)


def left_shape(A: MPX) -> MPX:
    """MPS_matrix::left_shape (MPS_matrix.cpp:113-124): (sigma, a_in, a_out), 2 row indices."""
    if A.indices[0].physical:
        return A
    return reorder(A, False, [1, 0, 2], 2)


# --------------------------------------------------------------------------
# superblock
# --------------------------------------------------------------------------
class SuperBlock:
    """SuperBlock (DMRG_routines.cpp:188-444) with in-memory environments."""

    def __init__(self, H: MPX, target=None, tol=1e-14, heff="dense"):
        """heff: "dense" solves with the dense restatement of
        TwoVertexComponents; "blocks" with the folded block port and
        "canonical" with the canonical-order block port
        (``blocks.BlockTwoVertex``, the same operator), for vertices too large
        for the dense form."""
        if heff not in ("dense", "blocks", "canonical"):
            raise ValueError(heff)
        self.heff = heff
        self.H = H
        self.rules = H.rules
        self.target = np.zeros(H.nq, np.int64) if target is None else np.asarray(target, np.int64)
        self.tol = tol
        self.size = 0
        self.nleft = 0
        self.left_blocks = {}
        self.right_blocks = {}
        self.left_mps = {}
        self.right_mps = {}
        self.dec = None
        self.prev_lambda = None
        self.guess = None
        self.aux = None
        self.last_heff = None

    @property
    def nright(self):
        return self.size - self.nleft - 2

    def initialise(self, chi=0, trunc=0.0):
        """SuperBlock::initialise (DMRG_routines.cpp:309-344)."""
        H = self.H
        self.left_blocks[0] = make_dummy_left_block(H, self.target)
        self.right_blocks[0] = make_dummy_right_block(H, self.target)
        self.LeftH = left_open_bc(H)
        self.RightH = right_open_bc(H)
        bond = H.indices[0].size if (chi < 1 and trunc <= 0.0) else chi
        e, theta = two_vertex_initial_wavefunction(self.LeftH, self.RightH, self.target)
        self.dec = block_svd(theta, bond, trunc)
        self.dec.square_rescale(1.0)
        self.size = 2
        self.nleft = 0
        self.left_mps[1] = self.dec.U
        self.right_mps[1] = self.dec.Vd
        self.left_blocks[1] = make_initial_left_block(self.LeftH, self.dec.U)
        self.right_blocks[1] = make_initial_right_block(self.RightH, self.dec.Vd)
        self.prev_lambda = np.ones(1)
        self.guess, self.aux = make_prediction(self.dec, self.prev_lambda)
        fid = check_convergence(self.aux, self.prev_lambda)
        return dict(energy=e, energy_per=e / 2.0, entropy=entropy(self.dec.values),
                    truncation=self.dec.truncation, fidelity=fid, chi=len(self.dec.values))

    def grow(self, chi=0, trunc=0.0):
        """SuperBlock::grow_two_vertex (DMRG_routines.cpp:346-374)."""
        if self.size < 2:
            return self.initialise(chi, trunc)
        if self.size > 2:
            Lb = make_left_block(self.left_blocks[self.nleft], self.H, self.dec.U)
            Rb = make_right_block(self.right_blocks[self.nleft], self.H, self.dec.Vd)
            self.left_blocks[self.nleft + 1] = Lb
            self.right_blocks[self.nleft + 1] = Rb
        self.size += 2
        self.nleft += 1
        self.prev_lambda = self.dec.values.copy()
        L = self.left_blocks[self.nleft]
        R = self.right_blocks[self.nleft]
        e, theta = self._solve(L, R, self.guess)
        self.dec = block_svd(theta, chi, trunc)
        self.dec.square_rescale(1.0)
        self.left_mps[self.nleft + 1] = self.dec.U
        self.right_mps[self.nleft + 1] = self.dec.Vd
        self.guess, self.aux = make_prediction(self.dec, self.prev_lambda)
        fid = check_convergence(self.aux, self.prev_lambda)
        return dict(energy=e, energy_per=e / self.size, entropy=entropy(self.dec.values),
                    truncation=self.dec.truncation, fidelity=fid, chi=len(self.dec.values))

    def _solve(self, L, R, guess):
        if self.heff in ("blocks", "canonical"):
            from .blocks import BlockTwoVertex
            h = BlockTwoVertex(L, self.H, R, order="folded" if self.heff == "blocks" else "canonical")
        else:
            h = TwoVertexComponents(L, self.H, R)
        self.last_heff = h
        e, full = h.hed(guess_full=guess if guess is not None and guess.size == h.length else None,
                        tol=self.tol)
        theta = from_matrix(self.rules, h.indices, 2, full.reshape((h.vrows, h.vcols), order="F"))
        return e, theta

    # finite sweeps -------------------------------------------------------
    def finish_growth(self):
        """Record the right blocks by distance from the right end."""
        # right_blocks[k]: block of the k rightmost vertices (k = nleft at growth)
        self.rblocks = dict(self.right_blocks)
        self.lblocks = dict(self.left_blocks)
        self.rmps = {k: right_shape(v) for k, v in self.right_mps.items()}
        self.lmps = {k: left_shape(v) for k, v in self.left_mps.items()}

    def move_right(self, chi=0, trunc=0.0):
        """SuperBlock::move_right_two_vertex (DMRG_routines.cpp:376-409)."""
        nl, nr = self.nleft, self.nright
        if nr < 1:
            raise RuntimeError("at right end")
        A = left_shape(self.dec.U)
        if nl < 1:
            newL = make_initial_left_block(self.LeftH, A)
        else:
            newL = make_left_block(self.lblocks[nl], self.H, A)
        self.lmps[nl + 1] = A
        self.nleft = nl + 1
        self.lblocks[self.nleft] = newL
        nr = self.nright
        self.prev_lambda = self.dec.values.copy()
        B = self.rmps[nr + 1]
        guess = make_r_finite_prediction(self.dec, B)
        L = self.lblocks[self.nleft]
        R = self.rblocks[nr]
        e, theta = self._solve(L, R, guess)
        self.dec = block_svd(theta, chi, -0.0 if nr <= 1 else trunc)
        self.dec.square_rescale(1.0)
        self.lmps[self.nleft + 1] = left_shape(self.dec.U)
        self.rmps[nr + 1] = right_shape(self.dec.Vd)
        return dict(energy=e, energy_per=e / self.size, entropy=entropy(self.dec.values),
                    truncation=self.dec.truncation, chi=len(self.dec.values),
                    fidelity=check_convergence_finite(guess, self.dec))

    def move_left(self, chi=0, trunc=0.0):
        """SuperBlock::move_left_two_vertex (DMRG_routines.cpp:411-444)."""
        nl, nr = self.nleft, self.nright
        if nl < 1:
            raise RuntimeError("at left end")
        B = right_shape(self.dec.Vd)
        if nr < 1:
            newR = make_initial_right_block(self.RightH, B)
        else:
            newR = make_right_block(self.rblocks[nr], self.H, B)
        self.rmps[nr + 1] = B
        self.nleft = nl - 1
        nr = self.nright
        self.rblocks[nr] = newR
        self.prev_lambda = self.dec.values.copy()
        A = self.lmps[self.nleft + 1]
        guess = make_l_finite_prediction(self.dec, A)
        L = self.lblocks[self.nleft]
        R = self.rblocks[nr]
        e, theta = self._solve(L, R, guess)
        self.dec = block_svd(theta, chi, -0.0 if self.nleft <= 1 else trunc)
        self.dec.square_rescale(1.0)
        self.lmps[self.nleft + 1] = left_shape(self.dec.U)
        self.rmps[nr + 1] = right_shape(self.dec.Vd)
        return dict(energy=e, energy_per=e / self.size, entropy=entropy(self.dec.values),
                    truncation=self.dec.truncation, chi=len(self.dec.values),
                    fidelity=check_convergence_finite(guess, self.dec))


def two_vertex_initial_wavefunction(LeftH: MPX, RightH: MPX, target):
    """TwoVertexInitialHamiltonian + TwoVertexInitialWavefunction
    (DMRG_routines.cpp:655-691): lowest state of the two-vertex Hamiltonian
    in the target sector."""
    H2 = reorder(contract(LeftH, False, RightH, False, [(3, 1)]), False, [0, 3, 2, 4, 1, 5], 2)
    M = H2.matrix()
    cs = H2.outgoing_col_states()
    cols = np.nonzero(q_eq(cs, np.asarray(target, np.int64)[None, :]))[0]
    sub = M[np.ix_(cols, cols)]
    sub = 0.5 * (sub + sub.conj().T)
    w, V = np.linalg.eigh(sub)
    vec = V[:, 0]
    small = np.abs(vec) < EPS
    vec = phase_fix(vec)
    vec[small] = 0
    full = np.zeros(M.shape[1], np.complex128)
    full[cols] = vec
    nq = H2.nq
    sig = LeftH.indices[0]
    t = np.asarray(target, np.int64)
    idx = [sig.with_dir(True), dummy_index(True, np.zeros(nq, np.int64), nq), sig.with_dir(True),
           dummy_index(False, t, nq)]
    d = sig.size
    theta = from_matrix(H2.rules, idx, 2, full.reshape((d, d), order="F"))
    return float(w[0]), theta


def run_idmrg(H, steps, chi, trunc=1e-16, target=None, tol=1e-14):
    sb = SuperBlock(H, target, tol=tol)
    out = []
    for _ in range(steps):
        out.append(sb.grow(chi, trunc))
    return sb, out


def run_fdmrg(H, nvertices, sweeps, chi, trunc=1e-16, target=None, tol=1e-14):
    """fDMRG_DRV growth + FiniteDMRG::run (fDMRG_routines.cpp:19-66); returns
    the rows written to the energies file."""
    sb = SuperBlock(H, target, tol=tol)
    rows = []
    for _ in range(nvertices // 2):
        rows.append(sb.grow(chi, trunc))
    sb.finish_growth()
    if sb.size == 2:
        return sb, rows
    for _ in range(sweeps):
        for _ in range(sb.nright, 0, -1):
            sb.move_right(chi, trunc)
        for _ in range(sb.nleft, 0, -1):
            r = sb.move_left(chi, trunc)
            if sb.nleft == sb.nright:
                rows.append(r)
        # for (r = right_size(); r > left_size(); --r): the condition reads the
        # left size as it grows, so the pass stops at the centre
        while sb.nright > sb.nleft:
            r = sb.move_right(chi, trunc)
            if sb.nleft == sb.nright:
                rows.append(r)
    return sb, rows
