"""CPU oracle (test infrastructure only): charge-sector block form of the
H_eff matvec, for sizes the dense restatement in ``dmrg.py`` cannot hold.

Same algorithm as ``TwoVertexMPOMPSMultiply`` (DMRG_routines.cpp:898-945):
LeftPart = contract(W, L) (DMRG_routines.cpp:779), M = LeftPart . V, then
theta' = M . RightPart with RightPart = contract(W, R); here every operand is
a set of dense charge-sector blocks multiplied with numpy (BLAS), instead of
the reference's CSC SpGEMM.  Used as the CPU baseline ("port") and for GPU
parity at medium sizes; it is itself checked against ``dmrg.py``.

Inputs are the reference-layout tensors as dense ``MPX`` objects or, for
large synthetic workloads, directly as per-b dense [a', a] matrices.
"""
from __future__ import annotations

import numpy as np

from .mpx import q_add, q_sub


def _key(q):
    return tuple(int(x) for x in np.asarray(q).ravel())


class BondSectors:
    def __init__(self, charges):
        charges = np.asarray(charges, np.int64)
        self.charges = charges
        self.keys = []
        self.elems = {}
        for e, q in enumerate(charges):
            k = _key(q)
            if k not in self.elems:
                self.elems[k] = []
                self.keys.append(k)
            self.elems[k].append(e)
        self.elems = {k: np.asarray(v, np.int64) for k, v in self.elems.items()}

    def dim(self, k):
        return self.elems[k].size if k in self.elems else 0


class BlockHeff:
    """Block-sparse H_eff.  L[b] and R[b] are dense [a', a] matrices for each
    MPO index b (None if zero); W is (d, D, d, D) [s', b_l, s, b_r]."""

    def __init__(self, rules, sigma_q, bond_l, bond_r, bq, W, Lmats, Rmats):
        self.rules = tuple(rules)
        r = self.rules
        self.d = sigma_q.shape[0]
        self.sig = [_key(q) for q in sigma_q]
        self.A0 = BondSectors(bond_l)
        self.A2 = BondSectors(bond_r)
        self.bq = [_key(q) for q in bq]
        D = len(self.bq)
        add = lambda a, b: _key(q_add(np.array(a), np.array(b), r))
        sub = lambda a, b: _key(q_sub(np.array(a), np.array(b), r))
        self.add, self.sub = add, sub
        d = self.d
        # theta sector layout
        rowm = {add(self.sig[s1], k) for s1 in range(d) for k in self.A0.keys}
        colm = {sub(k, self.sig[s2]) for s2 in range(d) for k in self.A2.keys}
        self.ms = sorted(rowm & colm)
        self.rowoff, self.coloff, self.nrows, self.ncols = {}, {}, {}, {}
        for m in self.ms:
            o = 0
            for s1 in range(d):
                k = sub(m, self.sig[s1])
                if self.A0.dim(k):
                    self.rowoff[(m, s1)] = o
                    o += self.A0.dim(k)
            self.nrows[m] = o
            o = 0
            for s2 in range(d):
                k = add(m, self.sig[s2])
                if self.A2.dim(k):
                    self.coloff[(m, s2)] = o
                    o += self.A2.dim(k)
            self.ncols[m] = o
        # allowed indices (ARPACK order, DMRG_routines.cpp:808-824) and block positions
        from .dmrg import allowed_indices
        chiL, chiR = bond_l.shape[0], bond_r.shape[0]
        self.allowed, _ = allowed_indices(r, sigma_q, bond_l, sigma_q, bond_r)
        lin = self.allowed
        s1 = lin % d
        a0 = (lin // d) % chiL
        s2 = (lin // (d * chiL)) % d
        a2 = lin // (d * chiL * d)
        pos0 = np.zeros(chiL, np.int64)
        for k, el in self.A0.elems.items():
            pos0[el] = np.arange(el.size)
        pos2 = np.zeros(chiR, np.int64)
        for k, el in self.A2.elems.items():
            pos2[el] = np.arange(el.size)
        midx = {m: i for i, m in enumerate(self.ms)}
        # middle charge of each (a2, s2) pair
        mid = np.full((chiR, d), -1, np.int64)
        for j in range(chiR):
            for t in range(d):
                mid[j, t] = midx.get(sub(_key(bond_r[j]), self.sig[t]), -1)
        ro = np.full((len(self.ms), d), -1, np.int64)
        co = np.full((len(self.ms), d), -1, np.int64)
        for (m, t), o in self.rowoff.items():
            ro[midx[m], t] = o
        for (m, t), o in self.coloff.items():
            co[midx[m], t] = o
        mi = mid[a2, s2]
        rows = ro[mi, s1] + pos0[a0]
        cols = co[mi, s2] + pos2[a2]
        self._scatter = {}
        for i, m in enumerate(self.ms):
            sel = np.nonzero(mi == i)[0]
            self._scatter[m] = (sel, rows[sel], cols[sel])
        # LeftPart blocks (b1, s1', s1, sector k): sum_b0 W[s1', b0, s1, b1] L^{b0}[k', k]
        nz = np.argwhere(W != 0)
        self.LP = {}
        for sp, b0, s, b1 in nz:
            if Lmats[b0] is None:
                continue
            w = W[sp, b0, s, b1]
            for k in self.A0.keys:
                kp = add(k, self.bq[b0])
                if not self.A0.dim(kp):
                    continue
                blk = Lmats[b0][np.ix_(self.A0.elems[kp], self.A0.elems[k])]
                key = (int(b1), int(sp), int(s), k)
                self.LP[key] = self.LP.get(key, 0) + w * blk
        # RightPart blocks (b1, s2, s2', sector t): sum_b2 W[s2', b1, s2, b2] R^{b2}[t', t]^T
        self.RP = {}
        for sp, b1, s, b2 in nz:
            if Rmats[b2] is None:
                continue
            w = W[sp, b1, s, b2]
            for t in self.A2.keys:
                tp = add(t, self.bq[b2])
                if not self.A2.dim(tp):
                    continue
                blk = Rmats[b2][np.ix_(self.A2.elems[tp], self.A2.elems[t])].T
                key = (int(b1), int(s), int(sp), t)
                self.RP[key] = self.RP.get(key, 0) + w * blk
        self.b1s = sorted({k[0] for k in self.LP} & {k[0] for k in self.RP})

    @property
    def n(self):
        return self.allowed.size

    def pack(self, x):
        blocks = {m: np.zeros((self.nrows[m], self.ncols[m]), np.complex128) for m in self.ms}
        for m, (ii, rr, cc) in self._scatter.items():
            blocks[m][rr, cc] = x[ii]
        return blocks

    def unpack(self, blocks):
        out = np.zeros(self.n, np.complex128)
        for m, (ii, rr, cc) in self._scatter.items():
            out[ii] = blocks[m][rr, cc]
        return out

    def matvec_blocks(self, th):
        d = self.d
        out = {m: np.zeros((self.nrows[m], self.ncols[m]), np.complex128) for m in self.ms}
        for b1 in self.b1s:
            for m in self.ms:
                mp = self.add(m, self.bq[b1])
                if mp not in self.nrows:
                    continue
                # stage 1: T = LeftPart^{b1} . Theta_m  (rows L(m'), cols R(m))
                T = np.zeros((self.nrows[mp], self.ncols[m]), np.complex128)
                used = False
                for s1p in range(d):
                    if (mp, s1p) not in self.rowoff:
                        continue
                    r0 = self.rowoff[(mp, s1p)]
                    kp = self.sub(mp, self.sig[s1p])
                    acc = None
                    for s1 in range(d):
                        if (m, s1) not in self.rowoff:
                            continue
                        k = self.sub(m, self.sig[s1])
                        A = self.LP.get((b1, s1p, s1, k))
                        if A is None:
                            continue
                        q0 = self.rowoff[(m, s1)]
                        prod = A @ th[m][q0:q0 + self.A0.dim(k)]
                        acc = prod if acc is None else acc + prod
                    if acc is not None:
                        T[r0:r0 + self.A0.dim(kp)] = acc
                        used = True
                if not used:
                    continue
                # stage 2: theta'_m' += T . RightPart^{b1}
                for s2p in range(d):
                    if (mp, s2p) not in self.coloff:
                        continue
                    c0 = self.coloff[(mp, s2p)]
                    tp = self.add(mp, self.sig[s2p])
                    for s2 in range(d):
                        if (m, s2) not in self.coloff:
                            continue
                        t = self.add(m, self.sig[s2])
                        B = self.RP.get((b1, s2, s2p, t))
                        if B is None:
                            continue
                        q0 = self.coloff[(m, s2)]
                        out[mp][:, c0:c0 + self.A2.dim(tp)] += T[:, q0:q0 + self.A2.dim(t)] @ B
        return out

    def matvec(self, x):
        return self.unpack(self.matvec_blocks(self.pack(x)))


def from_mpx(H, L, R):
    """BlockHeff from the reference-layout dense tensors (MPO H, left block L
    with a' = 1, b = 3, a = 5, right block R with a' = 0, b = 2, a = 4)."""
    D = H.indices[1].size
    chiL = L.indices[5].size
    chiR = R.indices[4].size
    Lt = np.asarray(L.data).reshape(L.indices[1].size, D, chiL)
    Rt = np.asarray(R.data).reshape(R.indices[0].size, D, chiR)
    Lm = [Lt[:, b, :] if np.any(Lt[:, b, :]) else None for b in range(D)]
    Rm = [Rt[:, b, :] if np.any(Rt[:, b, :]) else None for b in range(D)]
    return BlockHeff(H.rules, H.indices[0].charges, L.indices[5].charges, R.indices[4].charges,
                     H.indices[1].charges, H.data, Lm, Rm)


def env_matrices(rows, D, colptr, rowind, values):
    """Per-MPO-index dense [a', a] matrices of an environment block stored
    as the reference's CSC matrix (MPX_matrix storage, first index fastest):
    a left block (MakeLeftBlock layout: rows a'_dummy, a', b_dummy; columns
    b, a_dummy, a) or a right block (MakeRightBlock layout: rows a', a'_dummy;
    columns b, b_dummy, a, a_dummy) both have `rows` = dim a' row elements
    and column b + D * a.  Slots without entries give None."""
    colptr = np.asarray(colptr, np.int64)
    ncols = colptr.size - 1
    M = np.zeros((rows, ncols), np.complex128)
    cols = np.repeat(np.arange(ncols), np.diff(colptr))
    M[np.asarray(rowind, np.int64), cols] = np.asarray(values, np.complex128)
    T = M.reshape(rows, D, ncols // D, order="F")
    return [T[:, b, :].copy() if np.any(T[:, b, :]) else None for b in range(D)]


class BlockTwoVertex:
    """``TwoVertexComponents`` (DMRG_routines.cpp:779-896) with the matvec of
    the block port: the same allowed indices, vector indices, dense small-n
    branch and HED post-processing as ``dmrg.TwoVertexComponents``, for
    vertices whose dense LeftPart the dense restatement cannot hold (a
    64-state chain vertex at chi = 32 would need 1.7 GB for it)."""

    def __init__(self, L, H, R, order="folded"):
        """order: "folded" (LeftPart / RightPart blocks, ``BlockHeff``) or
        "canonical" (L, W1, W2, R one index at a time, ``canonical.CanonicalHeff``)."""
        self.rules = H.rules
        if order == "canonical":
            from . import canonical
            self.bh = canonical.from_mpx(H, L, R)
        elif order == "folded":
            self.bh = from_mpx(H, L, R)
        else:
            raise ValueError(order)
        sig = H.indices[2]
        self.indices = [sig.with_dir(True), L.indices[5].with_dir(True), sig.with_dir(True),
                        R.indices[4].with_dir(False)]
        s1, a0, s2, a2 = self.indices
        self.vrows = s1.size * a0.size
        self.vcols = s2.size * a2.size
        self.allowed = self.bh.allowed

    @property
    def length(self):
        return self.vrows * self.vcols

    def matvec(self, x):
        return self.bh.matvec(x)

    def hed(self, guess_full=None, tol=1e-14):
        from .dmrg import SPARSE_THRESHOLD, EPS, phase_fix, lanczos_ground, eigvec_postprocess
        n = self.allowed.size
        if n <= SPARSE_THRESHOLD:
            Hd = np.zeros((n, n), np.complex128)
            for j in range(n):
                e = np.zeros(n, np.complex128)
                e[j] = 1.0
                Hd[:, j] = self.matvec(e)
            Hd = 0.5 * (Hd + Hd.conj().T)
            w, V = np.linalg.eigh(Hd)
            e = float(w[0])
            vec = V[:, 0]
            small = np.abs(vec) < EPS
            vec = phase_fix(vec)
            vec[small] = 0.0
        else:
            e, vec = lanczos_ground(self.matvec, n,
                                    None if guess_full is None else guess_full[self.allowed], tol=tol)
            vec = eigvec_postprocess(vec)
        full = np.zeros(self.length, np.complex128)
        full[self.allowed] = vec
        return e, full
