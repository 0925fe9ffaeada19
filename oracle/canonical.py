"""CPU oracle (test infrastructure only): the two-site H_eff matvec in the
canonical four-stage contraction order.

The reference applies H_eff as LeftPart . V . RightPart
(``TwoVertexMPOMPSMultiply``, DMRG_routines.cpp:898-945), where LeftPart
and RightPart fold the MPO W into the environments (``TwoVertexComponents``,
DMRG_routines.cpp:779-806).  The same linear map, contracted one index at a
time, is

    X^{b0}  = L^{b0} . theta                      (contract a0)
    Y^{b1}  = sum_{b0, s1} W[s1', b0, s1, b1] X^{b0}   (contract sigma1)
    Z^{b2}  = sum_{b1, s2} W[s2', b1, s2, b2] Y^{b1}   (contract sigma2)
    theta'  = sum_{b2} Z^{b2} . R^{b2}^T            (contract a2)

with L^{b0}[a0', a0] (a0' in sector q(a0) + q(b0)) and R^{b2}[a2', a2]
(a2' in sector q(a2) + q(b2)), exactly the blocks the reference's
environments hold (``MakeLeftBlock`` / ``MakeRightBlock`` layouts).  For a
vertex with a large local basis whose operators are dense within charge
classes (a chain cut to 64 states) this order costs a small fraction of the
folded one; it is the order the survey of the path prescribes for the GPU.

Every operand is a set of dense blocks keyed by (class of sigma1, sector of
a0, class of sigma2, sector of a2); a class is the set of physical states
with one charge.  The allowed indices and ARPACK order are those of
``dmrg.allowed_indices`` (DMRG_routines.cpp:808-824).  Checked against the
dense restatement ``dmrg.TwoVertexComponents`` in tests.
"""
from __future__ import annotations

import numpy as np

from .mpx import q_add, q_sub


def _key(q):
    return tuple(int(x) for x in np.asarray(q).ravel())


def _groups(charges):
    """charge key -> element indices (ascending), keys in first-seen order."""
    out = {}
    for e, q in enumerate(np.asarray(charges, np.int64)):
        out.setdefault(_key(q), []).append(e)
    return {k: np.asarray(v, np.int64) for k, v in out.items()}


class CanonicalHeff:
    """H_eff of one two-vertex window in the canonical contraction order.
    W is (d, D, d, D) [s', b_l, s, b_r]; Lmats[b] / Rmats[b] are dense
    [a', a] matrices (None for an empty slot)."""

    def __init__(self, rules, sigma_q, bond_l, bond_r, bq, W, Lmats, Rmats):
        from .dmrg import allowed_indices
        self.rules = tuple(rules)
        r = self.rules
        self.add = lambda a, b: _key(q_add(np.array(a), np.array(b), r))
        self.sub = lambda a, b: _key(q_sub(np.array(a), np.array(b), r))
        sigma_q = np.asarray(sigma_q, np.int64)
        self.d = sigma_q.shape[0]
        self.cls = _groups(sigma_q)          # class key -> physical states
        self.A0 = _groups(bond_l)            # sector key -> a0 elements
        self.A2 = _groups(bond_r)
        self.bq = [_key(q) for q in bq]
        self.W = np.asarray(W)
        self.L = Lmats
        self.R = Rmats
        chiL, chiR = np.asarray(bond_l).shape[0], np.asarray(bond_r).shape[0]
        d = self.d
        self.allowed, _ = allowed_indices(r, sigma_q, np.asarray(bond_l, np.int64), sigma_q,
                                          np.asarray(bond_r, np.int64))
        lin = self.allowed
        s1 = lin % d
        a0 = (lin // d) % chiL
        s2 = (lin // (d * chiL)) % d
        a2 = lin // (d * chiL * d)
        # class / sector of every state and its position inside it
        ckey = [None] * d
        cpos = np.zeros(d, np.int64)
        for k, el in self.cls.items():
            for i, e in enumerate(el):
                ckey[e] = k
                cpos[e] = i

        def sec(groups, n):
            key = [None] * n
            pos = np.zeros(n, np.int64)
            for k, el in groups.items():
                for i, e in enumerate(el):
                    key[e] = k
                    pos[e] = i
            return key, pos
        k0key, k0pos = sec(self.A0, chiL)
        k2key, k2pos = sec(self.A2, chiR)
        # ARPACK entry -> (block, position inside the block)
        self.blocks = {}
        bk = [(ckey[a], k0key[b], ckey[c], k2key[e]) for a, b, c, e in zip(s1, a0, s2, a2)]
        for i, key in enumerate(bk):
            self.blocks.setdefault(key, []).append(i)
        self.maps = {}
        for key, ii in self.blocks.items():
            ii = np.asarray(ii, np.int64)
            self.maps[key] = (ii, cpos[s1[ii]], k0pos[a0[ii]], cpos[s2[ii]], k2pos[a2[ii]])
        # the MPO as d x d operator blocks per (b_l, b_r) pair, split by class
        self.ops = {}
        D = len(self.bq)
        for bl in range(D):
            for br in range(D):
                O = self.W[:, bl, :, br]
                if not np.any(O):
                    continue
                for ci, ei in self.cls.items():
                    for co, eo in self.cls.items():
                        blk = O[np.ix_(eo, ei)]
                        if np.any(blk):
                            self.ops.setdefault((bl, br), []).append((ci, co, blk))

    @property
    def n(self):
        return self.allowed.size

    def shape(self, key):
        c1, k0, c2, k2 = key
        return (self.cls[c1].size, self.A0[k0].size, self.cls[c2].size, self.A2[k2].size)

    def pack(self, x):
        th = {}
        for key, (ii, p1, p0, p2, p3) in self.maps.items():
            blk = np.zeros(self.shape(key), np.complex128)
            blk[p1, p0, p2, p3] = x[ii]
            th[key] = blk
        return th

    def unpack(self, th):
        out = np.zeros(self.n, np.complex128)
        for key, (ii, p1, p0, p2, p3) in self.maps.items():
            if key in th:
                out[ii] = th[key][p1, p0, p2, p3]
        return out

    def _acc(self, dst, key, val):
        if key in dst:
            dst[key] += val
        else:
            dst[key] = val

    def _used(self):
        """MPO slots some operator block reads on its left (b_l) and writes on
        its right (b_r): environment slots outside them (the reference's padded
        all-zero MPO slots) contribute nothing."""
        return {k[0] for k in self.ops}, {k[1] for k in self.ops}

    def matvec_blocks(self, th):
        D = len(self.bq)
        used_l, used_r = self._used()
        # stage L: X^{b0}[s1, a0', s2, a2] = sum_a0 L^{b0}[a0', a0] theta[s1, a0, s2, a2]
        X = {}
        for b0 in range(D):
            Lb = self.L[b0]
            if Lb is None or b0 not in used_l:
                continue
            for (c1, k0, c2, k2), t in th.items():
                k0p = self.add(k0, self.bq[b0])
                if k0p not in self.A0:
                    continue
                blk = Lb[np.ix_(self.A0[k0p], self.A0[k0])]
                if not np.any(blk):
                    continue
                n1, a, n2, b = t.shape
                v = np.matmul(blk, t.reshape(n1, a, n2 * b)).reshape(n1, blk.shape[0], n2, b)
                self._acc(X.setdefault(b0, {}), (c1, k0p, c2, k2), v)
        # stage W1: Y^{b1}[s1', a0', s2, a2] = sum_{b0, s1} W[s1', b0, s1, b1] X^{b0}[s1, ...]
        Y = {}
        for (b0, b1), ops in self.ops.items():
            if b0 not in X:
                continue
            for (c1, k0p, c2, k2), t in X[b0].items():
                for ci, co, O in ops:
                    if ci != c1:
                        continue
                    n1 = t.shape[0]
                    v = (O @ t.reshape(n1, -1)).reshape((O.shape[0],) + t.shape[1:])
                    self._acc(Y.setdefault(b1, {}), (co, k0p, c2, k2), v)
        # stage W2: Z^{b2}[s1', a0', s2', a2] = sum_{b1, s2} W[s2', b1, s2, b2] Y^{b1}[..., s2, a2]
        Z = {}
        for (b1, b2), ops in self.ops.items():
            if b1 not in Y:
                continue
            for (c1, k0p, c2, k2), t in Y[b1].items():
                for ci, co, O in ops:
                    if ci != c2:
                        continue
                    n1, a, n2, b = t.shape
                    v = np.matmul(O, t.reshape(n1 * a, n2, b)).reshape(n1, a, O.shape[0], b)
                    self._acc(Z.setdefault(b2, {}), (c1, k0p, co, k2), v)
        # stage R: theta'[s1', a0', s2', a2'] = sum_{b2, a2} Z^{b2}[..., a2] R^{b2}[a2', a2]
        out = {}
        for b2, blocks in Z.items():
            Rb = self.R[b2]
            if Rb is None or b2 not in used_r:
                continue
            for (c1, k0p, c2, k2), t in blocks.items():
                k2p = self.add(k2, self.bq[b2])
                if k2p not in self.A2:
                    continue
                blk = Rb[np.ix_(self.A2[k2p], self.A2[k2])]
                if not np.any(blk):
                    continue
                n1, a, n2, b = t.shape
                v = (t.reshape(-1, b) @ blk.T).reshape(n1, a, n2, blk.shape[0])
                self._acc(out, (c1, k0p, c2, k2p), v)
        return out

    def matvec(self, x):
        return self.unpack(self.matvec_blocks(self.pack(np.asarray(x, np.complex128))))

    def flops(self):
        """Algorithmic complex flops of one matvec in this order (8 per
        complex multiply-add, non-zero blocks only)."""
        D = len(self.bq)
        used_l, used_r = self._used()
        f = 0.0
        shapes = {key: self.shape(key) for key in self.maps}
        X = {}
        for b0 in range(D):
            if self.L[b0] is None or b0 not in used_l:
                continue
            for (c1, k0, c2, k2), (n1, a, n2, b) in shapes.items():
                k0p = self.add(k0, self.bq[b0])
                if k0p in self.A0 and np.any(self.L[b0][np.ix_(self.A0[k0p], self.A0[k0])]):
                    f += 8.0 * self.A0[k0p].size * a * n1 * n2 * b
                    X.setdefault(b0, set()).add((c1, k0p, c2, k2))
        Y = {}
        for (b0, b1), ops in self.ops.items():
            for (c1, k0p, c2, k2) in X.get(b0, ()):
                for ci, co, O in ops:
                    if ci == c1:
                        f += 8.0 * O.shape[0] * O.shape[1] * self.A0[k0p].size * self.cls[c2].size * self.A2[k2].size
                        Y.setdefault(b1, set()).add((co, k0p, c2, k2))
        Z = {}
        for (b1, b2), ops in self.ops.items():
            for (c1, k0p, c2, k2) in Y.get(b1, ()):
                for ci, co, O in ops:
                    if ci == c2:
                        f += 8.0 * O.shape[0] * O.shape[1] * self.cls[c1].size * self.A0[k0p].size * self.A2[k2].size
                        Z.setdefault(b2, set()).add((c1, k0p, co, k2))
        for b2, keys in Z.items():
            if self.R[b2] is None:
                continue
            for (c1, k0p, c2, k2) in keys:
                k2p = self.add(k2, self.bq[b2])
                if k2p in self.A2 and np.any(self.R[b2][np.ix_(self.A2[k2p], self.A2[k2])]):
                    f += 8.0 * self.cls[c1].size * self.A0[k0p].size * self.cls[c2].size * self.A2[k2].size * \
                        self.A2[k2p].size
        return f


def from_mpx(H, L, R):
    """CanonicalHeff from the reference-layout dense tensors (MPO H, left
    block L with a' = 1, b = 3, a = 5, right block R with a' = 0, b = 2,
    a = 4)."""
    D = H.indices[1].size
    chiL = L.indices[5].size
    chiR = R.indices[4].size
    Lt = np.asarray(L.data).reshape(L.indices[1].size, D, chiL)
    Rt = np.asarray(R.data).reshape(R.indices[0].size, D, chiR)
    Lm = [Lt[:, b, :] if np.any(Lt[:, b, :]) else None for b in range(D)]
    Rm = [Rt[:, b, :] if np.any(Rt[:, b, :]) else None for b in range(D)]
    return CanonicalHeff(H.rules, H.indices[0].charges, L.indices[5].charges, R.indices[4].charges,
                         H.indices[1].charges, H.data, Lm, Rm)
