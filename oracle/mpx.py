"""CPU oracle (test infrastructure only): labelled charge tensors.

This module restates, in numpy, the tensor layer of ChainAMPS that the DMRG
hot path runs on.  It is the checker for the CUDA library and is imported
only by ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py``.  Nothing in the product path
imports it.

Reference semantics restated here (file:line in andyjaj/chainamps):

* charges: ``State::operator+=`` / ``-=`` -- Z_N charges add modulo N, N<=0
  charges are plain integers (``states.hpp:176-206``);
* directed indices with per-element charges (``MPXIndex.hpp:17-65``);
  ``flip`` reverses the direction (``MPXIndex.hpp:56``);
* a tensor is one matrix whose rows combine the first ``nrow`` indices and
  whose columns combine the rest, the first index running fastest
  (``sparse_interface.cpp:85-91`` ``index_decompose``,
  ``MPX_matrix.cpp:316-363``);
* ``contract`` keeps A's free indices then B's free indices, the result has
  as many row indices as A has free indices, and conjugation flips the
  direction of every index of the conjugated operand
  (``MPX_matrix.cpp:744-791``);
* ``reorder`` permutes indices (``MPX_matrix.cpp:630-638``);
* ``IngoingRowState`` / ``OutgoingColState`` / ``GetAllBlockColumns``
  (``MPX_matrix.cpp:331-385``).

The reference stores each tensor as one CSC matrix.  The oracle stores the
same tensor densely (numpy array with one axis per index), which gives the
same numbers at the sizes the oracle is used for; CSC conversion lives in
``to_csc`` / ``from_csc`` for feeding the library's C ABI exactly what the
reference would hand it.
"""
from __future__ import annotations

from dataclasses import dataclass, field
import numpy as np

EPS = np.finfo(np.float64).eps  # SPARSETOL (sparse_interface.hpp:15)


# --------------------------------------------------------------------------
# charges
# --------------------------------------------------------------------------
def q_add(a, b, rules):
    """State::operator+= (states.hpp:176-188); arrays (..., nq)."""
    out = np.asarray(a, dtype=np.int64) + np.asarray(b, dtype=np.int64)
    for i, n in enumerate(rules):
        if n > 0:
            out[..., i] %= n
    return out


def q_sub(a, b, rules):
    """State::operator-= (states.hpp:190-206)."""
    out = np.asarray(a, dtype=np.int64) - np.asarray(b, dtype=np.int64)
    for i, n in enumerate(rules):
        if n > 0:
            out[..., i] %= n
    return out


def q_neg(a, rules):
    return q_sub(np.zeros_like(np.asarray(a, dtype=np.int64)), a, rules)


def q_eq(a, b):
    return np.all(np.asarray(a) == np.asarray(b), axis=-1)


# --------------------------------------------------------------------------
# indices and tensors
# --------------------------------------------------------------------------
@dataclass
class Index:
    """MPXIndex: direction, physical flag, one charge vector per element."""
    inward: bool
    physical: bool
    charges: np.ndarray  # (size, nq) int64

    @property
    def size(self) -> int:
        return int(self.charges.shape[0])

    def flip(self) -> "Index":
        return Index(not self.inward, self.physical, self.charges)

    def with_dir(self, inward: bool) -> "Index":
        return Index(inward, self.physical, self.charges)


def dummy_index(inward: bool, charge, nq: int) -> Index:
    c = np.asarray(charge, dtype=np.int64).reshape(1, nq)
    return Index(inward, False, c)


@dataclass
class MPX:
    """Labelled tensor: ``data`` has one axis per index (index order)."""
    rules: tuple
    indices: list
    nrow: int
    data: np.ndarray = field(repr=False)

    def __post_init__(self):
        shp = tuple(ix.size for ix in self.indices)
        if self.data.shape != shp:
            raise ValueError(f"data shape {self.data.shape} != index sizes {shp}")

    @property
    def nq(self) -> int:
        return len(self.rules)

    def dims(self):
        return [ix.size for ix in self.indices]

    def rows(self) -> int:
        return int(np.prod([ix.size for ix in self.indices[: self.nrow]], dtype=np.int64))

    def cols(self) -> int:
        return int(np.prod([ix.size for ix in self.indices[self.nrow:]], dtype=np.int64))

    def matrix(self) -> np.ndarray:
        """Rows = first nrow indices, first index fastest (column-major)."""
        return self.data.reshape((self.rows(), self.cols()), order="F")

    def copy(self) -> "MPX":
        return MPX(self.rules, list(self.indices), self.nrow, self.data.copy())

    # charge bookkeeping ---------------------------------------------------
    def _combined(self, idx_list, sign_in):
        """Charge of every combined element of ``idx_list`` (first fastest).

        sign_in=+1: ingoing adds, outgoing subtracts (IngoingRowState);
        sign_in=-1: outgoing adds, ingoing subtracts (OutgoingColState).
        """
        acc = np.zeros((1, self.nq), dtype=np.int64)
        for ix in idx_list:
            add = ix.inward if sign_in > 0 else (not ix.inward)
            c = ix.charges
            # new combined = old (fast) + c (slow): element l = i + n_old * j
            if add:
                acc = q_add(acc[None, :, :], c[:, None, :], self.rules).reshape(-1, self.nq)
            else:
                acc = q_sub(acc[None, :, :], c[:, None, :], self.rules).reshape(-1, self.nq)
        return acc

    def ingoing_row_states(self):
        """IngoingRowState for every row (MPX_matrix.cpp:347-363)."""
        return self._combined(self.indices[: self.nrow], +1)

    def outgoing_col_states(self):
        """OutgoingColState for every column (MPX_matrix.cpp:331-345)."""
        return self._combined(self.indices[self.nrow:], -1)

    def block_columns(self):
        """GetAllBlockColumns (MPX_matrix.cpp:365-385): groups of columns with
        equal outgoing charge, groups in order of first appearance."""
        cs = self.outgoing_col_states()
        groups = {}
        order = []
        for c in range(cs.shape[0]):
            key = tuple(int(v) for v in cs[c])
            if key not in groups:
                groups[key] = []
                order.append(key)
            groups[key].append(c)
        return [(k, groups[k]) for k in order]

    def is_consistent(self, tol=0.0) -> bool:
        """isConsistent (MPX_matrix.cpp:275-302): every stored entry conserves charge."""
        M = self.matrix()
        rs = self.ingoing_row_states()
        cs = self.outgoing_col_states()
        nz = np.nonzero(np.abs(M) > tol)
        return bool(np.all(q_eq(rs[nz[0]], cs[nz[1]])))


def from_matrix(rules, indices, nrow, M) -> MPX:
    shp = tuple(ix.size for ix in indices)
    return MPX(tuple(rules), list(indices), nrow, np.asarray(M, dtype=np.complex128).reshape(shp, order="F"))


# --------------------------------------------------------------------------
# operations
# --------------------------------------------------------------------------
def contract(A: MPX, conjA: bool, B: MPX, conjB: bool, pairs) -> MPX:
    """contract (MPX_matrix.cpp:744-791) on dense data."""
    for a, b in pairs:
        ia, ib = A.indices[a], B.indices[b]
        if ia.physical != ib.physical or ia.size != ib.size:
            raise ValueError("indices don't match")
        # A outgoing (after conj) must meet B ingoing (after conj): match() MPXIndex.cpp:47-72
        if ((not ia.inward) != conjA) != (ib.inward != conjB):
            raise ValueError("index directions don't match")
    ad = np.conj(A.data) if conjA else A.data
    bd = np.conj(B.data) if conjB else B.data
    axa = [p[0] for p in pairs]
    axb = [p[1] for p in pairs]
    data = np.tensordot(ad, bd, axes=(axa, axb))
    idx = []
    for i, ix in enumerate(A.indices):
        if i not in axa:
            idx.append(ix.flip() if conjA else ix)
    nrow = len(idx)
    for i, ix in enumerate(B.indices):
        if i not in axb:
            idx.append(ix.flip() if conjB else ix)
    return MPX(A.rules, idx, nrow, np.ascontiguousarray(data))


def reorder(A: MPX, conj: bool, order, nrow) -> MPX:
    """reorder (MPX_matrix.cpp:630-638)."""
    data = np.transpose(A.data, order)
    if conj:
        data = np.conj(data)
    idx = [(A.indices[o].flip() if conj else A.indices[o]) for o in order]
    return MPX(A.rules, idx, nrow, np.ascontiguousarray(data))


def remove_dummy(A: MPX, which) -> MPX:
    """RemoveDummyIndices (MPX_matrix.cpp:415-457)."""
    which = list(which)
    for i in which:
        if A.indices[i].size != 1:
            raise ValueError("not a dummy index")
    keep = [i for i in range(len(A.indices)) if i not in which]
    nrow = A.nrow - sum(1 for i in which if i < A.nrow)
    shp = tuple(A.indices[i].size for i in keep)
    return MPX(A.rules, [A.indices[i] for i in keep], nrow, A.data.reshape(shp))


def shift_num_rows(A: MPX, nrow) -> MPX:
    """ShiftNumRowIndices (MPX_matrix.cpp:72-85): same tensor, new row split."""
    return MPX(A.rules, list(A.indices), nrow, A.data)


def move_dummy(A: MPX, order) -> MPX:
    """MoveDummyIndices (MPX_matrix.cpp:87-109): permute index labels, the
    first column index keeps being the first column index."""
    nrow = A.nrow
    for pos, o in enumerate(order):
        if o == nrow:
            nrow = pos
    nondummy = [o for o in order if A.indices[o].size > 1]
    if any(nondummy[i] <= nondummy[i - 1] for i in range(1, len(nondummy))):
        raise ValueError("non dummy order shouldn't change")
    return MPX(A.rules, [A.indices[o] for o in order], nrow, np.ascontiguousarray(np.transpose(A.data, order)))


def diag_mpx(rules, index: Index, values, inverse=False, rindex: Index | None = None) -> MPX:
    """Diagonal MPX_matrix(spectrum, index, values) (MPX_matrix.cpp:37-70):
    index ingoing on the rows, outgoing on the columns."""
    v = np.asarray(values, dtype=np.complex128)
    if inverse:
        v = 1.0 / v
    li = index.with_dir(True)
    ri = (rindex if rindex is not None else index).with_dir(False)
    return from_matrix(rules, [li, ri], 1, np.diag(v))


# --------------------------------------------------------------------------
# CSC interchange (the reference's storage, sparse_interface.hpp:78-202)
# --------------------------------------------------------------------------
def to_csc(A: MPX, drop=0.0):
    """Return (rows, cols, colptr, rowind, values) of the matrix form,
    entries with |x| <= drop omitted, row indices ascending per column."""
    M = A.matrix()
    rows, cols = M.shape
    colptr = np.zeros(cols + 1, dtype=np.int64)
    ri = []
    vals = []
    for c in range(cols):
        col = M[:, c]
        nz = np.nonzero(np.abs(col) > drop)[0]
        ri.append(nz)
        vals.append(col[nz])
        colptr[c + 1] = colptr[c] + nz.size
    rowind = np.concatenate(ri).astype(np.int64) if ri else np.zeros(0, np.int64)
    values = np.concatenate(vals).astype(np.complex128) if vals else np.zeros(0, np.complex128)
    return rows, cols, colptr, rowind, values


def from_csc(rules, indices, nrow, rows, cols, colptr, rowind, values) -> MPX:
    M = np.zeros((rows, cols), dtype=np.complex128)
    for c in range(cols):
        for p in range(colptr[c], colptr[c + 1]):
            M[rowind[p], c] += values[p]
    return from_matrix(rules, indices, nrow, M)
