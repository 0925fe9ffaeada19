"""CPU restatement of the reference's binary MPX_matrix file format.  Test
infrastructure (the oracle): only tests use it.

The bytes follow the reference's writers, field by field, as they lay out
on x86-64 Linux (little-endian; size_t, SuiteSparse_long 8 bytes; bool 1;
QuantumNumberInt = short, common_defs.hpp:20):

* MPX_matrix::fprint_binary (MPX_matrix.cpp:219-233): size_t number of
  indices, Sparseint number of row indices, every MPXIndex, the matrix.
* MPXIndex::fprint_binary (MPXIndex.cpp:8-23): bool inward, bool physical,
  size_t size; the State of every element only for a non-physical index of
  non-zero size (State::fprint_binary, states.cpp:59-61: nq shorts).
* SparseMatrix::fprint_binary (sparse_interface.cpp:727-764): Sparseint
  nzmax, nz, m, n; p[n + 1]; if p[n] == 0 one Sparseint 0 and one complex 0,
  else i[nzmax] and x[nzmax] (complex<double>).

The reader follows load_MPX_matrix_binary (MPX_matrix.cpp:593-607),
load_MPXIndex_binary (MPXIndex.cpp:98-121: a physical index takes the basis)
and load_SparseMatrix_binary (sparse_interface.cpp:767-835: nz must be -1;
the placeholder of an empty matrix is not read back).

No file written by the reference ships with it, so this restatement is
pinned by the source only ("parity unpinned" by reference-written files).
"""
import struct

import numpy as np


def mpx_bytes(indices, nrow, rows, cols, colptr, rowind, values, nq, nzmax=None, fill=None):
    """Bytes of MPX_matrix::store for one MPX.  indices: (inward, physical,
    charges (size, nq)) triples.  nzmax defaults to max(nnz, 1), what a
    finalised reference matrix holds; a larger nzmax pads the entry arrays
    with `fill` (row index, value) pairs, as an unfinalised buffer would."""
    out = bytearray(struct.pack("<Qq", len(indices), nrow))
    for inward, physical, charges in indices:
        ch = np.asarray(charges).reshape(-1, nq)
        out += struct.pack("<??Q", bool(inward), bool(physical), ch.shape[0])
        if not physical and ch.shape[0] > 0:
            out += ch.astype("<i2").tobytes()
    colptr = np.asarray(colptr, np.int64)
    nnz = int(colptr[-1])
    if nzmax is None:
        nzmax = max(nnz, 1)
    out += struct.pack("<4q", nzmax, -1, rows, cols)
    out += colptr.astype("<i8").tobytes()
    if nnz == 0:
        out += struct.pack("<q", 0) + np.zeros(2, "<f8").tobytes()
    else:
        ri = np.zeros(nzmax, np.int64)
        x = np.zeros(nzmax, np.complex128)
        ri[:nnz] = rowind
        x[:nnz] = values
        if fill is not None and nzmax > nnz:
            ri[nnz:] = fill[0]
            x[nnz:] = fill[1]
        out += ri.astype("<i8").tobytes() + x.astype("<c16").tobytes()
    return bytes(out)


def parse(buf, nq, basis_charges=None):
    """Inverse of mpx_bytes: (indices, nrow, rows, cols, colptr, rowind,
    values); physical indices take basis_charges."""
    pos = 0

    def take(fmt):
        nonlocal pos
        v = struct.unpack_from(fmt, buf, pos)
        pos += struct.calcsize(fmt)
        return v

    n, nrow = take("<Qq")
    indices = []
    for _ in range(n):
        inward, physical, size = take("<??Q")
        if physical:
            ch = np.asarray(basis_charges, np.int64).reshape(-1, nq)
            if ch.shape[0] != size:
                raise ValueError("physical index size differs from the basis")
        elif size > 0:
            ch = np.frombuffer(buf, "<i2", size * nq, pos).reshape(size, nq).astype(np.int64)
            pos += 2 * size * nq
        else:
            ch = np.zeros((0, nq), np.int64)
        indices.append((inward, physical, ch))
    nzmax, nz, rows, cols = take("<4q")
    if nz != -1:
        raise ValueError("not in compressed-column form")
    colptr = np.frombuffer(buf, "<i8", cols + 1, pos).astype(np.int64)
    pos += 8 * (cols + 1)
    nnz = int(colptr[-1])
    rowind = np.zeros(0, np.int64)
    values = np.zeros(0, np.complex128)
    if nzmax > 0 and nnz > 0:
        rowind = np.frombuffer(buf, "<i8", nzmax, pos).astype(np.int64)[:nnz]
        pos += 8 * nzmax
        values = np.frombuffer(buf, "<c16", nzmax, pos).astype(np.complex128)[:nnz]
    return indices, nrow, rows, cols, colptr, rowind, values
