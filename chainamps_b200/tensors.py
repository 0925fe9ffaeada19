"""Containers of the reference's tensor storage, numpy only.

``MPXTensor`` is the MPX_matrix storage (MPX_matrix.hpp:61-66): directed,
charge-labelled indices, the number of row indices, and one CSC matrix
with the first index fastest.  ``MPXIndexSpec`` is one MPXIndex
(MPXIndex.hpp:17-65).  Building or holding these does not load the CUDA
library; only turning one into the C ABI descriptor (``_desc``, at a call
into the library) does.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class MPXIndexSpec:
    inward: bool
    physical: bool
    charges: np.ndarray  # (size, nq) int


@dataclass
class MPXTensor:
    """MPX_matrix storage (MPX_matrix.hpp:61-66): indices, number of row
    indices, CSC matrix (rows, cols, colptr, rowind, complex values)."""
    indices: list
    nrow: int
    rows: int
    cols: int
    colptr: np.ndarray
    rowind: np.ndarray
    values: np.ndarray

    def _desc(self):
        keep = []
        inward = np.array([1 if i.inward else 0 for i in self.indices], np.uint8)
        phys = np.array([1 if i.physical else 0 for i in self.indices], np.uint8)
        sizes = np.array([i.charges.shape[0] for i in self.indices], np.int64)
        charges = np.ascontiguousarray(np.concatenate([np.asarray(i.charges, np.int16).reshape(i.charges.shape[0], -1)
                                                       for i in self.indices], axis=0))
        colptr = np.ascontiguousarray(self.colptr, np.int64)
        rowind = np.ascontiguousarray(self.rowind, np.int64)
        vals = np.ascontiguousarray(np.asarray(self.values, np.complex128)).view(np.float64)
        if rowind.size == 0:
            rowind = np.zeros(1, np.int64)
            vals = np.zeros(2, np.float64)
        keep += [inward, phys, sizes, charges, colptr, rowind, vals]
        import ctypes as C

        from .capi import MpxDesc, _p  # the C ABI descriptor: loads the library
        d = MpxDesc(len(self.indices), self.nrow, _p(inward, C.c_uint8), _p(phys, C.c_uint8), _p(sizes, C.c_int64),
                    _p(charges, C.c_int16), self.rows, self.cols, _p(colptr, C.c_int64), _p(rowind, C.c_int64),
                    _p(vals, C.c_double))
        return d, keep
