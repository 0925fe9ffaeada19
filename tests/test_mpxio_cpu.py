"""The reference's binary MPX_matrix file format through the C ABI (host
only, no GPU): cmps_mpx_store writes the bytes of MPX_matrix::store, and
cmps_mpx_load reads them back as load_MPX_matrix does.

Checked against the oracle's restatement of the format (oracle/mpxio.py):
* the library's file equals the oracle's bytes exactly, for an MPO (with
  physical indices), a grown left environment block (the .BLOCK
  checkpoint), an MPS tensor from the block SVD (the .MPS_matrix file), a
  two-charge MPO, and an empty matrix;
* loading returns the same indices, row-index count and CSC matrix;
* an exported device block converts to the reference's 6-index block layout
  (block_mpx_tensor) with the same bytes as the oracle's block;
* the reader keeps the first colptr[cols] of nzmax stored entries, and
  refuses a matrix not in compressed-column form, a truncated file and a
  physical index without (or with the wrong) basis."""
import numpy as np
import pytest

from oracle import dmrg as od, mpxio as om
from oracle.mpx import MPX, to_csc
from tests.helpers import to_tensor, model_zoo

ZOO = model_zoo()


def lib():
    from chainamps_b200 import capi
    return capi


def oracle_bytes(A: MPX, **kw):
    rows, cols, cp, ri, vals = to_csc(A)
    idx = [(ix.inward, ix.physical, ix.charges) for ix in A.indices]
    return om.mpx_bytes(idx, A.nrow, rows, cols, cp, ri, vals, len(A.rules), **kw)


def basis_of(H: MPX):
    return next(ix.charges for ix in H.indices if ix.physical)


def samples():
    H = ZOO["xxz"]
    sb = od.SuperBlock(H, tol=1e-12)
    for _ in range(4):
        sb.grow(12, 1e-16)
    out = {
        "mpo_xxz": (H, basis_of(H)),
        "mpo_twocharge": (ZOO["twocharge"], basis_of(ZOO["twocharge"])),
        "left_block": (sb.left_blocks[sb.nleft], None),
        "right_block": (sb.right_blocks[sb.nleft], None),
        "mps_U": (sb.dec.U, basis_of(H)),
    }
    # an empty matrix: the zero MPO of the same indices
    Z = MPX(H.rules, list(H.indices), H.nrow, np.zeros_like(H.data))
    out["empty"] = (Z, basis_of(H))
    return out


SAMPLES = samples()


@pytest.mark.parametrize("name", sorted(SAMPLES))
def test_store_writes_the_reference_bytes_and_loads_back(tmp_path, name):
    capi = lib()
    A, basis = SAMPLES[name]
    path = tmp_path / f"{name}.MPX_matrix"
    capi.store_mpx(to_tensor(A), len(A.rules), path)
    data = path.read_bytes()
    assert data == oracle_bytes(A)
    t = capi.load_mpx(path, len(A.rules), basis)
    ref = to_tensor(A)
    assert t.nrow == A.nrow and t.rows == ref.rows and t.cols == ref.cols
    assert len(t.indices) == len(A.indices)
    for a, b in zip(t.indices, A.indices):
        assert a.inward == b.inward and a.physical == b.physical
        np.testing.assert_array_equal(a.charges, np.asarray(b.charges, np.int64))
    np.testing.assert_array_equal(t.colptr, ref.colptr)
    np.testing.assert_array_equal(t.rowind, ref.rowind)
    np.testing.assert_array_equal(t.values, ref.values)
    # the oracle reads the library's file the same way
    idx, nrow, rows, cols, cp, ri, vals = om.parse(data, len(A.rules), basis)
    assert nrow == A.nrow and (rows, cols) == (ref.rows, ref.cols)
    np.testing.assert_array_equal(cp, ref.colptr)
    np.testing.assert_array_equal(vals, ref.values)


def test_reader_keeps_the_first_colptr_entries_of_nzmax(tmp_path):
    capi = lib()
    A = SAMPLES["left_block"][0]
    ref = to_tensor(A)
    nnz = int(ref.colptr[-1])
    path = tmp_path / "padded.BLOCK"
    path.write_bytes(oracle_bytes(A, nzmax=nnz + 7, fill=(0, 3.0 - 1.0j)))
    t = capi.load_mpx(path, len(A.rules))
    np.testing.assert_array_equal(t.rowind, ref.rowind)
    np.testing.assert_array_equal(t.values, ref.values)


def test_reader_refuses_bad_files(tmp_path):
    capi = lib()
    A, basis = SAMPLES["mpo_xxz"]
    nq = len(A.rules)
    good = oracle_bytes(A)
    # nz != -1 (triplet form): the reference exits, the library returns an error;
    # the matrix header starts after the index records
    rows, cols, cp, ri, vals = to_csc(A)
    head = len(good) - (8 * 4 + 8 * (cols + 1) + (8 + 16) * max(int(cp[-1]), 1))
    bad = bytearray(good)
    bad[head + 8:head + 16] = np.int64(0).tobytes()
    p = tmp_path / "triplet.MPX_matrix"
    p.write_bytes(bytes(bad))
    with pytest.raises(capi.CmpsError):
        capi.load_mpx(p, nq, basis)
    # truncated
    p = tmp_path / "short.MPX_matrix"
    p.write_bytes(good[:-5])
    with pytest.raises(capi.CmpsError):
        capi.load_mpx(p, nq, basis)
    # physical index without the basis, and with a basis of the wrong size
    p = tmp_path / "mpo.MPX_matrix"
    p.write_bytes(good)
    with pytest.raises(capi.CmpsError):
        capi.load_mpx(p, nq, None)
    with pytest.raises(capi.CmpsError):
        capi.load_mpx(p, nq, np.vstack([basis, basis]))
    # a missing file
    with pytest.raises(capi.CmpsError):
        capi.load_mpx(tmp_path / "none.MPX_matrix", nq, basis)


def test_reader_refuses_counts_beyond_the_file_size(tmp_path):
    """A corrupt header whose nzmax or column count claims more data than the
    file holds is refused with an error before anything of that size is
    allocated (no std::bad_alloc escapes the C ABI)."""
    capi = lib()
    A, basis = SAMPLES["mpo_xxz"]
    nq = len(A.rules)
    good = oracle_bytes(A)
    rows, cols, cp, ri, vals = to_csc(A)
    head = len(good) - (8 * 4 + 8 * (cols + 1) + (8 + 16) * max(int(cp[-1]), 1))
    for field, value in ((0, 1 << 60), (0, 1 << 33)):
        bad = bytearray(good)
        bad[head + 8 * field:head + 8 * field + 8] = np.int64(value).tobytes()
        p = tmp_path / f"nzmax{value}.MPX_matrix"
        p.write_bytes(bytes(bad))
        with pytest.raises(capi.CmpsError, match="truncated"):
            capi.load_mpx(p, nq, basis)
    # columns: shape check or size check refuses it, never an allocation of 2^39 entries
    bad = bytearray(good)
    bad[head + 24:head + 32] = np.int64(1 << 39).tobytes()
    p = tmp_path / "cols.MPX_matrix"
    p.write_bytes(bytes(bad))
    with pytest.raises(capi.CmpsError):
        capi.load_mpx(p, nq, basis)


def test_store_refuses_inconsistent_shapes(tmp_path):
    capi = lib()
    A = SAMPLES["left_block"][0]
    t = to_tensor(A)
    t.rows += 1
    with pytest.raises(capi.CmpsError):
        capi.store_mpx(t, len(A.rules), tmp_path / "bad.BLOCK")


@pytest.mark.parametrize("target", [(0,), (2,)])
@pytest.mark.parametrize("right", [False, True])
def test_block_layout_from_the_export(tmp_path, target, right):
    """block_mpx_tensor turns a block in cmps_block_copy's export layout (a'
    charges; CSC rows a', cols b + D a) into the reference's 6-index block:
    the same indices, charges and matrix as the oracle's MakeLeftBlock /
    MakeRightBlock result, hence the same .BLOCK bytes."""
    capi = lib()
    H = ZOO["xxz"]
    sb = od.SuperBlock(H, target=list(target), tol=1e-12)
    for _ in range(4):
        sb.grow(12, 1e-16)
    B = (sb.right_blocks if right else sb.left_blocks)[sb.nleft]
    bond = B.indices[0 if right else 1].charges
    rows, cols, cp, ri, vals = to_csc(B)        # rows a', cols b + D a: the export layout
    D = H.indices[1].size
    assert (rows, cols) == (bond.shape[0], D * bond.shape[0])
    t = capi.block_mpx_tensor(bond, (cp, ri, vals), D, H.indices[1].charges, right, target)
    ref = to_tensor(B)
    assert t.nrow == ref.nrow
    for a, b in zip(t.indices, ref.indices):
        assert a.inward == b.inward and a.physical == b.physical
        np.testing.assert_array_equal(a.charges, np.asarray(b.charges, np.int64))
    p1, p2 = tmp_path / "mine.BLOCK", tmp_path / "ref.BLOCK"
    capi.store_mpx(t, 1, p1)
    capi.store_mpx(ref, 1, p2)
    assert p1.read_bytes() == p2.read_bytes() == oracle_bytes(B)


def test_mps_decomposition_files():
    """mps_decomposition_tensors turns an SVD result in SVDResult.copy's
    layout (CSC of U rows (sigma1, a0) and of V^dagger cols (sigma2, a2), new
    bond charges, values) into the LeftMatrix, RightMatrix and Lambda files
    MPSDecomposition::store writes: the same bytes as the oracle's block SVD
    factors and its diagonal Lambda."""
    import os
    import tempfile
    from oracle.mpx import diag_mpx
    capi = lib()
    H = ZOO["xxz"]
    sb = od.SuperBlock(H, tol=1e-12)
    for _ in range(5):
        sb.grow(10, 1e-16)
    dec = sb.dec
    _, _, ucp, uri, uv = to_csc(dec.U)
    _, _, vcp, vri, vv = to_csc(dec.Vd)
    copy = dict(values=dec.values, charges=dec.U.indices[2].charges, u=(ucp, uri, uv), vd=(vcp, vri, vv))
    basis = basis_of(H)
    U, Vd, Lam = capi.mps_decomposition_tensors(copy, basis, dec.U.indices[1].charges, dec.Vd.indices[2].charges)
    lam_ref = diag_mpx(H.rules, dec.U.indices[2], dec.values)
    with tempfile.TemporaryDirectory() as tmp:
        for t, ref in ((U, dec.U), (Vd, dec.Vd), (Lam, lam_ref)):
            p = os.path.join(tmp, "x.MPS_matrix")
            capi.store_mpx(t, len(H.rules), p)
            assert open(p, "rb").read() == oracle_bytes(ref)


def test_reader_takes_a_file_with_nzmax_zero(tmp_path):
    """load_SparseMatrix_binary's nzmax == 0 branch (sparse_interface.cpp:
    820-830): only the column pointers follow the header; the matrix is
    empty."""
    capi = lib()
    A, basis = SAMPLES["empty"]
    rows, cols, cp, ri, vals = to_csc(A)
    data = oracle_bytes(A)
    head = len(data) - (8 * 4 + 8 * (cols + 1) + 8 + 16)
    buf = bytearray(data[:head + 8 * 4 + 8 * (cols + 1)])     # no placeholder entry
    buf[head:head + 8] = np.int64(0).tobytes()                # nzmax = 0
    p = tmp_path / "nzmax0.MPX_matrix"
    p.write_bytes(bytes(buf))
    t = capi.load_mpx(p, len(A.rules), basis)
    assert (t.rows, t.cols) == (rows, cols)
    assert t.colptr[-1] == 0 and t.rowind.size == 0 and t.values.size == 0
