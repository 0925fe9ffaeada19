"""The C++ shim of the reference's seams on the GPU, against the oracle.

tests/abi/shim_window.cpp is a C++ client of
include/chainamps_b200_shim_core.hpp linked against the library.  It reads
one two-vertex window -- environments L, R and the MPO W -- from
MPX_matrix files written in the reference's format by the oracle's writer,
then drives it through the reference's seams: the ARPACK MV callback shape
of TwoVertexMPOMPSMultiply on host std::complex<double> buffers, the lowest
eigenpair (TwoVertexComponents::HED) and the block SVD.  Checked: the
allowed indices exactly, the matvec within 1e-12 relative (max-norm), the
energy within 1e-10 relative, the kept singular values within 1e-8."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import dmrg as od, mpxio as om
from oracle.mpx import from_matrix, to_csc
from tests.helpers import model_zoo

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "chainamps_b200", "libchainamps_b200.so")
ZOO = model_zoo()


def write_mpx(A, path, nq):
    rows, cols, cp, ri, vals = to_csc(A)
    idx = [(ix.inward, ix.physical, ix.charges) for ix in A.indices]
    with open(path, "wb") as f:
        f.write(om.mpx_bytes(idx, A.nrow, rows, cols, cp, ri, vals, nq))


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    if not os.path.exists(LIB):
        pytest.fail("libchainamps_b200.so is not built")
    out = tmp_path_factory.mktemp("shim") / "shim_window"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "abi", "shim_window.cpp"), LIB,
                    "-Wl,-rpath," + os.path.dirname(LIB), "-o", str(out)], check=True)
    return str(out)


@pytest.mark.parametrize("name,steps,chi", [("xxz", 6, 24), ("ladder4", 2, 16)])
def test_shim_window_matches_the_oracle(tmp_path, exe, name, steps, chi):
    H = ZOO[name]
    nq = len(H.rules)
    sb = od.SuperBlock(H, tol=1e-12)
    for _ in range(steps):
        sb.grow(chi, 1e-16)
    L = od.make_left_block(sb.left_blocks[sb.nleft], H, sb.dec.U)
    R = od.make_right_block(sb.right_blocks[sb.nleft], H, sb.dec.Vd)
    ref = od.TwoVertexComponents(L, H, R)
    write_mpx(L, tmp_path / "L.MPX_matrix", nq)
    write_mpx(H, tmp_path / "W.MPX_matrix", nq)
    write_mpx(R, tmp_path / "R.MPX_matrix", nq)
    np.asarray(H.rules, "<i2").tofile(tmp_path / "rules.i16")
    basis = next(ix.charges for ix in H.indices if ix.physical)
    np.asarray(basis, "<i2").reshape(-1).tofile(tmp_path / "basis.i16")
    rng = np.random.default_rng(3)
    n = ref.allowed.size
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    x.astype("<c16").tofile(tmp_path / "x.c128")
    r = subprocess.run([exe, str(tmp_path), str(nq), str(chi), "1e-16"], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    np.testing.assert_array_equal(np.fromfile(tmp_path / "allowed.i64", "<i8"), ref.allowed)
    y = np.fromfile(tmp_path / "y.c128", "<c16")
    want = ref.matvec(x)
    assert np.max(np.abs(y - want)) <= 1e-12 * np.max(np.abs(want))
    e_ref, full_ref = ref.hed(tol=1e-14)
    e = float(np.fromfile(tmp_path / "energy.f64", "<f8")[0])
    assert abs(e - e_ref) <= 1e-10 * abs(e_ref)
    v = np.fromfile(tmp_path / "evec.c128", "<c16")
    assert abs(abs(np.vdot(full_ref[ref.allowed], v)) - 1.0) <= 1e-8
    theta = from_matrix(H.rules, ref.indices, 2, full_ref.reshape((ref.vrows, ref.vcols), order="F"))
    dref = od.block_svd(theta, chi, 1e-16)
    vals = np.fromfile(tmp_path / "values.f64", "<f8")
    assert vals.size == dref.values.size
    np.testing.assert_allclose(vals, dref.values, atol=1e-8)
