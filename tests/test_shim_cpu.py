"""The C++ shims of the reference's seams compile (no GPU, no reference
library needed).

* include/chainamps_b200_shim_core.hpp -- the reference-independent layer --
  and the shim_window client compile as C++11 and C++17 with -Wall -Wextra
  -Werror;
* include/chainamps_b200_shim.hpp -- the layer that keeps the reference's
  signatures (TwoVertexMPOMPSMultiply, TwoVertexComponents::HED,
  MPX_matrix::SVD, MakeLeftBlock / MakeRightBlock) -- compiles against the
  reference's own headers, where a checkout of the reference is present
  (CHAINAMPS_REFERENCE, default the usual checkout path), with a
  declarations-only cs.h standing in for CXSparse's; the shim's own lines
  raise no warning under -Wall -Wextra."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
REF = os.environ.get("CHAINAMPS_REFERENCE", "/root/reference")


def gxx():
    g = shutil.which("g++")
    if not g:
        pytest.skip("g++ not available")
    return g


@pytest.mark.parametrize("std", ["c++11", "c++17"])
def test_core_shim_compiles(tmp_path, std):
    src = tmp_path / "tu.cpp"
    src.write_text('#include "chainamps_b200_shim_core.hpp"\nint main() { return 0; }\n')
    subprocess.run([gxx(), f"-std={std}", "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-I", INC, str(src)],
                   check=True)
    subprocess.run([gxx(), f"-std={std}", "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-I", INC,
                    os.path.join(ROOT, "tests", "abi", "shim_window.cpp")], check=True)


def test_reference_shim_compiles_against_the_reference_headers(tmp_path):
    if not os.path.exists(os.path.join(REF, "DMRG_routines.hpp")):
        pytest.skip("the reference's headers are not present here")
    src = tmp_path / "tu.cpp"
    src.write_text('#include "chainamps_b200_shim.hpp"\n')
    r = subprocess.run([gxx(), "-std=c++11", "-Wall", "-Wextra", "-fsyntax-only", "-I", INC, "-I",
                        os.path.join(ROOT, "tests", "abi", "refshim"), "-I", REF, str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    own = [ln for ln in r.stderr.splitlines() if "chainamps_b200_shim" in ln and ("warning" in ln or "error" in ln)]
    assert not own, "\n".join(own)
