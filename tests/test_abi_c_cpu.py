"""The public header as a C99 client sees it (no GPU): tests/abi/mpx_roundtrip.c
includes include/chainamps_b200.h, is compiled with gcc -std=c99 -Wall
-Werror, links against the library and round-trips an MPX_matrix file
through cmps_mpx_store / cmps_mpx_stat / cmps_mpx_load."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "chainamps_b200", "libchainamps_b200.so")


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not installed")
def test_c99_client_round_trips_an_mpx_file(tmp_path):
    if not os.path.exists(LIB):
        pytest.fail("libchainamps_b200.so is not built")
    exe = tmp_path / "mpx_roundtrip"
    src = os.path.join(ROOT, "tests", "abi", "mpx_roundtrip.c")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), src,
                    LIB, "-Wl,-rpath," + os.path.dirname(LIB), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), str(tmp_path / "m.MPX_matrix")], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    assert r.stdout.startswith("ok ")
