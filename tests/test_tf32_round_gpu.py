"""The converter warps' integer TF32 rounding equals cvt.rna.tf32.f32 bit for
bit on 2^24 finite inputs (random patterns, exact ties, subnormals): the
check program is compiled from tests/cuda/tf32_round_check.cu against the
library's own header and run on the GPU."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "chainamps_b200", "csrc")


def test_integer_tf32_rounding_matches_cvt(tmp_path):
    from chainamps_b200.build import CUDA
    exe = str(tmp_path / "tf32_round_check")
    subprocess.run([os.path.join(CUDA, "bin", "nvcc"), "-gencode", "arch=compute_100a,code=sm_100a", "-O2",
                    "-I", CSRC, os.path.join(HERE, "cuda", "tf32_round_check.cu"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert " mismatches=0 " in r.stdout, r.stdout
