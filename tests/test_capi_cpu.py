"""CPU-side checks of the C ABI library: it loads, exports every entry
point the header declares, and rejects bad arguments without a GPU."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "chainamps_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(cmps_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_header_symbol():
    from chainamps_b200 import capi
    names = header_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(capi.lib, n), n
    # the Python mirror binds every one of them
    assert set(names) <= set(capi.exported_symbols())


def test_version_and_arch():
    from chainamps_b200 import capi
    assert "sm_100a" in capi.version()


def test_null_arguments_are_errors_not_crashes():
    from chainamps_b200 import capi
    lib = capi.lib
    n = C.c_int64()
    assert lib.cmps_heff_length(None, C.byref(n), None) == 1      # CMPS_ERR_ARG
    assert lib.cmps_heff_apply(None, None, None) == 1
    assert lib.cmps_svd_info(None, None, None, None, None) == 1
    assert lib.cmps_block_info(None, None, None, None) == 1
    assert b"null" in lib.cmps_last_error()
    h = C.c_void_p()
    assert lib.cmps_context_create(-1, C.byref(h)) != 0
    assert not h.value


def test_library_is_sm100a_only():
    """The shared object carries sm_100a code (checked from the build recipe)."""
    from chainamps_b200 import build
    for src in build.sources():
        cmd, _ = build.nvcc_compile(src)
        assert "arch=compute_100a,code=sm_100a" in " ".join(cmd)
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.nvcc_link(["x.o"]))


def test_library_matches_its_sources():
    """The built library's stamp is the digest of the current sources and
    flags: a library built from other sources is not reused."""
    from chainamps_b200 import build
    assert build.up_to_date(), "libchainamps_b200.so is stale: run python -m chainamps_b200.build"
