"""The H_eff matvec that allocates nothing, for callers that cannot call
cudaMalloc while applying H_eff (an eigensolver callback inside an
application whose device memory belongs to its own pool allocator).

Called through the C ABI on device buffers; its result must equal the
handle-scratch entry point (cmps_heff_apply_device) within the tolerance
the other FP64 tests use (1e-12 relative, max-norm), on two calls in a row
with different inputs, since every call reuses the same static scratch.
Collected last on purpose; it also passes on its own in a fresh process."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _envs(H, chi_l, chi_r, seed):
    from tests.helpers import random_bond, random_left_block, random_right_block, charge_pool_for
    rng = np.random.default_rng(seed)
    pool = charge_pool_for(H)
    bq = H.indices[1].charges
    return (random_left_block(rng, H.rules, random_bond(rng, chi_l, pool), bq),
            random_right_block(rng, H.rules, random_bond(rng, chi_r, pool), bq))


def test_noalloc_matvec_matches_handle_scratch_matvec():
    import torch
    from chainamps_b200 import Context, TwoVertexComponents
    from chainamps_b200.capi import lib
    from tests.helpers import to_tensor, model_zoo

    H = model_zoo()["ladder4"]
    L, R = _envs(H, 9, 7, 31)
    ctx = Context(0)
    h = TwoVertexComponents(ctx, H.rules, to_tensor(L), to_tensor(H), to_tensor(R))
    n = h.n
    rng = np.random.default_rng(8)
    stream = torch.cuda.Stream()
    for call in range(2):
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        # the copy and the NaN fill run on torch's current stream; the matvecs
        # run on `stream`, a non-blocking stream, so order them explicitly
        dx = torch.from_numpy(x).cuda()
        want = torch.empty_like(dx)
        got = torch.full_like(dx, complex(np.nan, np.nan))
        stream.wait_stream(torch.cuda.current_stream())
        h.multiply_device(dx.data_ptr(), want.data_ptr(), stream.cuda_stream)
        rc = lib.cmps_heff_apply_device_noalloc(h.h, C.c_void_p(dx.data_ptr()), C.c_void_p(got.data_ptr()),
                                                C.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.cmps_last_error().decode()
        stream.synchronize()
        w, g = want.cpu().numpy(), got.cpu().numpy()
        assert np.all(np.isfinite(g)), f"call {call}: output not fully written"
        assert np.max(np.abs(g - w)) <= 1e-12 * np.max(np.abs(w)), f"call {call}"
    del h
    ctx.close()


def test_noalloc_matvec_rejects_problems_above_the_static_maximum():
    import torch
    from chainamps_b200 import Context, TwoVertexComponents
    from chainamps_b200.capi import lib
    from chainamps_b200 import models

    rules, ch, W, bq = models.ladder_model(4, 1.0, 0.5)
    used_l = sorted({int(b) for b in np.nonzero(np.any(W != 0, axis=(0, 2, 3)))[0]})
    used_r = sorted({int(b) for b in np.nonzero(np.any(W != 0, axis=(0, 1, 2)))[0]})
    bond = models.gaussian_bond(96)
    rng = np.random.default_rng(3)
    L = models.random_environment(rng, rules, bond, bq, used_l, right=False)
    R = models.random_environment(rng, rules, bond, bq, used_r, right=True)
    ctx = Context(0)
    h = TwoVertexComponents(ctx, rules, L, models.mpo_tensor(ch, W, bq), R)
    dx = torch.zeros(h.n, dtype=torch.complex128, device="cuda")
    dy = torch.zeros_like(dx)
    rc = lib.cmps_heff_apply_device_noalloc(h.h, C.c_void_p(dx.data_ptr()), C.c_void_p(dy.data_ptr()), None)
    assert rc == 1
    assert b"static maximum" in lib.cmps_last_error()
    del h
    ctx.close()
