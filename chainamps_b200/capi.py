"""ctypes binding of the chainamps_b200 C ABI (include/chainamps_b200.h).

The host-side mirror of the reference's call surface for the DMRG hot path:

* ``TwoVertexComponents`` -- the reference class of the same name
  (DMRG_routines.hpp:189-214): built from the left block, the MPO and the
  right block; ``multiply`` is ``TwoVertexMPOMPSMultiply``
  (DMRG_routines.hpp:248), ``HED`` the lowest eigenpair
  (DMRG_routines.cpp:835-896);
* ``TwoVertexComponents.SVD`` -- ``TwoVertexSVD`` / ``MPX_matrix::SVD``
  (DMRG_routines.hpp:225, MPX_matrix.cpp:157-192);
* ``make_left_block`` / ``make_right_block`` -- ``MakeLeftBlock`` /
  ``MakeRightBlock`` (DMRG_routines.hpp:238-239).

Tensors cross the boundary as ``MPXTensor``: the reference's MPX_matrix
storage (directed charge-labelled indices plus one CSC matrix, first index
fastest).  Errors raise ``CmpsError`` with the library's message, the
counterpart of the reference printing and exiting.  There is no CPU
fallback: if the CUDA library is missing, importing this module fails.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libchainamps_b200.so")

CMPS_FP64 = 0
CMPS_SPLIT_TF32 = 1
CMPS_SPLIT_BF16 = 2
CMPS_ORDER_AUTO = 0
CMPS_ORDER_FOLDED = 1
CMPS_ORDER_CANONICAL = 2
CMPS_FORM_NONE = 0
CMPS_FORM_FOLDED_TC = 1
CMPS_FORM_CANONICAL_FP32 = 2
CMPS_FORM_CANONICAL_TC = 3


class CmpsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"chainamps_b200 error {code}: {msg}")
        self.code = code


def _load():
    if not os.path.exists(LIBPATH):
        raise ImportError(f"{LIBPATH} is not built: run `python -m chainamps_b200.build` "
                          "(the CUDA library is required; there is no CPU fallback)")
    return C.CDLL(LIBPATH)


lib = _load()

c_i64p = C.POINTER(C.c_int64)
c_dblp = C.POINTER(C.c_double)


class ChargeRules(C.Structure):
    _fields_ = [("nq", C.c_int32), ("rules", C.POINTER(C.c_int16))]


class MpxDesc(C.Structure):
    _fields_ = [("num_indices", C.c_int32), ("num_row_indices", C.c_int32),
                ("inward", C.POINTER(C.c_uint8)), ("physical", C.POINTER(C.c_uint8)),
                ("sizes", c_i64p), ("charges", C.POINTER(C.c_int16)),
                ("rows", C.c_int64), ("cols", C.c_int64),
                ("colptr", c_i64p), ("rowind", c_i64p), ("values", c_dblp)]


_SIGS = {
    "cmps_context_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "cmps_context_destroy": (C.c_int, [C.c_void_p]),
    "cmps_context_reserve": (C.c_int, [C.c_void_p, C.c_uint64]),
    "cmps_last_error": (C.c_char_p, []),
    "cmps_version": (C.c_char_p, []),
    "cmps_heff_create": (C.c_int, [C.c_void_p, C.POINTER(ChargeRules), C.POINTER(MpxDesc), C.POINTER(MpxDesc),
                                   C.POINTER(MpxDesc), C.c_int, C.POINTER(C.c_void_p)]),
    "cmps_heff_create_from_blocks": (C.c_int, [C.c_void_p, C.POINTER(ChargeRules), C.c_void_p, C.POINTER(MpxDesc),
                                               C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "cmps_block_create": (C.c_int, [C.c_void_p, C.POINTER(ChargeRules), C.POINTER(MpxDesc), C.POINTER(MpxDesc),
                                    C.c_int, C.POINTER(C.c_void_p)]),
    "cmps_heff_destroy": (C.c_int, [C.c_void_p]),
    "cmps_heff_length": (C.c_int, [C.c_void_p, c_i64p, c_i64p]),
    "cmps_heff_allowed_indices": (C.c_int, [C.c_void_p, c_i64p]),
    "cmps_heff_apply": (C.c_int, [C.c_void_p, c_dblp, c_dblp]),
    "cmps_heff_apply_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "cmps_heff_flops": (C.c_int, [C.c_void_p, c_dblp, c_dblp]),
    "cmps_heff_apply_device_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "cmps_heff_time_stages": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, c_dblp]),
    "cmps_heff_set_precision": (C.c_int, [C.c_void_p, C.c_int]),
    "cmps_heff_set_order": (C.c_int, [C.c_void_p, C.c_int]),
    "cmps_heff_order": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), c_dblp, c_dblp]),
    "cmps_heff_split_form": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "cmps_heff_status": (C.c_int, [C.c_void_p]),
    "cmps_heff_eigs": (C.c_int, [C.c_void_p, c_dblp, C.c_double, C.c_int, C.c_int, c_dblp, c_dblp,
                                 C.POINTER(C.c_int)]),
    "cmps_heff_eigs_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                       c_dblp]),
    "cmps_heff_set_theta": (C.c_int, [C.c_void_p, c_dblp]),
    "cmps_heff_theta_svd": (C.c_int, [C.c_void_p, C.c_int64, C.c_double, C.POINTER(C.c_void_p)]),
    "cmps_svd_destroy": (C.c_int, [C.c_void_p]),
    "cmps_svd_info": (C.c_int, [C.c_void_p, c_i64p, c_dblp, c_i64p, c_i64p]),
    "cmps_svd_routes": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "cmps_svd_copy": (C.c_int, [C.c_void_p, c_dblp, C.POINTER(C.c_int16), c_i64p, c_i64p, c_dblp, c_i64p, c_i64p,
                                c_dblp]),
    "cmps_heff_left_block": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]),
    "cmps_heff_right_block": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]),
    "cmps_block_destroy": (C.c_int, [C.c_void_p]),
    "cmps_block_info": (C.c_int, [C.c_void_p, c_i64p, c_i64p, c_i64p]),
    "cmps_block_copy": (C.c_int, [C.c_void_p, C.POINTER(C.c_int16), c_i64p, c_i64p, c_dblp]),
    "cmps_dmrg_create": (C.c_int, [C.c_void_p, C.POINTER(ChargeRules), C.POINTER(MpxDesc), C.POINTER(C.c_int16),
                                   C.c_int, C.POINTER(C.c_void_p)]),
    "cmps_dmrg_destroy": (C.c_int, [C.c_void_p]),
    "cmps_dmrg_set_solver": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.c_int]),
    "cmps_dmrg_grow": (C.c_int, [C.c_void_p, C.c_int64, C.c_double, c_dblp, c_i64p, C.POINTER(C.c_int), c_dblp]),
    "cmps_dmrg_values": (C.c_int, [C.c_void_p, c_dblp]),
    "cmps_dmrg_profile": (C.c_int, [C.c_void_p, c_dblp, C.c_int]),
    "cmps_dmrg_keep_blocks": (C.c_int, [C.c_void_p, C.c_int]),
    "cmps_dmrg_set_fidelity": (C.c_int, [C.c_void_p, C.c_int]),
    "cmps_dmrg_set_order": (C.c_int, [C.c_void_p, C.c_int]),
    "cmps_dmrg_move": (C.c_int, [C.c_void_p, C.c_int, C.c_int64, C.c_double, c_dblp, c_i64p, C.POINTER(C.c_int),
                                 c_dblp]),
    "cmps_dmrg_position": (C.c_int, [C.c_void_p, c_i64p, c_i64p]),
    "cmps_dmrg_project_state": (C.c_int, [C.c_void_p, C.c_double]),
    "cmps_dmrg_projected_states": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "cmps_dmrg_solve": (C.c_int, [C.c_void_p, C.c_int64, C.c_double, c_dblp, c_i64p, C.POINTER(C.c_int), c_dblp]),
    "cmps_dmrg_projector": (C.c_int, [C.c_void_p, C.c_int, c_dblp]),
    "cmps_dmrg_window_length": (C.c_int, [C.c_void_p, c_i64p, c_i64p]),
    "cmps_heff_adjoint": (C.c_int, [C.c_void_p, C.POINTER(MpxDesc), C.c_void_p, C.c_void_p, c_dblp]),
    "cmps_dmrg_set_gradient": (C.c_int, [C.c_void_p, C.POINTER(MpxDesc)]),
    "cmps_dmrg_gradient": (C.c_int, [C.c_void_p, c_dblp]),
    "cmps_dmrg_unit_cell": (C.c_int, [C.c_void_p, C.c_double, C.c_int, c_dblp]),
    "cmps_heff_set_projectors": (C.c_int, [C.c_void_p, C.c_int, c_dblp, c_dblp]),
    "cmps_heff_sector_table": (C.c_int, [C.c_void_p, c_i64p, c_i64p, c_dblp]),
    "cmps_heff_set_owned": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint8)]),
    "cmps_heff_input_sectors": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint8)]),
    "cmps_heff_autotune": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), c_dblp, c_dblp]),
    "cmps_dmrg_set_autotune": (C.c_int, [C.c_void_p, C.c_int]),
    "cmps_dmrg_autotune_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), c_dblp, c_dblp]),
    "cmps_heff_set_windows": (C.c_int, [C.c_void_p, c_i64p, C.c_int64, c_i64p, C.c_int64]),
    "cmps_heff_apply_theta_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "cmps_heff_theta_from_arpack": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "cmps_heff_theta_to_arpack": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "cmps_mpx_store": (C.c_int, [C.POINTER(MpxDesc), C.c_int32, C.c_char_p]),
    "cmps_mpx_stat": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32), c_i64p, c_i64p,
                                c_i64p, c_i64p]),
    "cmps_mpx_load": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(C.c_int16), C.c_int64, C.POINTER(C.c_uint8),
                                C.POINTER(C.c_uint8), c_i64p, C.POINTER(C.c_int16), c_i64p, c_i64p, c_dblp]),
}

for _name, (_res, _args) in _SIGS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


def exported_symbols():
    return list(_SIGS)


def _check(code):
    if code != 0:
        raise CmpsError(code, lib.cmps_last_error().decode())


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


# ---------------------------------------------------------------------------
# the tensor containers are numpy-only (chainamps_b200.tensors); re-exported here
from .tensors import MPXIndexSpec, MPXTensor  # noqa: E402,F401


def _rules(rules):
    r = np.ascontiguousarray(np.asarray(rules, np.int16))
    return ChargeRules(len(r), _p(r, C.c_int16)), r


class Context:
    def __init__(self, device=0):
        h = C.c_void_p()
        _check(lib.cmps_context_create(device, C.byref(h)))
        self.h = h

    def reserve(self, nbytes):
        """Map `nbytes` of device memory into the library's pool up front
        (0: return the pool's unused memory); see cmps_context_reserve."""
        _check(lib.cmps_context_reserve(self.h, int(nbytes)))

    def close(self):
        if self.h:
            lib.cmps_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TwoVertexComponents:
    """TwoVertexComponents (DMRG_routines.hpp:189-214) on the GPU."""

    def __init__(self, ctx: Context, rules, L, W: MPXTensor, R, precision=CMPS_FP64):
        """L and R: MPXTensor (host, reference layout) or Block (device)."""
        self.ctx = ctx
        cr, self._r = _rules(rules)
        dw, kw = W._desc()
        h = C.c_void_p()
        if isinstance(L, Block) and isinstance(R, Block):
            _check(lib.cmps_heff_create_from_blocks(ctx.h, C.byref(cr), L.h, C.byref(dw), R.h, precision,
                                                    C.byref(h)))
        else:
            dl, kl = L._desc()
            dr, kr = R._desc()
            _check(lib.cmps_heff_create(ctx.h, C.byref(cr), C.byref(dl), C.byref(dw), C.byref(dr), precision,
                                        C.byref(h)))
        self.h = h
        self.nq = len(self._r)
        n = C.c_int64()
        full = C.c_int64()
        _check(lib.cmps_heff_length(h, C.byref(n), C.byref(full)))
        self.n = n.value
        self.full_length = full.value

    def close(self):
        if getattr(self, "h", None):
            lib.cmps_heff_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def length(self):
        return self.full_length

    @property
    def allowed_indices(self):
        out = np.zeros(self.n, np.int64)
        _check(lib.cmps_heff_allowed_indices(self.h, _p(out, C.c_int64)))
        return out

    def multiply(self, x, out=None):
        """TwoVertexMPOMPSMultiply: host vector in ARPACK order -> host vector
        (written into ``out`` when given, e.g. a pinned buffer)."""
        x = np.ascontiguousarray(np.asarray(x, np.complex128))
        if x.shape != (self.n,):
            raise ValueError("vector length differs from allowed_indices.size()")
        if out is None:
            out = np.empty_like(x)
        elif out.shape != x.shape or out.dtype != np.complex128 or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous complex128 vector of the same length")
        _check(lib.cmps_heff_apply(self.h, _p(x.view(np.float64), C.c_double), _p(out.view(np.float64), C.c_double)))
        return out

    def multiply_device(self, d_in, d_out, stream=None):
        """Device pointers (ints) to n complex doubles each."""
        _check(lib.cmps_heff_apply_device(self.h, C.c_void_p(d_in), C.c_void_p(d_out),
                                          C.c_void_p(stream) if stream else None))

    def set_projectors(self, tensors, weights):
        """ProjectorTensors: every application of H_eff adds
        sum_p w_p (P_p . x) conj(P_p) (DMRG_routines.cpp:947-973).  tensors:
        vectors of length n in ARPACK order; an empty list removes them."""
        P = np.ascontiguousarray(np.asarray(tensors, np.complex128).reshape(-1, self.n)) if len(tensors) else \
            np.zeros((0, self.n), np.complex128)
        w = np.ascontiguousarray(np.asarray(weights, np.float64).reshape(-1))
        if w.size != P.shape[0]:
            raise ValueError("one weight per projector tensor")
        pv = P.view(np.float64) if P.size else np.zeros(2, np.float64)
        wv = w if w.size else np.zeros(1, np.float64)
        _check(lib.cmps_heff_set_projectors(self.h, P.shape[0], _p(pv, C.c_double), _p(wv, C.c_double)))

    def sector_table(self):
        """theta layout: (offsets[n_sectors + 1], flops[n_sectors]); output
        sector m occupies elements offsets[m]:offsets[m + 1] of each plane."""
        n = C.c_int64(0)
        _check(lib.cmps_heff_sector_table(self.h, C.byref(n), None, None))
        off = np.zeros(n.value + 1, np.int64)
        fl = np.zeros(max(1, n.value), np.float64)
        _check(lib.cmps_heff_sector_table(self.h, C.byref(n), _p(off, C.c_int64), _p(fl, C.c_double)))
        return off, fl[:n.value]

    def set_owned(self, owned):
        """Compute only the output sectors with owned[m] true (sharded matvec)."""
        mask = np.ascontiguousarray(np.asarray(owned, bool).astype(np.uint8))
        _check(lib.cmps_heff_set_owned(self.h, _p(mask, C.c_uint8)))

    def autotune(self):
        """Measured tile shapes of the matvec's grouped GEMM plans; returns
        dict(tuned, cached, ms_heuristic, ms_best) (cmps_heff_autotune)."""
        t, c = C.c_int(), C.c_int()
        a, b = C.c_double(), C.c_double()
        _check(lib.cmps_heff_autotune(self.h, C.byref(t), C.byref(c), C.byref(a), C.byref(b)))
        return dict(tuned=t.value, cached=c.value, ms_heuristic=a.value, ms_best=b.value)

    def input_sectors(self):
        """Mask of the input sectors the owned output sectors read."""
        n = len(self.sector_table()[1])
        out = np.zeros(max(n, 1), np.uint8)
        _check(lib.cmps_heff_input_sectors(self.h, _p(out, C.c_uint8)))
        return out[:n].astype(bool)

    def set_windows(self, in_base, in_len, out_base, out_len):
        """Vector windows of the theta-layout matvec (see cmps_heff_set_windows)."""
        ib = np.ascontiguousarray(np.asarray(in_base, np.int64))
        ob = np.ascontiguousarray(np.asarray(out_base, np.int64))
        _check(lib.cmps_heff_set_windows(self.h, _p(ib, C.c_int64), int(in_len), _p(ob, C.c_int64), int(out_len)))

    def multiply_theta_device(self, d_in, d_out, stream=None):
        """theta-layout matvec on device pointers (planar; the windows' lengths
        when set, else 2 * total doubles each)."""
        _check(lib.cmps_heff_apply_theta_device(self.h, C.c_void_p(d_in), C.c_void_p(d_out),
                                                C.c_void_p(stream) if stream else None))

    def theta_from_arpack_device(self, d_arpack, d_theta, stream=None):
        _check(lib.cmps_heff_theta_from_arpack(self.h, C.c_void_p(d_arpack), C.c_void_p(d_theta),
                                               C.c_void_p(stream) if stream else None))

    def theta_to_arpack_device(self, d_theta, d_arpack, stream=None):
        _check(lib.cmps_heff_theta_to_arpack(self.h, C.c_void_p(d_theta), C.c_void_p(d_arpack),
                                             C.c_void_p(stream) if stream else None))

    def time_stages(self, d_in, d_out, stream=None, reps=3):
        """Average ms of [gather, stage 1, stage 2, scatter] (CUDA events)."""
        ms = np.zeros(4, np.float64)
        _check(lib.cmps_heff_time_stages(self.h, C.c_void_p(d_in), C.c_void_p(d_out),
                                         C.c_void_p(stream) if stream else None, reps, _p(ms, C.c_double)))
        return ms

    def flops(self):
        a = C.c_double()
        b = C.c_double()
        _check(lib.cmps_heff_flops(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def status(self):
        """Raise if a device kernel recorded an asynchronous failure."""
        _check(lib.cmps_heff_status(self.h))

    def set_precision(self, p):
        _check(lib.cmps_heff_set_precision(self.h, p))

    def set_order(self, order):
        """Contraction order of the FP64 matvec: CMPS_ORDER_AUTO, _FOLDED or
        _CANONICAL."""
        _check(lib.cmps_heff_set_order(self.h, order))

    def order(self):
        """(order in use, executed flops folded, executed flops canonical)."""
        a = C.c_int()
        f = C.c_double()
        c = C.c_double()
        _check(lib.cmps_heff_order(self.h, C.byref(a), C.byref(f), C.byref(c)))
        return a.value, f.value, c.value

    def split_form(self):
        """Form of the split operator the precision runs (CMPS_FORM_*)."""
        f = C.c_int()
        _check(lib.cmps_heff_split_form(self.h, C.byref(f)))
        return f.value

    def HED(self, guess=None, tol=1e-10, max_restarts=50, krylov_dim=24, want_vector=True):
        """Lowest eigenpair; returns (energy, eigenvector in ARPACK order or
        None, matvec count)."""
        g = None
        if guess is not None:
            g = np.ascontiguousarray(np.asarray(guess, np.complex128))
        ev = C.c_double()
        mv = C.c_int()
        vec = np.empty(self.n, np.complex128) if want_vector else None
        _check(lib.cmps_heff_eigs(self.h, None if g is None else _p(g.view(np.float64), C.c_double), tol,
                                  max_restarts, krylov_dim, C.byref(ev),
                                  None if vec is None else _p(vec.view(np.float64), C.c_double), C.byref(mv)))
        return ev.value, vec, mv.value

    def eigs_stats(self):
        """Work of the last HED: dict(split_matvecs, fp64_matvecs, cycles,
        ms_split, ms_fp64, ms_total) (device time, CUDA events)."""
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        ms = np.zeros(3, np.float64)
        _check(lib.cmps_heff_eigs_stats(self.h, C.byref(a), C.byref(b), C.byref(c), _p(ms, C.c_double)))
        return dict(split_matvecs=a.value, fp64_matvecs=b.value, cycles=c.value, ms_split=ms[0], ms_fp64=ms[1],
                    ms_total=ms[2])

    def set_theta(self, theta):
        t = np.ascontiguousarray(np.asarray(theta, np.complex128))
        _check(lib.cmps_heff_set_theta(self.h, _p(t.view(np.float64), C.c_double)))

    def SVD(self, chi=0, max_trunc=0.0):
        s = C.c_void_p()
        _check(lib.cmps_heff_theta_svd(self.h, chi, max_trunc, C.byref(s)))
        return SVDResult(s, self.nq)

    def adjoint(self, dW: MPXTensor, dL: "Block" = None, dR: "Block" = None):
        """dE/dlambda = Re <theta|dH_eff|theta> / <theta|theta> for W = W0 +
        lambda dW, with optional environment derivatives dL / dR."""
        d, keep = dW._desc()
        g = C.c_double()
        _check(lib.cmps_heff_adjoint(self.h, C.byref(d), dL.h if dL is not None else None,
                                     dR.h if dR is not None else None, C.byref(g)))
        return g.value

    def make_left_block(self, svd: "SVDResult"):
        b = C.c_void_p()
        _check(lib.cmps_heff_left_block(self.h, svd.h, C.byref(b)))
        return Block(b, self.nq)

    def make_right_block(self, svd: "SVDResult"):
        b = C.c_void_p()
        _check(lib.cmps_heff_right_block(self.h, svd.h, C.byref(b)))
        return Block(b, self.nq)


class SVDResult:
    def __init__(self, h, nq):
        self.h = h
        self.nq = nq
        kept = C.c_int64()
        disc = C.c_double()
        nu = C.c_int64()
        nv = C.c_int64()
        _check(lib.cmps_svd_info(h, C.byref(kept), C.byref(disc), C.byref(nu), C.byref(nv)))
        self.kept = kept.value
        self.discarded = disc.value
        self._nu, self._nv = nu.value, nv.value

    def routes(self):
        """Sectors factored by each route: dict(exact, gram, randomized)."""
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        _check(lib.cmps_svd_routes(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return dict(exact=a.value, gram=b.value, randomized=c.value)

    def copy(self, u_rows, vd_cols):
        k = self.kept
        vals = np.zeros(k, np.float64)
        ch = np.zeros((k, self.nq), np.int16)
        ucp = np.zeros(k + 1, np.int64)
        uri = np.zeros(max(1, self._nu), np.int64)
        uv = np.zeros(max(1, self._nu), np.complex128)
        vcp = np.zeros(vd_cols + 1, np.int64)
        vri = np.zeros(max(1, self._nv), np.int64)
        vv = np.zeros(max(1, self._nv), np.complex128)
        _check(lib.cmps_svd_copy(self.h, _p(vals, C.c_double), _p(ch, C.c_int16), _p(ucp, C.c_int64),
                                 _p(uri, C.c_int64), _p(uv.view(np.float64), C.c_double), _p(vcp, C.c_int64),
                                 _p(vri, C.c_int64), _p(vv.view(np.float64), C.c_double)))
        nu, nv = ucp[-1], vcp[-1]
        return dict(values=vals, charges=ch.astype(np.int64), u=(ucp, uri[:nu], uv[:nu]),
                    vd=(vcp, vri[:nv], vv[:nv]))

    def store(self, name, nl, nr, basis_charges, a0_charges, a2_charges, store_lambda=True):
        """MPSDecomposition::store (MPS_matrix.cpp:151-165): <name>_Left_<nl>
        and <name>_Right_<nr>.MPS_matrix, and <name>_Lambda_<nl>_<nr>
        .MPX_matrix if store_lambda.  basis_charges: the vertex basis (d, nq);
        a0 / a2: the charges of the left / right environment bonds."""
        d = np.asarray(basis_charges).reshape(-1, self.nq).shape[0]
        out = self.copy(d * len(a0_charges), d * len(a2_charges))
        U, Vd, Lam = mps_decomposition_tensors(out, basis_charges, a0_charges, a2_charges)
        store_mpx(U, self.nq, f"{name}_Left_{nl}.MPS_matrix")
        store_mpx(Vd, self.nq, f"{name}_Right_{nr}.MPS_matrix")
        if store_lambda:
            store_mpx(Lam, self.nq, f"{name}_Lambda_{nl}_{nr}.MPX_matrix")

    def close(self):
        if getattr(self, "h", None):
            lib.cmps_svd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Block:
    """A new environment block kept on the device."""

    def __init__(self, h, nq):
        self.h = h
        self.nq = nq
        chi = C.c_int64()
        D = C.c_int64()
        nnz = C.c_int64()
        _check(lib.cmps_block_info(h, C.byref(chi), C.byref(D), C.byref(nnz)))
        self.chi, self.D, self._nnz = chi.value, D.value, nnz.value

    def to_csc(self):
        ch = np.zeros((self.chi, self.nq), np.int16)
        cp = np.zeros(self.D * self.chi + 1, np.int64)
        ri = np.zeros(max(1, self._nnz), np.int64)
        v = np.zeros(max(1, self._nnz), np.complex128)
        _check(lib.cmps_block_copy(self.h, _p(ch, C.c_int16), _p(cp, C.c_int64), _p(ri, C.c_int64),
                                   _p(v.view(np.float64), C.c_double)))
        n = cp[-1]
        return ch.astype(np.int64), (cp, ri[:n], v[:n])

    def to_mpx(self, bq, right, target=None) -> "MPXTensor":
        """The block as the reference's 6-index MPX_matrix (see
        block_mpx_tensor); bq: MPO bond charges (D, nq)."""
        ch, csc = self.to_csc()
        return block_mpx_tensor(ch, csc, self.D, bq, right, target)

    def store(self, path, bq, right, target=None):
        """BlocksStructure::save_left_block / save_right_block
        (DMRG_routines.cpp:65-84): write the block as a .BLOCK file."""
        store_mpx(self.to_mpx(bq, right, target), self.nq, path)

    def close(self):
        if getattr(self, "h", None):
            lib.cmps_block_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def block_mpx_tensor(charges, csc, D, bq, right, target=None) -> "MPXTensor":
    """An exported environment block (cmps_block_copy: a' charges, CSC of rows
    a', cols b + D a) as the 6-index MPX_matrix the reference holds:
    MakeLeftBlock's (dummy, a', dummy, b, dummy, a; 3 row indices) or
    MakeRightBlock's (a', dummy, b, dummy, a, dummy; 2 row indices)
    (DMRG_routines.cpp:594-611).  The matrix is the export itself: the dummy
    indices have size 1.  The right block's first and last dummies carry the
    target charge (from MakeDummyRightBlock, :634-653), every other dummy zero."""
    ch = np.asarray(charges, np.int64)
    nq = ch.shape[1]
    bq = np.asarray(bq, np.int64).reshape(-1, nq)
    if bq.shape[0] != D:
        raise ValueError("bq must have one charge per MPO bond state")
    z = np.zeros((1, nq), np.int64)
    t = z if target is None else np.asarray(target, np.int64).reshape(1, nq)
    if not right:
        idx = [MPXIndexSpec(False, False, z), MPXIndexSpec(True, False, ch), MPXIndexSpec(True, False, z),
               MPXIndexSpec(False, False, bq), MPXIndexSpec(True, False, z), MPXIndexSpec(False, False, ch)]
        nrow = 3
    else:
        idx = [MPXIndexSpec(False, False, ch), MPXIndexSpec(True, False, t), MPXIndexSpec(True, False, bq),
               MPXIndexSpec(False, False, z), MPXIndexSpec(True, False, ch), MPXIndexSpec(False, False, t)]
        nrow = 2
    cp, ri, v = csc
    chi = ch.shape[0]
    return MPXTensor(idx, nrow, chi, D * chi, np.asarray(cp, np.int64), np.asarray(ri, np.int64),
                     np.asarray(v, np.complex128))


class iDMRG:
    """Device-resident iDMRG growth (SuperBlock::grow_two_vertex,
    DMRG_routines.cpp:346-374; iDMRG::run, iDMRG_routines.cpp:19-33)."""

    def __init__(self, ctx: Context, rules, W: MPXTensor, target=None, precision=CMPS_FP64, tol=1e-10,
                 max_restarts=50, krylov_dim=24, gradient=None, order=CMPS_ORDER_AUTO, autotune=False):
        """gradient: optional dW (MPXTensor, the MPO's derivative with respect
        to one coupling); each grow() then also returns dE/dlambda.  order:
        contraction order of each step's H_eff (CMPS_ORDER_*).  autotune:
        measured tile shapes for each step's grouped GEMM plans."""
        self.ctx = ctx
        cr, self._r = _rules(rules)
        dw, kw = W._desc()
        t = None
        if target is not None:
            self._t = np.ascontiguousarray(np.asarray(target, np.int16))
            t = _p(self._t, C.c_int16)
        h = C.c_void_p()
        _check(lib.cmps_dmrg_create(ctx.h, C.byref(cr), C.byref(dw), t, precision, C.byref(h)))
        self.h = h
        _check(lib.cmps_dmrg_set_solver(h, tol, max_restarts, krylov_dim))
        _check(lib.cmps_dmrg_set_order(h, order))
        if autotune:
            _check(lib.cmps_dmrg_set_autotune(h, 1))
        self._grad = gradient is not None
        if self._grad:
            gd, gk = gradient._desc()
            _check(lib.cmps_dmrg_set_gradient(h, C.byref(gd)))
        self.last = None

    def grow(self, chi=0, max_trunc=0.0):
        """One step; returns dict(energy, energy_per, entropy, truncation,
        fidelity, chi, matvecs, ms=[env, eigensolve, svd, total])."""
        row = np.zeros(5, np.float64)
        bd = C.c_int64()
        mv = C.c_int()
        ms = np.zeros(4, np.float64)
        _check(lib.cmps_dmrg_grow(self.h, chi, max_trunc, _p(row, C.c_double), C.byref(bd), C.byref(mv),
                                  _p(ms, C.c_double)))
        self.last = dict(energy=row[0], energy_per=row[1], entropy=row[2], truncation=row[3], fidelity=row[4],
                         chi=bd.value, matvecs=mv.value, ms=ms)
        if self._grad:
            g = C.c_double()
            _check(lib.cmps_dmrg_gradient(self.h, C.byref(g)))
            self.last["gradient"] = g.value
        return self.last

    def autotune_stats(self):
        t, c = C.c_int(), C.c_int()
        a, b = C.c_double(), C.c_double()
        _check(lib.cmps_dmrg_autotune_stats(self.h, C.byref(t), C.byref(c), C.byref(a), C.byref(b)))
        return dict(tuned=t.value, cached=c.value, ms_heuristic=a.value, ms_best=b.value)

    def profile(self):
        """Breakdown of the last step: device times (CUDA events) of the
        environment update, H_eff build, eigensolve, SVD and whole step; the
        eigensolver's matvec counts and times; host wall times per phase."""
        keys = ("env_ms", "build_ms", "eig_ms", "svd_ms", "total_ms", "split_matvecs", "fp64_matvecs", "cycles",
                "split_mv_ms", "fp64_mv_ms", "host_env_ms", "host_build_ms", "host_split_ms", "host_predict_ms",
                "host_release_ms", "host_svd_ms", "host_total_ms", "svd_exact", "svd_gram", "svd_randomized",
                "order")
        ints = ("split_matvecs", "fp64_matvecs", "cycles", "svd_exact", "svd_gram", "svd_randomized", "order")
        v = np.zeros(len(keys), np.float64)
        _check(lib.cmps_dmrg_profile(self.h, _p(v, C.c_double), len(keys)))
        return {k: (int(x) if k in ints else float(x)) for k, x in zip(keys, v)}

    def values(self):
        v = np.zeros(self.last["chi"], np.float64)
        _check(lib.cmps_dmrg_values(self.h, _p(v, C.c_double)))
        return v

    def unit_cell(self, tol=1e-12, krylov_dim=30):
        """Orthogonalise + iTwoVertexEnergy of the last growth step
        (iDMRG_DRV.cpp:71-77): energy per vertex of the translation-invariant
        cell, entropy of its boundary values, the dominant transfer-matrix
        eigenvalues and the number of boundary values."""
        v = np.zeros(6, np.float64)
        _check(lib.cmps_dmrg_unit_cell(self.h, tol, krylov_dim, _p(v, C.c_double)))
        return dict(energy=float(v[0]), entropy=float(v[1]), eta_left=float(v[2]), eta_right=float(v[3]),
                    chi=int(v[4]), energy_imag=float(v[5]))

    def close(self):
        if getattr(self, "h", None):
            lib.cmps_dmrg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# the reference's default projector weight (command_line_input.hpp:470)
DEFAULT_PROJECTOR_WEIGHT = 100.0


def run_excited_fdmrg(ctx, rules, W, nvertices, sweeps, chi, max_trunc=1e-16, nstates=1,
                      weight=DEFAULT_PROJECTOR_WEIGHT, target=None, precision=CMPS_FP64, tol=1e-10, max_restarts=50,
                      krylov_dim=24):
    """fDMRG_DRV -X nstates (fDMRG_DRV.cpp:60-72) on the device: the ground
    state by finite DMRG, then each excited state by the same sweeps with
    every earlier state projected out.  Returns (ground-state rows, [rows of
    excited state 1, ...]) and the driver."""
    run = fDMRG(ctx, rules, W, nvertices, target, precision, tol, max_restarts, krylov_dim)
    gs = run.run(sweeps, chi, max_trunc)
    out = []
    for _ in range(nstates):
        run.project_state(weight)
        out.append(run.run_excited(sweeps, chi, max_trunc))
    return gs, out, run


class fDMRG(iDMRG):
    """Finite DMRG on the device: fDMRG_DRV's growth to `nvertices`, then
    FiniteDMRG::run's sweeps (fDMRG_routines.cpp:19-66) with every block kept
    in device memory."""

    def __init__(self, ctx: Context, rules, W: MPXTensor, nvertices, target=None, precision=CMPS_FP64, tol=1e-10,
                 max_restarts=50, krylov_dim=24, gradient=None):
        """gradient: optional dW, as for iDMRG; the gradient is then carried
        through the growth and every sweep step (derivative blocks kept
        beside the blocks) and each row gets dE/dlambda."""
        super().__init__(ctx, rules, W, target, precision, tol, max_restarts, krylov_dim, gradient=gradient)
        _check(lib.cmps_dmrg_keep_blocks(self.h, 1))
        self.nvertices = int(nvertices)

    def position(self):
        """(vertices left of the two-vertex window, chain length)."""
        nl, n = C.c_int64(), C.c_int64()
        _check(lib.cmps_dmrg_position(self.h, C.byref(nl), C.byref(n)))
        return nl.value, n.value

    def move(self, direction, chi=0, max_trunc=0.0):
        """One sweep step, +1 right / -1 left (move_{right,left}_two_vertex)."""
        row = np.zeros(5, np.float64)
        bd = C.c_int64()
        mv = C.c_int()
        ms = np.zeros(4, np.float64)
        _check(lib.cmps_dmrg_move(self.h, int(direction), chi, max_trunc, _p(row, C.c_double), C.byref(bd),
                                  C.byref(mv), _p(ms, C.c_double)))
        return self._row(row, bd, mv, ms)

    def _row(self, row, bd, mv, ms):
        self.last = dict(energy=row[0], energy_per=row[1], entropy=row[2], truncation=row[3], fidelity=row[4],
                         chi=bd.value, matvecs=mv.value, ms=ms)
        if self._grad:
            g = C.c_double()
            _check(lib.cmps_dmrg_gradient(self.h, C.byref(g)))
            self.last["gradient"] = g.value
        return self.last

    def solve(self, chi=0, max_trunc=0.0):
        """Solve the current window again with its environments, without
        moving (ExcitedStateFiniteDMRG::init, fDMRG_routines.cpp:68-91)."""
        row = np.zeros(5, np.float64)
        bd = C.c_int64()
        mv = C.c_int()
        ms = np.zeros(4, np.float64)
        _check(lib.cmps_dmrg_solve(self.h, chi, max_trunc, _p(row, C.c_double), C.byref(bd), C.byref(mv),
                                   _p(ms, C.c_double)))
        return self._row(row, bd, mv, ms)

    def project_state(self, weight=DEFAULT_PROJECTOR_WEIGHT):
        """Store the current state as a state to project out of every later
        solve, with weight `weight` (next_state, fDMRG_routines.hpp:39-44)."""
        _check(lib.cmps_dmrg_project_state(self.h, float(weight)))

    def projected_states(self):
        n = C.c_int()
        _check(lib.cmps_dmrg_projected_states(self.h, C.byref(n)))
        return n.value

    def window_length(self):
        """(allowed entries, full length) of the current window."""
        n, full = C.c_int64(), C.c_int64()
        _check(lib.cmps_dmrg_window_length(self.h, C.byref(n), C.byref(full)))
        return n.value, full.value

    def projector(self, index):
        """The current window's projector tensor P of stored state `index`
        (ARPACK order)."""
        out = np.zeros(2 * self.window_length()[0], np.float64)
        _check(lib.cmps_dmrg_projector(self.h, int(index), _p(out, C.c_double)))
        return out[0::2] + 1j * out[1::2]

    def _sweeps(self, sweeps, chi, max_trunc, rows):
        for _ in range(sweeps):
            nl, n = self.position()
            for _ in range(n - nl - 2):
                self.move(+1, chi, max_trunc)
            nl, n = self.position()
            for _ in range(nl):
                r = self.move(-1, chi, max_trunc)
                a, b = self.position()
                if a == b - a - 2:
                    rows.append(r)
            # back to the centre: for (r = right_size(); r > left_size(); --r)
            # reads the left size as it grows (fDMRG_routines.cpp:52-58)
            nl, n = self.position()
            while n - nl - 2 > nl:
                r = self.move(+1, chi, max_trunc)
                nl, n = self.position()
                if nl == n - nl - 2:
                    rows.append(r)
        return rows

    def run(self, sweeps, chi, max_trunc=1e-16):
        """Growth rows, then the rows written when the window passes the
        middle of the chain (twice per sweep): the rows of the energies file."""
        rows = [self.grow(chi, max_trunc) for _ in range(self.nvertices // 2)]
        nl, n = self.position()
        if n <= 2:
            return rows
        return self._sweeps(sweeps, chi, max_trunc, rows)

    def run_excited(self, sweeps, chi, max_trunc=1e-16):
        """ExcitedStateFiniteDMRG::run (fDMRG_routines.cpp:198-242) for the
        states stored so far: the init row (a solve at the current window),
        then the rows at the centre of every sweep."""
        return self._sweeps(sweeps, chi, max_trunc, [self.solve(chi, max_trunc)])


def upload_block(ctx: Context, rules, block: MPXTensor, W: MPXTensor, right: bool):
    """A reference-layout environment block (e.g. MakeDummyLeftBlock) as a
    device Block."""
    cr, r = _rules(rules)
    db, kb = block._desc()
    dw, kw = W._desc()
    h = C.c_void_p()
    _check(lib.cmps_block_create(ctx.h, C.byref(cr), C.byref(db), C.byref(dw), 1 if right else 0, C.byref(h)))
    return Block(h, len(r))


def mps_decomposition_tensors(svd_copy, basis_charges, a0_charges, a2_charges):
    """The MPSDecomposition of a device SVD (SVDResult.copy) as the reference
    holds it (MPX_matrix.cpp:174-191): LeftMatrix (sigma1 in, a0 in, a1 out;
    2 row indices), RightMatrix (a1 in, sigma2 in, a2 out; 1 row index) and
    the diagonal Lambda MPX_matrix(spectrum, LeftMatrix.Index(2), values)
    (a1 in, a1 out; MPX_matrix.cpp:55-60).  The physical indices carry the
    basis charges; the matrices are the copy's CSC arrays."""
    ch = np.asarray(svd_copy["charges"], np.int64)
    nq = ch.shape[1]
    basis = np.asarray(basis_charges, np.int64).reshape(-1, nq)
    a0 = np.asarray(a0_charges, np.int64).reshape(-1, nq)
    a2 = np.asarray(a2_charges, np.int64).reshape(-1, nq)
    d, k = basis.shape[0], ch.shape[0]
    ucp, uri, uv = svd_copy["u"]
    vcp, vri, vv = svd_copy["vd"]
    U = MPXTensor([MPXIndexSpec(True, True, basis), MPXIndexSpec(True, False, a0), MPXIndexSpec(False, False, ch)],
                  2, d * a0.shape[0], k, np.asarray(ucp, np.int64), np.asarray(uri, np.int64),
                  np.asarray(uv, np.complex128))
    Vd = MPXTensor([MPXIndexSpec(True, False, ch), MPXIndexSpec(True, True, basis), MPXIndexSpec(False, False, a2)],
                   1, k, d * a2.shape[0], np.asarray(vcp, np.int64), np.asarray(vri, np.int64),
                   np.asarray(vv, np.complex128))
    vals = np.asarray(svd_copy["values"], np.float64)
    Lam = MPXTensor([MPXIndexSpec(True, False, ch), MPXIndexSpec(False, False, ch)], 1, k, k,
                    np.arange(k + 1, dtype=np.int64), np.arange(k, dtype=np.int64), vals.astype(np.complex128))
    return U, Vd, Lam


def load_block(ctx: Context, rules, path, W: MPXTensor, right: bool):
    """BlocksStructure::load_left_block / load_right_block
    (DMRG_routines.cpp:89-101): a .BLOCK file (written by the reference or by
    Block.store) as a device Block."""
    return upload_block(ctx, rules, load_mpx(path, len(rules)), W, right)


def store_mpx(t: MPXTensor, nq: int, path):
    """Write t as the reference writes an MPX_matrix file (MPX_matrix::store):
    the .BLOCK / .MPS_matrix / .MPX_matrix format.  Host only."""
    d, keep = t._desc()
    _check(lib.cmps_mpx_store(C.byref(d), int(nq), os.fsencode(path)))


def load_mpx(path, nq: int, basis_charges=None) -> MPXTensor:
    """Read an MPX_matrix file (load_MPX_matrix).  basis_charges ((d, nq)
    int) gives the charges of physical indices, which the file does not
    store.  Host only."""
    p = os.fsencode(path)
    ni, nr = C.c_int32(), C.c_int32()
    tot, rows, cols, nnz = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
    _check(lib.cmps_mpx_stat(p, int(nq), C.byref(ni), C.byref(nr), C.byref(tot), C.byref(rows), C.byref(cols),
                             C.byref(nnz)))
    n = ni.value
    inward = np.zeros(max(n, 1), np.uint8)
    phys = np.zeros(max(n, 1), np.uint8)
    sizes = np.zeros(max(n, 1), np.int64)
    charges = np.zeros(max(tot.value * nq, 1), np.int16)
    colptr = np.zeros(cols.value + 1, np.int64)
    rowind = np.zeros(max(nnz.value, 1), np.int64)
    vals = np.zeros(max(nnz.value, 1), np.complex128)
    if basis_charges is None:
        bc, bsize = None, 0
    else:
        bc = np.ascontiguousarray(np.asarray(basis_charges, np.int16).reshape(-1, nq))
        bsize = bc.shape[0]
    _check(lib.cmps_mpx_load(p, int(nq), None if bc is None else _p(bc, C.c_int16), bsize, _p(inward, C.c_uint8),
                             _p(phys, C.c_uint8), _p(sizes, C.c_int64), _p(charges, C.c_int16), _p(colptr, C.c_int64),
                             _p(rowind, C.c_int64), _p(vals.view(np.float64), C.c_double)))
    idx, off = [], 0
    for i in range(n):
        sz = int(sizes[i])
        idx.append(MPXIndexSpec(bool(inward[i]), bool(phys[i]),
                                charges[off * nq:(off + sz) * nq].reshape(sz, nq).astype(np.int64)))
        off += sz
    k = nnz.value
    return MPXTensor(idx, nr.value, rows.value, cols.value, colptr, rowind[:k].copy(), vals[:k].copy())


def version():
    return lib.cmps_version().decode()
