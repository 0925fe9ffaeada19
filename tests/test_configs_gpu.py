"""The benchmark configurations that are parity cases, through the C ABI.

* Plain iDMRG on the spin-1/2 XXZ chain (Jxy = Jz = 1, h = 0, MPO D = 11),
  chi = 100, 20 growth steps: the device run in FP64 and in mixed precision
  against the oracle's rows in ``tests/golden/oracle_configs.json`` (made by
  ``tests/golden/make_oracle_fixtures.py``).  Energies 1e-9 relative (the
  accuracy target), entropies 1e-7, truncation weights 1e-12 absolute or
  1e-4 relative, fidelities 1e-7, kept bond dimension exact.
* The synthetic charge-sector matvec: 40 bond sectors of uneven sizes drawn
  log-uniform from a seed, no physical charges, MPO bond dimension 16,
  complex Gaussian environments and MPO.  The configuration's sizes (local
  dimension 64, sector dimensions up to 512) need a 30 GB wavefunction and a
  ~0.5 TB intermediate in this contraction order; the test keeps its shape at
  local dimension 4 and sector dimensions 8..64 so that the oracle's block
  matvec runs in seconds.  FP64 within 1e-12 of the oracle (max-norm,
  relative to the largest entry).  Split-TF32 within 3e-4 max-norm and 1e-4
  rms: its K reaches ~4e3 terms (all 16 MPO slots dense), the regime of the
  chi = 512 benchmark matvec, where FP32 accumulation in the tensor cores
  sets the error (measured on B200: 4.9e-5 max-norm)."""
import json
import os

import numpy as np
import pytest

from oracle import blocks as ob
from tests.helpers import to_tensor

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "oracle_configs.json")


@pytest.fixture(scope="module")
def ctx():
    from chainamps_b200 import Context
    c = Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_xxz_idmrg_chi100_matches_oracle(ctx, precision):
    from chainamps_b200 import iDMRG, CMPS_FP64, CMPS_SPLIT_TF32
    from oracle import model as om
    ref = json.load(open(GOLD))["xxz_idmrg_chi100"]
    H = om.make_general_hmpo(om.spin_half_vertex(), om.xxz_couplings(1.0, 1.0, 0.0))
    prec = CMPS_FP64 if precision == "fp64" else CMPS_SPLIT_TF32
    run = iDMRG(ctx, H.rules, to_tensor(H), precision=prec, tol=1e-12, krylov_dim=32)
    for step, e in enumerate(ref["rows"]):
        r = run.grow(ref["chi"], ref["trunc"])
        assert r["chi"] == e["chi"], (step, r, e)
        assert abs(r["energy"] - e["energy"]) <= 1e-9 * abs(e["energy"]), (step, r, e)
        assert abs(r["entropy"] - e["entropy"]) <= 1e-7, (step, r, e)
        assert abs(r["truncation"] - e["truncation"]) <= max(1e-12, 1e-4 * e["truncation"]), (step, r, e)
        assert abs(r["fidelity"] - e["fidelity"]) <= 1e-7, (step, r, e)
    run.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed", "mixed_bf16"])
def test_coupled_ising_idmrg_matches_oracle(ctx, precision):
    """The benchmarked coupled-chain model: coupled transverse-field Ising
    chains, each vertex the periodic 12-site chain at g = 1.2 cut to its 64
    lowest states (Z2 parity), J_perp = 0.05 sum_i X_i X_i, MPO D = 26;
    iDMRG at chi = 32 for 5 steps against the oracle's rows (canonical-order
    block port; ``coupled_ising_12x64_chi32`` in oracle_configs.json).  The
    device takes the canonical contraction order for this vertex: in FP32
    under split TF32, on tcgen05 under split BF16.  Energies
    1e-9 relative, entropies 1e-8, kept bond dimension exact, truncation
    weights 1e-12 absolute or 1e-4 relative, fidelities 1e-7, kept singular
    values 1e-7."""
    from chainamps_b200 import iDMRG, CMPS_FP64, CMPS_SPLIT_TF32, CMPS_SPLIT_BF16
    from tests.helpers import ising_mpo
    ref = json.load(open(GOLD))["coupled_ising_12x64_chi32"]
    H = ising_mpo(12, 64)
    prec = {"fp64": CMPS_FP64, "mixed": CMPS_SPLIT_TF32, "mixed_bf16": CMPS_SPLIT_BF16}[precision]
    run = iDMRG(ctx, H.rules, to_tensor(H), precision=prec, tol=1e-12, krylov_dim=32)
    for step, e in enumerate(ref["rows"]):
        r = run.grow(ref["chi"], ref["trunc"])
        assert r["chi"] == e["chi"], (step, r, e)
        assert abs(r["energy"] - e["energy"]) <= 1e-9 * abs(e["energy"]), (step, r, e)
        assert abs(r["entropy"] - e["entropy"]) <= 1e-8, (step, r, e)
        assert abs(r["truncation"] - e["truncation"]) <= max(1e-12, 1e-4 * e["truncation"]), (step, r, e)
        assert abs(r["fidelity"] - e["fidelity"]) <= 1e-7, (step, r, e)
        np.testing.assert_allclose(run.values(), e["values"], rtol=1e-7, atol=1e-10)
    run.close()


def synthetic_sectors(seed=20261203, nsec=40, lo=8, hi=64):
    """Bond charges 0..nsec-1 with left / right sector dimensions drawn
    log-uniform in [lo, hi] from the seed."""
    rng = np.random.default_rng(seed)
    ls = np.round(np.exp(rng.uniform(np.log(lo), np.log(hi), nsec))).astype(int)
    rs = np.round(np.exp(rng.uniform(np.log(lo), np.log(hi), nsec))).astype(int)
    bl = np.concatenate([np.full(n, s) for s, n in enumerate(ls)]).reshape(-1, 1)
    br = np.concatenate([np.full(n, s) for s, n in enumerate(rs)]).reshape(-1, 1)
    return rng, bl, br


def env_mats(t, chi, D):
    M = np.zeros((chi, D * chi), np.complex128)
    cols = np.repeat(np.arange(t.cols), np.diff(t.colptr))
    M[t.rowind, cols] = t.values
    T = M.reshape(chi, D, chi, order="F")
    return [T[:, b, :] if np.any(T[:, b, :]) else None for b in range(D)]


def test_synthetic_sector_matvec_matches_oracle(ctx):
    from chainamps_b200 import TwoVertexComponents, CMPS_FP64, CMPS_SPLIT_TF32, models
    d, D = 4, 16
    rng, bl, br = synthetic_sectors()
    rules = (0,)                                     # Z charge on the bonds only
    ch = np.zeros((d, 1), np.int64)
    bq = np.zeros((D, 1), np.int64)
    W = (rng.standard_normal((d, D, d, D)) + 1j * rng.standard_normal((d, D, d, D))) / np.sqrt(2)
    L = models.random_environment(rng, rules, bl, bq, list(range(D)), right=False)
    R = models.random_environment(rng, rules, br, bq, list(range(D)), right=True)
    Wt = models.mpo_tensor(ch, W, bq)
    bh = ob.BlockHeff(rules, ch, bl, br, bq, W, env_mats(L, bl.shape[0], D), env_mats(R, br.shape[0], D))
    x = rng.standard_normal(bh.n) + 1j * rng.standard_normal(bh.n)
    want = bh.matvec(x)
    scale = np.max(np.abs(want))
    g64 = TwoVertexComponents(ctx, rules, L, Wt, R, precision=CMPS_FP64)
    assert g64.n == bh.n
    assert np.max(np.abs(g64.multiply(x) - want)) <= 1e-12 * scale
    del g64
    g32 = TwoVertexComponents(ctx, rules, L, Wt, R, precision=CMPS_SPLIT_TF32)
    err = g32.multiply(x) - want
    rms = np.sqrt(np.mean(np.abs(err) ** 2) / np.mean(np.abs(want) ** 2))
    assert np.max(np.abs(err)) <= 3e-4 * scale, np.max(np.abs(err)) / scale
    assert rms <= 1e-4, rms
