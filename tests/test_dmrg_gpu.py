"""The device-resident iDMRG growth (environment update -> H_eff ->
predicted start vector -> Lanczos -> block SVD, all on the GPU) against the
reference's own example output and against the oracle, step by step.

Tolerances: energies 1e-10 relative to the reference example (printed to
16 digits) and 1e-9 relative to the oracle; entropies 1e-8; kept bond
dimension exact; truncation weights 1e-12 absolute.  The split-TF32 form
must give the same energies as FP64 within 1e-9 relative."""
import json
import os

import numpy as np
import pytest

from oracle import dmrg as od
from oracle.model import parse_user_vertex, parse_couplings, make_general_hmpo
from tests.helpers import to_tensor, model_zoo

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "kat_examples.json")


@pytest.fixture(scope="module")
def ctx():
    from chainamps_b200 import Context
    c = Context(0)
    yield c
    c.close()


def test_device_growth_reproduces_spin_half_example(ctx):
    from chainamps_b200 import iDMRG
    k = json.load(open(GOLD))["spin_half_fdmrg"]
    v = parse_user_vertex(k["basis"], k["hamiltonian"], k["operators"])
    H = make_general_hmpo(v, parse_couplings(k["input"].splitlines()[2]))
    run = iDMRG(ctx, H.rules, to_tensor(H), tol=1e-12, krylov_dim=32)
    for row in k["energies"][:5]:        # growth rows: 2, 4, ..., 10 vertices
        r = run.grow(k["chi"], k["trunc"])
        assert abs(r["energy"] - row[1]) <= 1e-10 * abs(row[1]), (r, row)
        assert abs(r["entropy"] - row[3]) <= 1e-8, (r, row)
        assert abs(r["truncation"] - row[4]) <= 1e-12
        assert abs(r["fidelity"] - row[5]) <= 1e-10, (r, row)      # CheckConvergence


@pytest.mark.parametrize("name,chi,steps", [("xxz", 32, 10), ("tfim", 24, 5)])
def test_device_idmrg_matches_oracle(ctx, name, chi, steps):
    from chainamps_b200 import iDMRG
    H = model_zoo()[name]
    sb = od.SuperBlock(H)
    run = iDMRG(ctx, H.rules, to_tensor(H), tol=1e-12, krylov_dim=32)
    for _ in range(steps):
        ref = sb.grow(chi, 1e-16)
        got = run.grow(chi, 1e-16)
        assert got["chi"] == ref["chi"]
        assert abs(got["energy"] - ref["energy"]) <= 1e-9 * abs(ref["energy"]), (got, ref)
        assert abs(got["entropy"] - ref["entropy"]) <= 1e-8
        assert abs(got["truncation"] - ref["truncation"]) <= 1e-12
        assert abs(got["fidelity"] - ref["fidelity"]) <= 1e-9, (got, ref)
        np.testing.assert_allclose(run.values(), sb.dec.values, rtol=1e-7, atol=1e-10)


def test_split_precision_idmrg_energies(ctx):
    from chainamps_b200 import iDMRG, CMPS_SPLIT_TF32, CMPS_FP64
    H = model_zoo()["xxz"]
    a = iDMRG(ctx, H.rules, to_tensor(H), precision=CMPS_FP64, tol=1e-12, krylov_dim=32)
    b = iDMRG(ctx, H.rules, to_tensor(H), precision=CMPS_SPLIT_TF32, tol=1e-12, krylov_dim=32)
    for _ in range(10):
        ra = a.grow(40, 1e-16)
        rb = b.grow(40, 1e-16)
        assert abs(ra["energy"] - rb["energy"]) <= 1e-9 * abs(ra["energy"]), (ra, rb)
        assert ra["chi"] == rb["chi"]


def test_coupled_ising_idmrg_matches_oracle(ctx):
    """Coupled transverse-field Ising chains (each vertex a 4-site periodic
    chain cut to its 8 lowest states, Z2 parity only): device iDMRG in FP64
    and mixed precision against the oracle's SuperBlock, step by step."""
    from chainamps_b200 import iDMRG, CMPS_SPLIT_TF32, models
    from oracle import model as om
    ch, ops, Hv, _, _ = models.ising_chain_vertex(4, 1.2, 8)
    H = om.make_general_hmpo(om.Vertex((2,), ch, ops, Hv),
                             [om.Coupling(f"J{i}", f"X{i}", f"X{i}", 0.05) for i in range(4)])
    sb = od.SuperBlock(H)
    run = iDMRG(ctx, H.rules, to_tensor(H), tol=1e-12, krylov_dim=32)
    mixed = iDMRG(ctx, H.rules, to_tensor(H), precision=CMPS_SPLIT_TF32, tol=1e-12, krylov_dim=32)
    for _ in range(4):
        ref = sb.grow(24, 1e-16)
        got = run.grow(24, 1e-16)
        mx = mixed.grow(24, 1e-16)
        assert got["chi"] == ref["chi"]
        assert abs(got["energy"] - ref["energy"]) <= 1e-9 * abs(ref["energy"]), (got, ref)
        assert abs(got["entropy"] - ref["entropy"]) <= 1e-8
        assert abs(mx["energy"] - got["energy"]) <= 1e-9 * abs(got["energy"]), (mx, got)


def test_device_fdmrg_reproduces_spin_half_example(ctx):
    """fDMRG_DRV -B 50 -F 2 on 10 vertices, entirely on the device: the 5
    growth rows and the 4 sweep rows of the reference's example README
    (energy 1e-10 relative, entropy 1e-8, truncation 1e-12)."""
    from chainamps_b200 import fDMRG
    k = json.load(open(GOLD))["spin_half_fdmrg"]
    v = parse_user_vertex(k["basis"], k["hamiltonian"], k["operators"])
    H = make_general_hmpo(v, parse_couplings(k["input"].splitlines()[2]))
    run = fDMRG(ctx, H.rules, to_tensor(H), k["vertices"], tol=1e-12, krylov_dim=32)
    rows = run.run(k["sweeps"], k["chi"], k["trunc"])
    assert len(rows) == len(k["energies"])
    for r, e in zip(rows, k["energies"]):
        assert abs(r["energy"] - e[1]) <= 1e-10 * abs(e[1]), (r, e)
        assert abs(r["energy_per"] - e[2]) <= 1e-10 * abs(e[2])
        assert abs(r["entropy"] - e[3]) <= 1e-8, (r, e)
        assert abs(r["truncation"] - e[4]) <= 1e-12
    # fidelity: growth rows as printed; sweep rows as the oracle's restatement
    # of CheckConvergence(Prediction, MPSDecomposition), 0 to rounding for
    # these converged sweeps (the README prints 1 there; see the oracle's KAT)
    for r, e in zip(rows[:5], k["energies"][:5]):
        assert abs(r["fidelity"] - e[5]) <= 1e-10, (r, e)
    for r in rows[5:]:
        assert 0.0 <= r["fidelity"] <= 1e-10, r


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_fdmrg_matches_oracle_with_truncation(ctx, precision):
    """XXZ chain of 16 vertices at chi = 12 (truncating): every energies-file
    row of the device sweeps against the oracle's run_fdmrg."""
    from chainamps_b200 import fDMRG, CMPS_FP64, CMPS_SPLIT_TF32
    H = model_zoo()["xxz"]
    _, ref = od.run_fdmrg(H, 16, 2, 12, 1e-16, tol=1e-13)
    prec = CMPS_FP64 if precision == "fp64" else CMPS_SPLIT_TF32
    run = fDMRG(ctx, H.rules, to_tensor(H), 16, precision=prec, tol=1e-12, krylov_dim=32)
    rows = run.run(2, 12, 1e-16)
    assert len(rows) == len(ref)
    for r, e in zip(rows, ref):
        assert r["chi"] == e["chi"]
        assert abs(r["energy"] - e["energy"]) <= 1e-9 * abs(e["energy"]), (r, e)
        assert abs(r["entropy"] - e["entropy"]) <= 1e-7, (r, e)
        assert abs(r["truncation"] - e["truncation"]) <= 1e-11
        # growth rows: CheckConvergence(Prediction, previous values); sweep
        # rows: CheckConvergence(Prediction, MPSDecomposition)
        assert abs(r["fidelity"] - e["fidelity"]) <= (1e-8 if precision == "fp64" else 1e-6), (r, e)


def test_finite_prediction_starts_sweep_steps_close():
    """MakeR/LFinitePrediction on the device: once the sweeps have converged,
    a sweep step's Lanczos starts from the predicted wavefunction and needs
    far fewer matvecs than from a random start (16-20 against 40-48 for this
    chain at tol 1e-12); energies are unchanged sweep to sweep."""
    from chainamps_b200 import Context, fDMRG
    c = Context(0)
    H = model_zoo()["xxz"]
    run = fDMRG(c, H.rules, to_tensor(H), 16, tol=1e-12, krylov_dim=32)
    for _ in range(8):
        run.grow(12, 1e-16)
    mv, energies = [], []
    for sweep in range(3):
        for d in (+1, -1, +1):
            nl, size = run.position()
            for _ in range((size - nl - 2) if d > 0 else nl):
                r = run.move(d, 12, 1e-16)
                if sweep == 2:
                    mv.append(r["matvecs"])
                    energies.append(r["energy"])
    assert max(mv) <= 25, mv
    e0 = energies[len(energies) // 2]
    assert all(abs(e - e0) <= 1e-7 * abs(e0) for e in energies), energies
    run.close()
    c.close()
