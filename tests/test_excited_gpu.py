"""Excited states on the device: the projector tensors of stored states
(ProjectorBlocks, DMRG_routines.cpp:446-581) built on the GPU from the
stored and the current MPS tensors, and the excited-state finite DMRG
(fDMRG_DRV -X, ExcitedStateFiniteDMRG, fDMRG_routines.cpp:68-244) driven
through cmps_dmrg_project_state / cmps_dmrg_solve / cmps_dmrg_move.

* The reference's example (fDMRG_DRV -B 50 -F 2 -X 2 on 10 vertices,
  examples/user_defined/spin_half_example/README.md:58-70): each excited
  state's converged final row, energy 1e-10 relative and entropy 1e-8, and
  the number of rows, as the oracle's excited-state DMRG reproduces them;
  the mixed-precision form within 1e-9.
* The stored state seen from its own window is the window's normalised
  wavefunction: |P| = 1 (1e-12).
* After each excited state has converged, its energy lies above the earlier
  ones and the oracle's excited energies agree (1e-10).
* Growth steps and negative weights are refused."""
import json
import os

import numpy as np
import pytest

from oracle.model import parse_user_vertex, parse_couplings, make_general_hmpo
from tests.helpers import to_tensor

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "kat_examples.json")


@pytest.fixture(scope="module")
def ctx():
    from chainamps_b200 import Context
    c = Context(0)
    yield c
    c.close()


def example():
    k = json.load(open(GOLD))["spin_half_fdmrg"]
    v = parse_user_vertex(k["basis"], k["hamiltonian"], k["operators"])
    return k, make_general_hmpo(v, parse_couplings(k["input"].splitlines()[2]))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_excited_states_reproduce_the_example(ctx, precision):
    from chainamps_b200 import run_excited_fdmrg, CMPS_FP64, CMPS_SPLIT_TF32
    k, H = example()
    prec = CMPS_FP64 if precision == "fp64" else CMPS_SPLIT_TF32
    tol = 1e-10 if precision == "fp64" else 1e-9
    gs, ex, run = run_excited_fdmrg(ctx, H.rules, to_tensor(H), k["vertices"], k["sweeps"], k["chi"], k["trunc"],
                                    nstates=2, precision=prec, tol=1e-12, krylov_dim=32)
    assert abs(gs[-1]["energy"] - k["energies"][-1][1]) <= 1e-10 * abs(k["energies"][-1][1])
    assert run.projected_states() == 2
    ref = k["excited_energies"]
    last = gs[-1]["energy"]
    for s, rows in enumerate(ex, start=1):
        rr = [r for r in ref if r[1] == float(s)]
        assert len(rows) == len(rr)
        assert abs(rows[-1]["energy"] - rr[-1][2]) <= tol * abs(rr[-1][2]), (s, rows[-1], rr[-1])
        assert abs(rows[-1]["entropy"] - rr[-1][3]) <= 1e-8 * (1 if precision == "fp64" else 100), (s, rows[-1])
        assert rows[-1]["energy"] > last
        last = rows[-1]["energy"]


def test_projector_of_the_state_itself_is_normalised(ctx):
    from chainamps_b200 import fDMRG
    k, H = example()
    run = fDMRG(ctx, H.rules, to_tensor(H), k["vertices"], tol=1e-12, krylov_dim=32)
    run.run(k["sweeps"], k["chi"], k["trunc"])
    run.project_state(100.0)
    # the solve installs the stored state's projector for the current window,
    # whose bases are still the stored state's own
    row = run.solve(k["chi"], k["trunc"])
    p = run.projector(0)
    assert p.size == run.window_length()[0]
    assert abs(np.linalg.norm(p) - 1.0) <= 1e-12
    # the lowest eigenvalue of H + 100 |P*><P*| on that window, as the
    # oracle's ExcitedStateFiniteDMRG::init finds it
    from oracle import excited as oe
    from oracle.dmrg import run_fdmrg
    sb, _ = run_fdmrg(H, k["vertices"], k["sweeps"], k["chi"], k["trunc"], tol=1e-14)
    exs = oe.ExcitedSuperBlock.from_superblock(sb, tol=1e-14)
    exs.add_state(oe.state_tensors(sb))
    want = exs.init(k["chi"], k["trunc"])
    assert abs(row["energy"] - want["energy"]) <= 1e-10 * abs(want["energy"]), (row, want)
    assert abs(row["entropy"] - want["entropy"]) <= 1e-8


def test_growth_and_bad_weights_are_refused(ctx):
    from chainamps_b200 import fDMRG, CmpsError
    k, H = example()
    run = fDMRG(ctx, H.rules, to_tensor(H), 6, tol=1e-12, krylov_dim=32)
    run.run(1, 16, 1e-16)
    with pytest.raises(CmpsError):
        run.project_state(-1.0)
    run.project_state(100.0)
    with pytest.raises(CmpsError):
        run.grow(16, 1e-16)
