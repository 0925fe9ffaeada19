"""The device unit cell (cmps_dmrg_unit_cell: Orthogonalise +
iTwoVertexEnergy after an iDMRG step) through the C ABI.

* Against the oracle's restatement (oracle/unitcell.py, which regauges the
  cell as the reference does), on the same iDMRG run grown step by step on
  the device and in the oracle: the Heisenberg chain (Pauli couplings,
  Jxy = Jz = 1, chi = 24) and the transverse-field Ising chain (Z2).  The
  two runs' states agree to ~1e-7 in their singular values, so the energies
  per vertex are compared to 1e-8 relative and the entropies to 1e-6.
* The left and right dominant eigenvalues of the same transfer matrix
  agree to 1e-10.
* The energy per vertex of the chi = 100, 20-step XXZ run (the benchmark's
  first configuration) lies within 1e-4 above the exact infinite-chain
  value 1 - 4 ln 2 (Bethe ansatz)."""
import numpy as np
import pytest

from oracle import dmrg as od, model as om, unitcell as ou
from tests.helpers import model_zoo, to_tensor

pytestmark = pytest.mark.gpu

BETHE = 1.0 - 4.0 * np.log(2.0)


@pytest.fixture(scope="module")
def ctx():
    from chainamps_b200 import Context
    c = Context(0)
    yield c
    c.close()


def heisenberg():
    return om.make_general_hmpo(om.spin_half_vertex(), om.xxz_couplings(1.0, 1.0, 0.0))


@pytest.mark.parametrize("name,chi,steps,check", [("xxx", 24, 12, (4, 8, 12)), ("tfim", 16, 8, (8,))])
def test_unit_cell_matches_oracle(ctx, name, chi, steps, check):
    from chainamps_b200 import iDMRG
    H = heisenberg() if name == "xxx" else model_zoo()["tfim"]
    sb = od.SuperBlock(H, tol=1e-12)
    run = iDMRG(ctx, H.rules, to_tensor(H), tol=1e-12, krylov_dim=32)
    for step in range(1, steps + 1):
        sb.grow(chi, 1e-16)
        run.grow(chi, 1e-16)
        if step not in check:
            continue
        ref = ou.measure(sb.dec, sb.prev_lambda, H.data)
        got = run.unit_cell(tol=1e-13, krylov_dim=40)
        assert abs(got["energy"] - ref["energy"]) <= 1e-8 * abs(ref["energy"]), (step, got, ref["energy"])
        assert abs(got["entropy"] - ref["entropy"]) <= 1e-6, (step, got, ref["entropy"])
        assert abs(got["energy_imag"]) <= 1e-10
        assert abs(got["eta_left"] - got["eta_right"]) <= 1e-10 * got["eta_left"], got
    run.close()


def test_xxz_chi100_unit_cell_energy_near_bethe(ctx):
    from chainamps_b200 import iDMRG
    H = heisenberg()
    run = iDMRG(ctx, H.rules, to_tensor(H), tol=1e-12, krylov_dim=32)
    for _ in range(20):
        run.grow(100, 1e-16)
    got = run.unit_cell(tol=1e-13, krylov_dim=40)
    assert BETHE - 1e-10 <= got["energy"] <= BETHE + 1e-4, (got, BETHE)
    run.close()
