"""Invariants of the oracle's projector tensors (oracle/excited.py), the
parity targets of the device ProjectorBlocks (no GPU):
* the stored ground state seen from its own centre window is the window's
  wavefunction: |P . theta| = 1 with theta the normalised window vector;
* after an excited state has converged, it is orthogonal to every stored
  state seen from its window (|P . theta| <= 1e-8) and its energy lies
  above the ground state's."""
import json
import os

import numpy as np

from oracle import excited as oe
from oracle.dmrg import TwoVertexComponents, run_fdmrg
from oracle.model import make_general_hmpo, parse_couplings, parse_user_vertex

GOLD = os.path.join(os.path.dirname(__file__), "golden", "kat_examples.json")


def _example():
    k = json.load(open(GOLD))["spin_half_fdmrg"]
    v = parse_user_vertex(k["basis"], k["hamiltonian"], k["operators"])
    return k, make_general_hmpo(v, parse_couplings(k["input"].splitlines()[2]))


def window_vector(sb):
    """The superblock's window wavefunction U diag(s) V^dagger on the allowed
    entries of its H_eff, normalised."""
    h = TwoVertexComponents(sb.lblocks[sb.nleft], sb.H, sb.rblocks[sb.nright])
    T = oe.state_tensors(sb)
    T1, T2 = T[sb.nleft], T[sb.nleft + 1]
    th = np.einsum("asr,rtb->satb", T1, T2).reshape((h.vrows, h.vcols), order="F").reshape(-1, order="F")
    x = th[h.allowed]
    return h, x / np.linalg.norm(x)


def test_projector_of_the_state_itself_is_its_window_vector():
    k, H = _example()
    sb, _ = run_fdmrg(H, k["vertices"], k["sweeps"], k["chi"], k["trunc"])
    h, x = window_vector(sb)
    p = oe.p_tensor(sb, oe.state_tensors(sb), h)
    assert abs(abs(p @ x) - 1.0) <= 1e-12
    assert abs(np.linalg.norm(p) - 1.0) <= 1e-12


def test_excited_states_are_orthogonal_to_the_projected_states():
    k, H = _example()
    sb, gs_rows = run_fdmrg(H, k["vertices"], k["sweeps"], k["chi"], k["trunc"])
    ex = oe.ExcitedSuperBlock.from_superblock(sb)
    ex.add_state(oe.state_tensors(sb))
    energies = [gs_rows[-1]["energy"]]
    for s in range(2):
        if s > 0:
            ex.add_state(oe.state_tensors(ex))
        rows = ex.run(k["sweeps"], k["chi"], k["trunc"])
        h, x = window_vector(ex)
        for T, _ in ex.states:
            assert abs(oe.p_tensor(ex, T, h) @ x) <= 1e-8
        energies.append(rows[-1]["energy"])
    assert energies[0] < energies[1] < energies[2]
