"""The oracle reproduces the reference's own example outputs (its only
pinned results): spin-1/2 fDMRG and the quench example."""
import json
import os

import numpy as np
import pytest

from oracle.model import parse_user_vertex, parse_couplings, make_general_hmpo
from oracle.dmrg import run_fdmrg

GOLD = os.path.join(os.path.dirname(__file__), "golden", "kat_examples.json")


def _model(k):
    v = parse_user_vertex(k["basis"], k["hamiltonian"], k["operators"])
    return make_general_hmpo(v, parse_couplings(k["input"].splitlines()[2]))


def test_spin_half_fdmrg_kat():
    k = json.load(open(GOLD))["spin_half_fdmrg"]
    H = _model(k)
    assert H.indices[1].size == 11  # 2 + 3 couplings x 3 charge differences
    _, rows = run_fdmrg(H, k["vertices"], k["sweeps"], k["chi"], k["trunc"])
    ref = k["energies"]
    assert len(rows) == len(ref)
    for r, e in zip(rows, ref):
        assert abs(r["energy"] - e[1]) <= 1e-12 * abs(e[1])          # energy
        assert abs(r["energy_per"] - e[2]) <= 1e-12 * abs(e[2])
        assert abs(r["entropy"] - e[3]) <= 1e-12                      # entanglement entropy
        assert abs(r["truncation"] - e[4]) <= 1e-20                   # discarded weight
    for r, e in zip(rows[:5], ref[:5]):                               # growth-step fidelity
        assert abs(r["fidelity"] - e[5]) <= 1e-10


def test_quench_fdmrg_kat():
    k = json.load(open(GOLD))["quench_fdmrg"]
    H = _model(k)
    _, rows = run_fdmrg(H, k["vertices"], k["sweeps"], k["chi"], k["trunc"])
    ref = k["energies"]
    assert len(rows) == len(ref)
    for r, e in zip(rows, ref):
        assert abs(r["energy"] - e[1]) <= 1e-12 * abs(e[1])
        assert abs(r["entropy"] - e[3]) <= 1e-12
