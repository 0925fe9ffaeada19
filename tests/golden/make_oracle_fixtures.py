"""Generate ``oracle_configs.json``: oracle results for the benchmark configs
that are parity cases, too slow to recompute in every test run.

* ``xxz_idmrg_chi100``: plain iDMRG on the spin-1/2 XXZ chain (Jxy = Jz = 1,
  h = 0, Pauli operators, Sz charge, reference-padded MPO D = 11), chi = 100,
  20 growth steps, eigensolver tolerance 1e-12: per step the energy, energy
  per vertex, entropy, truncation weight, fidelity and kept bond dimension
  from the oracle's SuperBlock (a restatement of SuperBlock::grow_two_vertex,
  DMRG_routines.cpp:346-374).

Usage: python tests/golden/make_oracle_fixtures.py   (about one minute)
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import dmrg as od  # noqa: E402
from oracle import model as om  # noqa: E402


def xxz_idmrg_chi100():
    H = om.make_general_hmpo(om.spin_half_vertex(), om.xxz_couplings(1.0, 1.0, 0.0))
    sb = od.SuperBlock(H, tol=1e-12)
    rows = []
    for _ in range(20):
        r = sb.grow(100, 1e-16)
        rows.append({k: (int(v) if k == "chi" else float(v)) for k, v in r.items()})
    return {"model": "xxz jxy=1 jz=1 h=0", "chi": 100, "steps": 20, "trunc": 1e-16, "tol": 1e-12, "rows": rows}


def main():
    out = {"xxz_idmrg_chi100": xxz_idmrg_chi100()}
    with open(os.path.join(HERE, "oracle_configs.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
