"""Generate ``oracle_configs.json``: oracle results for the benchmark configs
that are parity cases, too slow to recompute in every test run.

* ``xxz_idmrg_chi100``: plain iDMRG on the spin-1/2 XXZ chain (Jxy = Jz = 1,
  h = 0, Pauli operators, Sz charge, reference-padded MPO D = 11), chi = 100,
  20 growth steps, eigensolver tolerance 1e-12: per step the energy, energy
  per vertex, entropy, truncation weight, fidelity and kept bond dimension
  from the oracle's SuperBlock (a restatement of SuperBlock::grow_two_vertex,
  DMRG_routines.cpp:346-374).
* ``coupled_ising_12x64_chi32``: iDMRG on coupled transverse-field Ising
  chains, each vertex the periodic 12-site chain at g = 1.2 cut to its 64
  lowest states (Z2 parity; ``models.ising_chain_vertex``), J_perp = 0.05
  sum_i X_i X_i between vertices (MPO D = 26), chi = 32, 5 growth steps,
  tolerance 1e-13: the same rows plus the kept singular values.  The
  oracle's SuperBlock solves each step with its canonical-order block port
  (``oracle/canonical.py``), the dense restatement being too large here.
  The rows are invariant under the sign gauge of the vertex basis.

Usage: python tests/golden/make_oracle_fixtures.py [name ...]
(all entries by default; the Ising entry takes about ten minutes)
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


def coupled_ising_12x64_chi32():
    from chainamps_b200 import models
    ch, ops, Hv, _, _ = models.ising_chain_vertex(12, 1.2, 64)
    H = om.make_general_hmpo(om.Vertex((2,), ch, ops, Hv),
                             [om.Coupling(f"J{i}", f"X{i}", f"X{i}", 0.05) for i in range(12)])
    sb = od.SuperBlock(H, tol=1e-13, heff="canonical")
    rows = []
    for _ in range(5):
        r = sb.grow(32, 1e-16)
        row = {k: (int(v) if k == "chi" else float(v)) for k, v in r.items()}
        row["values"] = [float(x) for x in sb.dec.values]
        rows.append(row)
    return {"model": "coupled TFIM chains: 12-site periodic chain, g=1.2, 64 lowest states (Z2), J_perp=0.05",
            "chi": 32, "steps": 5, "trunc": 1e-16, "tol": 1e-13, "rows": rows}


BUILDERS = {"xxz_idmrg_chi100": xxz_idmrg_chi100, "coupled_ising_12x64_chi32": coupled_ising_12x64_chi32}


def main(names):
    path = os.path.join(HERE, "oracle_configs.json")
    out = {}
    if os.path.exists(path):
        with open(path) as f:
            out = json.load(f)
    for name in names or sorted(BUILDERS):
        out[name] = BUILDERS[name]()
    with open(path, "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1:])
