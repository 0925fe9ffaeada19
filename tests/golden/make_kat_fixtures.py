"""Generate ``kat_examples.json`` from the reference's own example runs.

The reference (andyjaj/chainamps) ships no unit tests; its only pinned
results are the example inputs and the outputs printed in the example
READMEs.  This script reads them from a checkout of the reference and stores
them as a small fixture, so the oracle and the GPU path can be checked
against them on machines where the reference is not present:

* ``examples/user_defined/spin_half_example``: input files, the
  ``example_input_Energies.dat`` table printed in ``README.md``
  (``fDMRG_DRV.bin -B 50 -F 2 -X 2 example_input 10``; ground state rows)
  and the ``example_input_Excited_Energies.dat`` table of the two excited
  states (README.md:58-70);
* ``examples/user_defined/quench_example``: input files and
  ``initial_input_Energies.dat`` (``fDMRG_DRV.bin -F 1 initial_input 20``);
* ``examples/built_in/xxx_lattice_chains/README.md``: the raw iDMRG table
  (``iDMRG_DRV.bin -B50 -N 10 xxx_input``), kept for reference.

Usage: python tests/golden/make_kat_fixtures.py /path/to/chainamps
"""
import json
import os
import re
import sys


def read(p):
    with open(p) as f:
        return f.read()


def table_after(text, header_prefix):
    """Rows of numbers following the first line that starts with header_prefix."""
    lines = text.splitlines()
    rows = []
    for i, ln in enumerate(lines):
        if ln.strip().startswith(header_prefix):
            for ln2 in lines[i + 1:]:
                s = ln2.strip()
                if not s or s.startswith("~"):
                    break
                rows.append([float(x) for x in s.split()])
            break
    return rows


def main(ref):
    ex = os.path.join(ref, "examples")
    sh = os.path.join(ex, "user_defined", "spin_half_example")
    sh_readme = read(os.path.join(sh, "README.md"))
    spin_half = {
        "command": "fDMRG_DRV.bin -B 50 -F 2 -X 2 example_input 10",
        "chi": 50, "sweeps": 2, "vertices": 10, "trunc": 1e-16,
        "input": read(os.path.join(sh, "example_input")),
        "basis": read(os.path.join(sh, "vertex_basis.in")),
        "hamiltonian": read(os.path.join(sh, "vertex_hamiltonian.in")),
        "operators": [read(os.path.join(sh, n)) for n in ("Sx.in", "Sy.in", "Sz.in")],
        "energies": table_after(sh_readme, "# Index, Energy, Energy/vertices"),
        "source": "examples/user_defined/spin_half_example/README.md:28-40",
        "excited_energies": table_after(sh_readme, "# Sweep Index, State Index, Energy"),
        "excited_source": "examples/user_defined/spin_half_example/README.md:58-70",
    }
    q = os.path.join(ex, "user_defined", "quench_example")
    quench = {
        "command": "fDMRG_DRV.bin -F 1 initial_input 20",
        "chi": 0, "sweeps": 1, "vertices": 20, "trunc": 1e-16,
        "input": read(os.path.join(q, "initial_input")),
        "basis": read(os.path.join(q, "initial_defs", "vertex_basis.in")),
        "hamiltonian": read(os.path.join(q, "initial_defs", "vertex_hamiltonian.in")),
        "operators": [read(os.path.join(q, "initial_defs", "vertex_operators.in"))],
        "energies": [[float(x) for x in ln.split()] for ln in read(os.path.join(q, "initial_input_Energies.dat")).splitlines()
                     if ln.strip() and not ln.startswith("#")],
        "source": "examples/user_defined/quench_example/initial_input_Energies.dat",
    }
    xreadme = read(os.path.join(ex, "built_in", "xxx_lattice_chains", "README.md"))
    xxx = {
        "command": "iDMRG_DRV.bin -B50 -N 10 xxx_input",
        "energies": table_after(xreadme, "# Index, Energy, Energy/vertex"),
        "source": "examples/built_in/xxx_lattice_chains/README.md:16-29",
    }
    out = {"spin_half_fdmrg": spin_half, "quench_fdmrg": quench, "xxx_idmrg": xxx}
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "kat_examples.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    # the reference checkout: first argument, else $CHAINAMPS_REFERENCE
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CHAINAMPS_REFERENCE")
    if not src:
        sys.exit("usage: make_kat_fixtures.py <path to the ChainAMPS checkout> "
                 "(or set CHAINAMPS_REFERENCE)")
    main(src)
