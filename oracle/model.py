"""CPU oracle (test infrastructure only): model input and the Hamiltonian MPO.

Restates how ChainAMPS turns a "USER DEFINED" model into the MPO that the
DMRG hot path reads:

* the input file (model name / basis+hamiltonian+operator files / coupling
  line ``Name,(Op1,Op2):value``) -- ``make_model.hpp:72-253``,
  ``model.hpp:144-203``;
* the vertex basis, operators and vertex Hamiltonian files --
  ``make_model.hpp:269-469``;
* ``QNCombinations`` (charge-difference slots of the MPO bond) --
  ``states.cpp:191-252``;
* ``MakeGeneralHMPO``: lower-triangular MPO, bond dimension
  ``2 + n_couplings * n_charge_differences`` -- ``make_model.hpp:471-621``.

Also builds synthetic vertices used by the benchmark workloads (spin-1/2
sites, four-leg spin ladders as one vertex) through the same MPO builder, so
that their MPO has exactly the reference's padded slot structure.
"""
from __future__ import annotations

from dataclasses import dataclass, field
import re
import numpy as np

from .mpx import Index, MPX, q_add, q_sub, q_neg, q_eq


@dataclass
class Vertex:
    rules: tuple                      # charge rules (N of each Z_N; <=0 means Z)
    charges: np.ndarray               # (d, nq) basis charges
    operators: dict = field(default_factory=dict)  # name -> (d, d) complex matrix, M[row, col]
    hamiltonian: np.ndarray | None = None

    @property
    def d(self) -> int:
        return int(self.charges.shape[0])


@dataclass
class Coupling:
    name: str
    op1: str
    op2: str | None
    value: complex

    @property
    def two_vertex(self) -> bool:
        return bool(self.op2)


def _parse_complex(tok: str) -> complex:
    """std::complex<double> stream extraction: '1.0', '(1.0)', '(0.0,-1.0)'."""
    tok = tok.strip()
    if tok.startswith("("):
        inner = tok[1:-1] if tok.endswith(")") else tok[1:]
        parts = inner.split(",")
        if len(parts) == 1:
            return complex(float(parts[0]), 0.0)
        return complex(float(parts[0]), float(parts[1]))
    return complex(float(tok), 0.0)


def parse_couplings(line: str):
    """Coupling stream extraction (model.hpp:144-203)."""
    out = []
    for m in re.finditer(r"\s*([^,\s]+),\(([^)]*)\)\s*:\s*(\([^)]*\)|[^\s]+)", line):
        name, ops, val = m.group(1), m.group(2), m.group(3)
        names = [s.strip() for s in ops.split(",")]
        op1 = names[0]
        op2 = names[1] if len(names) > 1 else None
        out.append(Coupling(name, op1, op2, _parse_complex(val)))
    return out


def _state_from_values(rules, vals):
    """State(CHARGE_RULES, v) (states.cpp:13-26)."""
    v = list(vals) + [0] * (len(rules) - len(vals))
    out = []
    for n, x in zip(rules, v):
        if n > 1:
            out.append(int(x) % n)
        elif n == 1:
            out.append(0)
        else:
            out.append(int(x))
    return out


def parse_user_vertex(basis_text: str, ham_text: str, op_texts) -> Vertex:
    """MakeUserModel file reading (make_model.hpp:269-469)."""
    lines = basis_text.splitlines()
    first = lines[0].split()
    rules = []
    if first[0].startswith("D"):
        rules = [int(x) for x in first[1:]] or [0]
    elif first[0].startswith("#"):
        for w in first[1:]:
            rules.append(int(w[w.rfind("_") + 1:]) if "_" in w else 0)
    else:
        raise ValueError("no charge definitions")
    rules = tuple(rules)
    ch = []
    for ln in lines[1:]:
        toks = ln.split()
        if len(toks) >= 2:
            ch.append(_state_from_values(rules, [int(t) for t in toks[1:]]))
    charges = np.asarray(ch, dtype=np.int64).reshape(len(ch), len(rules))
    d = charges.shape[0]
    ops = {}
    for text in op_texts:
        olines = text.splitlines()
        names = olines[0].split()
        mats = [np.zeros((d, d), dtype=np.complex128) for _ in names]
        start = 1
        if len(olines) > 1 and olines[1].strip() and not olines[1].lstrip()[0].isdigit():
            start = 2  # optional dummy line
        for ln in olines[start:]:
            toks = ln.split()
            if len(toks) < 2 + len(names):
                continue
            r, c = int(toks[0]), int(toks[1])
            for k in range(len(names)):
                v = _parse_complex(toks[2 + k])
                if v != 0:
                    mats[k][r, c] += v
        for n, m in zip(names, mats):
            ops[n] = m
    H = np.zeros((d, d), dtype=np.complex128)
    for ln in ham_text.splitlines():
        toks = ln.split()
        if len(toks) >= 3:
            H[int(toks[0]), int(toks[1])] += _parse_complex(toks[2])
    return Vertex(rules, charges, ops, H)


# --------------------------------------------------------------------------
# QNCombinations (states.cpp:191-252)
# --------------------------------------------------------------------------
def qn_combinations(charges, rules, minus=True):
    """Return (involution_states, ordered_states) as lists of charge tuples."""
    unsorted = []
    for a in charges:
        for b in charges:
            s = q_sub(a, b, rules) if minus else q_add(a, b, rules)
            t = tuple(int(x) for x in s)
            if t not in unsorted:
                unsorted.append(t)
    invol = []
    rest = []
    for t in unsorted:
        if tuple(int(x) for x in q_neg(np.array(t), rules)) == t:
            invol.append(t)
        else:
            rest.append(t)
    # deque construction: front = newest test state, back = its negatives
    ordered_front = []
    ordered_back = []
    lst = list(rest)
    if lst:
        ordered_front.insert(0, lst.pop(0))
        i = 0
        while i < len(lst):
            neg = tuple(int(x) for x in q_neg(np.array(lst[i]), rules))
            if neg == ordered_front[0]:
                ordered_back.append(lst.pop(i))
                if not lst:
                    break
                ordered_front.insert(0, lst.pop(0))
                i = 0
            else:
                i += 1
    ordered = ordered_front + ordered_back
    return invol, ordered


# --------------------------------------------------------------------------
# MakeGeneralHMPO (make_model.hpp:471-621)
# --------------------------------------------------------------------------
def make_general_hmpo(v: Vertex, couplings) -> MPX:
    inter = [c for c in couplings if c.two_vertex]
    local = [c for c in couplings if not c.two_vertex]
    rules = v.rules
    d = v.d
    invol, ordered = qn_combinations(v.charges, rules, minus=True)
    ndiff = len(invol) + len(ordered)
    D = 2 + len(inter) * ndiff
    W = np.zeros((d, D, d, D), dtype=np.complex128)  # [sigma', b_l, sigma, b_r]
    for i in range(d):
        W[i, 0, i, 0] += 1.0
        W[i, D - 1, i, D - 1] += 1.0
    if v.hamiltonian is not None:
        W[:, D - 1, :, 0] += v.hamiltonian
    for l in local:
        W[:, D - 1, :, 0] += l.value * v.operators[l.op1]

    def slot_offsets(diff, same):
        """(row slot offset, col slot offset) for a charge difference."""
        t = tuple(int(x) for x in diff)
        tneg = tuple(int(x) for x in q_neg(diff, rules))
        if t == tneg:
            for li, s in enumerate(invol):
                if s == t:
                    return li, (li if same else 0)
            return 0, 0
        for li, s in enumerate(ordered):
            if s == tneg:
                return len(invol) + li, ndiff - li - 1
        return 0, 0

    def col_offset(diff):
        t = tuple(int(x) for x in diff)
        tneg = tuple(int(x) for x in q_neg(diff, rules))
        if t == tneg:
            for li, s in enumerate(invol):
                if s == t:
                    return li
            return 0
        for li, s in enumerate(ordered):
            if s == tneg:
                return ndiff - li - 1
        return 0

    for b, c in enumerate(inter):
        row_sp = v.operators[c.op1]
        col_sp = v.operators[c.op2]
        same = c.op1 == c.op2
        rbase = 1 + b * ndiff
        cbase = 1 + b * ndiff
        for col in range(d):
            for i in range(d):
                x = row_sp[i, col]
                if x == 0:
                    continue
                diff = q_sub(v.charges[i], v.charges[col], rules)
                ro, co = slot_offsets(diff, same)
                W[i, rbase + ro, col, 0] += x
                if same:
                    W[i, D - 1, col, cbase + co] += c.value * x
        if not same:
            for col in range(d):
                for i in range(d):
                    x = col_sp[i, col]
                    if x == 0:
                        continue
                    diff = q_sub(v.charges[i], v.charges[col], rules)
                    co = col_offset(diff)
                    W[i, D - 1, col, cbase + co] += c.value * x
    nq = len(rules)
    bq = [np.zeros(nq, dtype=np.int64)]
    for _ in inter:
        for s in invol:
            bq.append(np.array(s, dtype=np.int64))
        for s in ordered:
            bq.append(np.array(s, dtype=np.int64))
    bq.append(np.zeros(nq, dtype=np.int64))
    bq = np.stack(bq).reshape(D, nq)
    idx = [Index(True, True, v.charges), Index(True, False, bq),
           Index(False, True, v.charges), Index(False, False, bq)]
    return MPX(rules, idx, 2, W)


def mpo_extract(H: MPX, rows, cols) -> MPX:
    """MPO_matrix::ExtractMPOBlock (MPO_matrix.cpp:69-85): keep b_left in
    [rows[0], rows[1]] and b_right in [cols[0], cols[1]]."""
    r0, r1 = rows
    c0, c1 = cols
    data = H.data[:, r0:r1 + 1, :, c0:c1 + 1]
    bl = Index(True, False, H.indices[1].charges[r0:r1 + 1])
    br = Index(False, False, H.indices[3].charges[c0:c1 + 1])
    return MPX(H.rules, [H.indices[0], bl, H.indices[2], br], 2, np.ascontiguousarray(data))


def left_open_bc(H: MPX) -> MPX:
    """LeftOpenBCHamiltonian (DMRG_routines.hpp:218)."""
    D = H.indices[1].size
    return mpo_extract(H, (D - 1, D - 1), (0, H.indices[3].size - 1))


def right_open_bc(H: MPX) -> MPX:
    """RightOpenBCHamiltonian (DMRG_routines.hpp:222)."""
    return mpo_extract(H, (0, H.indices[1].size - 1), (0, 0))


# --------------------------------------------------------------------------
# synthetic vertices for the workloads
# --------------------------------------------------------------------------
def pauli():
    sx = np.array([[0, 1], [1, 0]], dtype=np.complex128)
    sy = np.array([[0, -1j], [1j, 0]], dtype=np.complex128)
    sz = np.array([[1, 0], [0, -1]], dtype=np.complex128)
    return sx, sy, sz


def spin_half_vertex(sz_charges=True) -> Vertex:
    """One spin-1/2 per vertex, Pauli operators, basis {up (+1), down (-1)}
    with a Z (total Sz) charge, as in the spin-half user model."""
    sx, sy, sz = pauli()
    ch = np.array([[1], [-1]], dtype=np.int64) if sz_charges else np.zeros((2, 1), np.int64)
    rules = (0,) if sz_charges else (1,)
    return Vertex(rules, ch, {"Sx": sx, "Sy": sy, "Sz": sz}, np.zeros((2, 2), np.complex128))


def ladder_vertex(legs=4, j_perp=0.5) -> Vertex:
    """``legs`` spin-1/2 sites (one per chain) as one vertex: basis = product
    states, charge = total Sz in units of 1/2 (Z), vertex Hamiltonian =
    open rung Heisenberg chain J_perp * sum_j S_j.S_{j+1} with S = sigma/2.
    Operators Sx_j, Sy_j, Sz_j are the spin-1/2 operators (sigma/2)."""
    sx, sy, sz = pauli()
    sx, sy, sz = sx / 2, sy / 2, sz / 2
    d = 2 ** legs
    eye = np.eye(2, dtype=np.complex128)

    def site_op(op, j):
        m = np.array([[1.0]], dtype=np.complex128)
        for k in range(legs):
            m = np.kron(m, op if k == j else eye)
        return m

    ops = {}
    for j in range(legs):
        ops[f"Sx{j}"] = site_op(sx, j)
        ops[f"Sy{j}"] = site_op(sy, j)
        ops[f"Sz{j}"] = site_op(sz, j)
    H = np.zeros((d, d), dtype=np.complex128)
    for j in range(legs - 1):
        for a in "xyz":
            H += j_perp * ops[f"S{a}{j}"] @ ops[f"S{a}{j + 1}"]
    # kron ordering: site 0 is the most significant bit; |0> = up (+1)
    ch = np.zeros((d, 1), dtype=np.int64)
    for s in range(d):
        tot = 0
        for k in range(legs):
            bit = (s >> (legs - 1 - k)) & 1
            tot += 1 if bit == 0 else -1
        ch[s, 0] = tot
    return Vertex((0,), ch, ops, H)


def ladder_couplings(legs=4, j=1.0):
    out = []
    for k in range(legs):
        for a in "xyz":
            out.append(Coupling(f"J{a}{k}", f"S{a}{k}", f"S{a}{k}", complex(j)))
    return out


def xxz_couplings(jxy=1.0, jz=1.0, h=0.0):
    out = [Coupling("Jx", "Sx", "Sx", complex(jxy)), Coupling("Jy", "Sy", "Sy", complex(jxy)),
           Coupling("Jz", "Sz", "Sz", complex(jz))]
    if h != 0.0:
        out.append(Coupling("hz", "Sz", None, complex(h)))
    return out
