"""Reference-layout inputs for the hot path: the Hamiltonian MPO of a vertex
model and seeded synthetic environment blocks, as ``MPXTensor`` objects
ready for the C ABI.

The MPO follows the reference's ``MakeGeneralHMPO`` (make_model.hpp:471-621):
bond index = [identity, one slot per (coupling, charge difference), local
terms row], bond dimension 2 + n_couplings * n_charge_differences, the
vertex Hamiltonian and single-vertex terms at (last, first), the first
operator of each coupling in column 0 and coupling * second operator in the
last row, split by the charge difference of each matrix element
(``QNCombinations``, states.cpp:191-252).  The padded zero slots are kept,
exactly as the reference builds them; the device structure skips them.

Vertex models used by the workloads:
* spin-1/2 XXZ chain (one site per vertex, total-Sz charge);
* ``legs`` coupled spin-1/2 Heisenberg chains with one rung per vertex
  (local dimension 2**legs, total-Sz charge, rung coupling inside the
  vertex Hamiltonian, intra-chain couplings between vertices).
"""
from __future__ import annotations

import numpy as np

from .tensors import MPXTensor, MPXIndexSpec


def _charge_add(a, b, rules):
    out = np.asarray(a, np.int64) + np.asarray(b, np.int64)
    for i, n in enumerate(rules):
        if n > 0:
            out[..., i] %= n
    return out


def _charge_neg(a, rules):
    out = -np.asarray(a, np.int64)
    for i, n in enumerate(rules):
        if n > 0:
            out[..., i] %= n
    return out


def charge_difference_slots(charges, rules):
    """QNCombinations(basis, minus): (involution states, ordered states)."""
    seen = []
    for a in charges:
        for b in charges:
            t = tuple(int(x) for x in _charge_add(a, _charge_neg(b, rules), rules))
            if t not in seen:
                seen.append(t)
    invol = [t for t in seen if tuple(int(x) for x in _charge_neg(np.array(t), rules)) == t]
    rest = [t for t in seen if t not in invol]
    front, back = [], []
    if rest:
        front.insert(0, rest.pop(0))
        i = 0
        while i < len(rest):
            if tuple(int(x) for x in _charge_neg(np.array(rest[i]), rules)) == front[0]:
                back.append(rest.pop(i))
                if not rest:
                    break
                front.insert(0, rest.pop(0))
                i = 0
            else:
                i += 1
    return invol, front + back


def general_hmpo(charges, rules, hamiltonian, operators, couplings):
    """MakeGeneralHMPO.  couplings: list of (op1, op2 or None, value)."""
    charges = np.asarray(charges, np.int64)
    d = charges.shape[0]
    nq = len(rules)
    inter = [c for c in couplings if c[1]]
    local = [c for c in couplings if not c[1]]
    invol, ordered = charge_difference_slots(charges, rules)
    ndiff = len(invol) + len(ordered)
    D = 2 + len(inter) * ndiff
    W = np.zeros((d, D, d, D), np.complex128)
    for i in range(d):
        W[i, 0, i, 0] = 1.0
        W[i, D - 1, i, D - 1] = 1.0
    W[:, D - 1, :, 0] += hamiltonian
    for op, _, val in local:
        W[:, D - 1, :, 0] += val * operators[op]

    def slot(diff, same):
        t = tuple(int(x) for x in diff)
        tn = tuple(int(x) for x in _charge_neg(diff, rules))
        if t == tn:
            li = invol.index(t) if t in invol else 0
            return li, li
        if tn in ordered:
            li = ordered.index(tn)
            return len(invol) + li, ndiff - li - 1
        return 0, 0

    for b, (o1, o2, val) in enumerate(inter):
        base = 1 + b * ndiff
        A, B = operators[o1], operators[o2]
        same = o1 == o2
        for col in range(d):
            for i in range(d):
                if A[i, col] != 0:
                    ro, co = slot(_charge_add(charges[i], _charge_neg(charges[col], rules), rules), same)
                    W[i, base + ro, col, 0] += A[i, col]
                    if same:
                        W[i, D - 1, col, base + co] += val * A[i, col]
        if not same:
            for col in range(d):
                for i in range(d):
                    if B[i, col] != 0:
                        _, co = slot(_charge_add(charges[i], _charge_neg(charges[col], rules), rules), True)
                        W[i, D - 1, col, base + co] += val * B[i, col]
    bq = [np.zeros(nq, np.int64)]
    for _ in inter:
        bq += [np.array(t, np.int64) for t in invol] + [np.array(t, np.int64) for t in ordered]
    bq.append(np.zeros(nq, np.int64))
    bq = np.stack(bq).reshape(D, nq)
    return W, bq


def dense_to_tensor(indices, nrow, data):
    """Dense tensor (one axis per index, index order) -> MPXTensor (CSC of
    the matrix form, first index fastest)."""
    shp = data.shape
    rows = int(np.prod(shp[:nrow]))
    cols = int(np.prod(shp[nrow:]))
    M = data.reshape((rows, cols), order="F")
    nzr, nzc = np.nonzero(M.T)  # column-major order of non-zeros
    colptr = np.zeros(cols + 1, np.int64)
    np.add.at(colptr, nzr + 1, 1)
    colptr = np.cumsum(colptr)
    return MPXTensor(indices, nrow, rows, cols, colptr, nzc.astype(np.int64), M[nzc, nzr])


def mpo_tensor(charges, W, bq):
    charges = np.asarray(charges, np.int64)
    idx = [MPXIndexSpec(True, True, charges), MPXIndexSpec(True, False, bq),
           MPXIndexSpec(False, True, charges), MPXIndexSpec(False, False, bq)]
    return dense_to_tensor(idx, 2, W)


def pauli():
    return (np.array([[0, 1], [1, 0]], np.complex128), np.array([[0, -1j], [1j, 0]], np.complex128),
            np.array([[1, 0], [0, -1]], np.complex128))


def xxz_model(jxy=1.0, jz=1.0, h=0.0):
    """Spin-1/2 XXZ chain, Pauli operators, basis {+1, -1} with a Z charge."""
    sx, sy, sz = pauli()
    ops = {"Sx": sx, "Sy": sy, "Sz": sz}
    ch = np.array([[1], [-1]], np.int64)
    cps = [("Sx", "Sx", jxy), ("Sy", "Sy", jxy), ("Sz", "Sz", jz)]
    if h:
        cps.append(("Sz", None, h))
    W, bq = general_hmpo(ch, (0,), np.zeros((2, 2), np.complex128), ops, cps)
    return (0,), ch, W, bq


def ladder_model(legs=4, j=1.0, j_perp=0.5):
    """``legs`` spin-1/2 chains, one rung per vertex (S = sigma/2)."""
    sx, sy, sz = [p / 2 for p in pauli()]
    eye = np.eye(2, dtype=np.complex128)
    d = 2 ** legs

    def site(op, k):
        m = np.array([[1.0]], np.complex128)
        for q in range(legs):
            m = np.kron(m, op if q == k else eye)
        return m
    ops = {}
    for k in range(legs):
        ops[f"Sx{k}"], ops[f"Sy{k}"], ops[f"Sz{k}"] = site(sx, k), site(sy, k), site(sz, k)
    H = np.zeros((d, d), np.complex128)
    for k in range(legs - 1):
        for a in "xyz":
            H += j_perp * ops[f"S{a}{k}"] @ ops[f"S{a}{k + 1}"]
    ch = np.zeros((d, 1), np.int64)
    for s in range(d):
        ch[s, 0] = sum(1 if ((s >> (legs - 1 - q)) & 1) == 0 else -1 for q in range(legs))
    cps = [(f"S{a}{k}", f"S{a}{k}", j) for k in range(legs) for a in "xyz"]
    W, bq = general_hmpo(ch, (0,), H, ops, cps)
    return (0,), ch, W, bq


def ising_chain_vertex(sites=12, g=1.2, keep=64, g_basis=None):
    """One vertex = a periodic transverse-field Ising chain
    H(g) = -sum_i X_i X_{i+1} - g sum_i Z_i, reduced to its `keep` lowest
    eigenstates (computed at g_basis, default g) with their Z2 parity
    (prod_i Z_i) as the charge, rules (2,).

    Returns (charges (keep, 1), ops {"X0".."X{sites-1}": keep x keep
    sigma^x_i in the kept basis (parity odd)}, H (keep x keep, the vertex
    Hamiltonian at g in that basis), dH_dg (keep x keep), gap at the cut).
    The basis is built per parity sector in the sigma^z product basis with bit
    operations; each eigenvector's sign makes its first largest component
    (to 1e-9) positive, and degenerate levels are split by a fixed diagonal
    operator without the chain's symmetries, so the
    basis does not depend on the LAPACK build or its thread count.
    Near-degenerate states (momentum pairs) are kept or cut together only if
    the cut falls in a gap; the gap at the cut is returned."""
    gb = g if g_basis is None else g_basis
    n = 1 << sites
    s = np.arange(n, dtype=np.int64)
    bits = (s[:, None] >> np.arange(sites)[None, :]) & 1            # 1 = spin down
    z = 1 - 2 * bits                                                  # Z_i eigenvalue
    zsum = z.sum(axis=1).astype(np.float64)
    parity = (bits.sum(axis=1) & 1)                                   # 0: even, 1: odd
    evals, vecs, labels = [], [], []
    for par in (0, 1):
        sel = np.nonzero(parity == par)[0]
        pos = -np.ones(n, np.int64)
        pos[sel] = np.arange(sel.size)
        Hs = np.zeros((sel.size, sel.size))
        Hs[np.arange(sel.size), np.arange(sel.size)] = -gb * zsum[sel]
        for i in range(sites):
            flip = (1 << i) | (1 << ((i + 1) % sites))
            Hs[np.arange(sel.size), pos[sel ^ flip]] -= 1.0
        w, v = np.linalg.eigh(Hs)
        # Exactly degenerate levels (momentum pairs of the periodic chain,
        # reflection multiplets): the eigensolver returns an arbitrary basis
        # of each such subspace, which would make the kept state at a cut
        # inside one depend on the LAPACK build and its thread count.  Fix
        # it: inside each cluster, rotate to the eigenvectors of a fixed
        # diagonal operator with no symmetry of the chain (cos(0.7 s + 0.3)
        # on product state s) restricted to the subspace, ordered by its
        # eigenvalue.
        tol = 1e-9 * max(1.0, float(np.max(np.abs(w))))
        splitter = np.cos(0.7 * sel.astype(np.float64) + 0.3)
        k = 0
        while k < w.size:
            e = k + 1
            while e < w.size and w[e] - w[e - 1] <= tol:
                e += 1
            if e - k > 1:
                sub = v[:, k:e]
                a, u = np.linalg.eigh(sub.T @ (splitter[:, None] * sub))
                v[:, k:e] = sub @ u
                w[k:e] = np.mean(w[k:e])
            k = e
        for k in range(w.size):
            vec = np.zeros(n)
            vec[sel] = v[:, k]
            # sign: the first component within 1e-9 (relative) of the largest
            # magnitude is positive (symmetric states have many equal ones)
            mag = np.abs(vec)
            j = int(np.argmax(mag >= mag.max() * (1.0 - 1e-9)))
            if vec[j] < 0:
                vec = -vec
            evals.append(w[k])
            vecs.append(vec)
            labels.append(par)
    # ascending energy; levels equal to 1e-9 (relative) keep parity-then-basis
    # order, so the order never rests on the last bits of the eigenvalues
    evals = np.asarray(evals)
    q = np.round(evals / (1e-9 * max(1.0, float(np.max(np.abs(evals)))))).astype(np.int64)
    order = np.lexsort((np.arange(evals.size), np.asarray(labels), q))
    ev = evals[order]
    gap = float(ev[keep] - ev[keep - 1]) if keep < ev.size else float("inf")
    order = order[:keep]
    V = np.stack([vecs[i] for i in order], axis=1)                   # n x keep, real
    ch = np.asarray([[labels[i]] for i in order], np.int64)
    ops = {}
    for i in range(sites):
        ops[f"X{i}"] = (V.T @ V[s ^ (1 << i)]).astype(np.complex128)
    Hxx = np.zeros((keep, keep))
    for i in range(sites):
        flip = (1 << i) | (1 << ((i + 1) % sites))
        Hxx -= V.T @ V[s ^ flip]
    Hz = -(V * zsum[:, None]).T @ V
    H = (Hxx + g * Hz).astype(np.complex128)
    H = 0.5 * (H + H.conj().T)
    return ch, ops, H, Hz.astype(np.complex128), gap


def coupled_ising_model(sites=12, g=1.2, keep=64, j_perp=0.05, g_basis=None):
    """Coupled transverse-field Ising chains: each vertex is the chain of
    ising_chain_vertex, neighbouring vertices coupled by
    j_perp * sum_i X_i X_i (chain-basis matrix elements, parity odd, so only
    the total Z2 parity is conserved).  Returns (rules, charges, W, bq) of
    the reference's MakeGeneralHMPO layout."""
    ch, ops, H, _, _ = ising_chain_vertex(sites, g, keep, g_basis)
    cps = [(f"X{i}", f"X{i}", j_perp) for i in range(sites)]
    W, bq = general_hmpo(ch, (2,), H, ops, cps)
    return (2,), ch, W, bq


def gaussian_bond(chi, step=2, width=3.5, offset=0):
    """Bond charges with a discretised Gaussian sector-size profile (the
    shape of a converged total-Sz distribution), ``chi`` elements, charges
    offset + step * k."""
    ks = np.arange(-40, 41)
    p = np.exp(-0.5 * (ks * step / width) ** 2)
    p /= p.sum()
    n = np.floor(p * chi).astype(int)
    rem = chi - n.sum()
    order = np.argsort(-(p * chi - n))
    n[order[:rem]] += 1
    q = np.concatenate([np.full(c, offset + step * k) for k, c in zip(ks, n) if c > 0])
    return q.reshape(-1, 1).astype(np.int64)


def random_environment(rng, rules, bond, bq, used_b, right):
    """Seeded random environment block obeying q(a') = q(b) + q(a), only on
    the MPO slots in ``used_b``; complex Gaussian entries, Hermitian in (a', a)
    for each b paired with its conjugate slot is not imposed."""
    chi = bond.shape[0]
    D = bq.shape[0]
    nq = len(rules)
    vals = np.zeros((chi, D, chi), np.complex128)
    for b in used_b:
        ok = np.all(bond[:, None, :] == _charge_add(bq[b][None, None, :], bond[None, :, :], rules), axis=-1)
        nzr, nzc = np.nonzero(ok)
        vals[nzr, b, nzc] = (rng.standard_normal(nzr.size) + 1j * rng.standard_normal(nzr.size)) / np.sqrt(2)
    z = np.zeros((1, nq), np.int64)
    if not right:
        idx = [MPXIndexSpec(False, False, z), MPXIndexSpec(True, False, bond), MPXIndexSpec(True, False, z),
               MPXIndexSpec(False, False, bq), MPXIndexSpec(True, False, z), MPXIndexSpec(False, False, bond)]
        return dense_to_tensor(idx, 3, vals.reshape(1, chi, 1, D, 1, chi))
    idx = [MPXIndexSpec(False, False, bond), MPXIndexSpec(True, False, z), MPXIndexSpec(True, False, bq),
           MPXIndexSpec(False, False, z), MPXIndexSpec(True, False, bond), MPXIndexSpec(False, False, z)]
    return dense_to_tensor(idx, 2, vals.reshape(chi, 1, D, 1, chi, 1))


def ladder_workload(chi, seed=20261203, width=3.5, legs=4, j=1.0, j_perp=0.5):
    """The synthetic H_eff workload of the ladder benchmark: the ``legs``-leg
    Heisenberg ladder vertex (reference-padded MPO) between seeded random
    left and right environments on a Gaussian total-Sz bond of ``chi``
    elements (charges 2k, sector profile width ``width``), entries only on
    the MPO slots the MPO uses.  Returns the model arrays and the three
    tensors (L, Wt, R) as the reference would hand them over."""
    rules, ch, W, bq = ladder_model(legs, j, j_perp)
    used_l = sorted({int(b) for b in np.nonzero(np.any(W != 0, axis=(0, 2, 3)))[0]})
    used_r = sorted({int(b) for b in np.nonzero(np.any(W != 0, axis=(0, 1, 2)))[0]})
    bond = gaussian_bond(chi, step=2, width=width)
    rng = np.random.default_rng(seed)
    L = random_environment(rng, rules, bond, bq, used_l, right=False)
    R = random_environment(rng, rules, bond, bq, used_r, right=True)
    Wt = mpo_tensor(ch, W, bq)
    return dict(rules=rules, ch=ch, W=W, bq=bq, bond=bond, L=L, R=R, Wt=Wt)


def ising_workload(chi, seed=20261203, sites=12, g=1.2, keep=64, j_perp=0.05):
    """The synthetic H_eff workload of the coupled-Ising chains: the
    ``sites``-site chain vertex cut to ``keep`` states (Z2 parity), between
    seeded random left and right environments on a Z2 bond of ``chi``
    elements (two sectors of chi / 2), entries only on the MPO slots the MPO
    uses.  Returns the model arrays and the three tensors (L, Wt, R)."""
    rules, ch, W, bq = coupled_ising_model(sites, g, keep, j_perp)
    used_l = sorted({int(b) for b in np.nonzero(np.any(W != 0, axis=(0, 2, 3)))[0]})
    used_r = sorted({int(b) for b in np.nonzero(np.any(W != 0, axis=(0, 1, 2)))[0]})
    bond = (np.arange(chi) % 2).reshape(-1, 1).astype(np.int64)
    rng = np.random.default_rng(seed)
    L = random_environment(rng, rules, bond, bq, used_l, right=False)
    R = random_environment(rng, rules, bond, bq, used_r, right=True)
    Wt = mpo_tensor(ch, W, bq)
    return dict(rules=rules, ch=ch, W=W, bq=bq, bond=bond, L=L, R=R, Wt=Wt)

