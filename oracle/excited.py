"""CPU restatement of the excited-state finite DMRG: ProjectorBlocks and
ExcitedStateFiniteDMRG.  Test infrastructure (the oracle): only tests use it.

The reference (fDMRG_DRV -X n) finds the ground state by finite DMRG, then
each excited state by the same sweeps with a projector term in the matvec
(TwoVertexMPOMPSMultiply, DMRG_routines.cpp:947-973):

    y = H x + sum_p w_p (P_p . x) conj(P_p),

P_p being the stored state p seen from the current two-vertex window
(ProjectorBlocks::makePTensor, DMRG_routines.cpp:532-537):

    P = contract(conj(psi_f) PL) conj(psi_s) PR,

with PL / PR the overlaps of state p with the current left / right bases
(ProjectorBlocks::move_right_two_vertex / move_left_two_vertex, :540-581:
PL' = psi^dag (PL A)), psi_f / psi_s state p's tensors on the window
(FetchProjectorStatePair / ShiftProjectorStatePair, :446-530, which fold the
centre's singular values into one of them), and the weight w = 100 by
default (command_line_input.hpp:470).

Restatement choices.  The stored state is held as one list of dense site
tensors T[a_in, sigma, a_out] whose product is the state (the centre's
values folded into the left window tensor): any exact representation gives
the same P, so the reference's files and the left / right / lambda naming
are not needed.  The overlaps are rebuilt from the current bases at every
window.  The driver (ExcitedStateFiniteDMRG::init / run,
fDMRG_routines.cpp:68-244) starts from the previous run's superblock at the
centre, solves there (init, fully converged) and sweeps right to the end,
left to the end and right back to the centre, with no prediction vector and
the environment blocks of positions not yet visited taken from the previous
run, as the reference's HBlocksName_ storage does.  Every solve here is
converged to tol; the reference runs the sweep solves with ARPACK capped at
two restarts and tol 0.1 (arpack_interface.cpp:28-29), so only its converged
final rows are comparable.  Its init rows lie below the exact lowest
eigenvalue of the centre window's projected operator as formed here; the
cause is not identified.
"""
import numpy as np

from oracle.dmrg import (EPS, SPARSE_THRESHOLD, SuperBlock, TwoVertexComponents, block_svd, entropy, from_matrix,
                         left_shape, phase_fix, right_shape, run_fdmrg)

DEFAULT_WEIGHT = 100.0


def state_tensors(sb: SuperBlock):
    """The superblock's current state as dense site tensors T[a_in, sigma,
    a_out] (left to right), the centre's values folded into the left window
    tensor.  sb must be mid-sweep with its window at sites nleft+1, nleft+2."""
    T = [left_shape(sb.lmps[k]).data.transpose(1, 0, 2) for k in range(1, sb.nleft + 1)]
    U = left_shape(sb.dec.U).data.transpose(1, 0, 2)          # (a0, sigma1, a1)
    T.append(U * sb.dec.values[None, None, :])
    T.append(right_shape(sb.dec.Vd).data)                     # (a1, sigma2, a2)
    T += [right_shape(sb.rmps[j]).data for j in range(sb.nright, 0, -1)]
    return T


def overlaps(sb: SuperBlock, T):
    """PL[ap, a] and PR[ap, a]: overlaps of the stored state's left / right
    parts (conjugated) with the current left / right bases at the window."""
    PL = np.ones((1, 1), np.complex128)
    for k in range(1, sb.nleft + 1):
        A = left_shape(sb.lmps[k]).data                        # (sigma, a_in, a_out)
        PL = np.einsum("pq,psr,sqa->ra", PL, T[k - 1].conj(), A)
    PR = np.ones((1, 1), np.complex128)
    n = len(T)
    for j in range(1, sb.nright + 1):
        B = right_shape(sb.rmps[j]).data                       # (a_in, sigma, a_out)
        PR = np.einsum("psr,ra,qsa->pq", T[n - j].conj(), PR, B)
    return PL, PR


def p_tensor(sb: SuperBlock, T, h: TwoVertexComponents):
    """makePTensor on the allowed entries of the window (ARPACK order)."""
    PL, PR = overlaps(sb, T)
    T1, T2 = T[sb.nleft], T[sb.nleft + 1]
    P = np.einsum("pa,psr,rtq,qb->satb", PL, T1.conj(), T2.conj(), PR)   # (sigma1, a0, sigma2, a2)
    return P.reshape((h.vrows, h.vcols), order="F").reshape(-1, order="F")[h.allowed]


class ExcitedSuperBlock(SuperBlock):
    """ExcitedStateFiniteDMRG on the oracle's superblock."""

    @classmethod
    def from_superblock(cls, sb: SuperBlock, tol=None):
        ex = cls.__new__(cls)
        ex.__dict__.update(sb.__dict__)
        for k in ("lblocks", "rblocks", "lmps", "rmps"):
            setattr(ex, k, dict(getattr(sb, k)))
        if tol is not None:
            ex.tol = tol
        ex.states = []   # (site tensors, weight) of the projected-out states
        return ex

    def add_state(self, T, weight=DEFAULT_WEIGHT):
        """next_state (fDMRG_routines.hpp:39-44): project out state T."""
        self.states.append((T, float(weight)))

    def _solve(self, L, R, guess):
        # no prediction vector on excited sweeps (fDMRG_routines.cpp:118-121)
        h = TwoVertexComponents(L, self.H, R)
        self.last_heff = h
        ps = [(p_tensor(self, T, h), w) for T, w in self.states]
        n = h.allowed.size
        if n <= SPARSE_THRESHOLD:
            Hd = h.dense()
            for p, w in ps:
                Hd = Hd + w * np.outer(p.conj(), p)
            Hd = 0.5 * (Hd + Hd.conj().T)
            ev, V = np.linalg.eigh(Hd)
            e, vec = float(ev[0]), V[:, 0]
        else:
            from scipy.sparse.linalg import LinearOperator, eigsh

            def mv(x):
                x = np.asarray(x).reshape(-1)
                y = h.matvec(x)
                for p, w in ps:
                    y = y + w * (p @ x) * p.conj()
                return y
            op = LinearOperator((n, n), matvec=mv, dtype=np.complex128)
            v0 = np.ones(n, np.complex128) / np.sqrt(n)
            ev, V = eigsh(op, k=1, which="SA", tol=self.tol, v0=v0, maxiter=100000)
            e, vec = float(ev[0]), V[:, 0]
        small = np.abs(vec) < EPS
        vec = phase_fix(vec)
        vec[small] = 0.0
        full = np.zeros(h.length, np.complex128)
        full[h.allowed] = vec
        theta = from_matrix(self.rules, h.indices, 2, full.reshape((h.vrows, h.vcols), order="F"))
        return e, theta

    def init(self, chi=0, trunc=0.0):
        """ExcitedStateFiniteDMRG::init (fDMRG_routines.cpp:68-91): solve at the
        centre with the current environments."""
        e, theta = self._solve(self.lblocks[self.nleft], self.rblocks[self.nright], None)
        self.dec = block_svd(theta, chi, trunc)
        self.dec.square_rescale(1.0)
        return dict(energy=e, entropy=entropy(self.dec.values), truncation=self.dec.truncation,
                    chi=len(self.dec.values))

    def run(self, sweeps, chi=0, trunc=0.0):
        """ExcitedStateFiniteDMRG::run (fDMRG_routines.cpp:198-242): the init
        row, then the rows at the centre of every sweep."""
        rows = [self.init(chi, trunc)]
        for _ in range(sweeps):
            for _ in range(self.nright, 0, -1):
                self.move_right(chi, trunc)
            for _ in range(self.nleft, 0, -1):
                r = self.move_left(chi, trunc)
                if self.nleft == self.nright:
                    rows.append(r)
            while self.nright > self.nleft:   # back to the centre
                r = self.move_right(chi, trunc)
                if self.nleft == self.nright:
                    rows.append(r)
        return rows


def run_excited_fdmrg(H, nvertices, sweeps, chi, trunc=1e-16, nstates=1, weight=DEFAULT_WEIGHT, target=None,
                      tol=1e-14):
    """fDMRG_DRV -X nstates (fDMRG_DRV.cpp:60-72): the ground-state run, then
    each excited state projected against all earlier ones.  Returns
    (ground-state rows, [rows of excited state 1, ...])."""
    sb, gs_rows = run_fdmrg(H, nvertices, sweeps, chi, trunc, target, tol)
    ex = ExcitedSuperBlock.from_superblock(sb)
    ex.add_state(state_tensors(sb), weight)
    out = []
    for s in range(nstates):
        if s > 0:
            ex.add_state(state_tensors(ex), weight)
        out.append(ex.run(sweeps, chi, trunc))
    return gs_rows, out
