"""The H_eff matvec and its Lanczos solver sharded across GPUs by output
charge sector.

The reference applies H_eff on one host: ARPACK calls the matvec
(``TwoVertexMPOMPSMultiply``, DMRG_routines.cpp:898-974) with the whole
vector.  Across GPUs the work splits by output sector of the theta layout
(one dense block per middle charge m): every rank holds the environments and
the MPO, computes the output sectors it owns from the whole input vector, and
the input vector is re-assembled by one all-gather per matvec.  Sectors are
dealt to ranks as contiguous ranges balanced by the executed flops of each
output sector, so each rank's slice of the theta layout is one contiguous
range of each plane.

The Krylov solver works on the owned slices.  Its scalars are all-reduced:
per Lanczos step one all-reduce of the re-orthogonalisation coefficients
(alpha among them) per Gram-Schmidt pass and one of the new norm.  Every rank
therefore sees the same tridiagonal matrix and takes the same decisions.

Vectors are (2, len) float64 tensors: the real plane, then the imaginary
plane, as in the theta layout.  The code runs on any torch device and any
``torch.distributed`` backend: NCCL between GPUs, gloo for the host-side
tests.
"""
import numpy as np
import torch
import torch.distributed as dist


def partition_sectors(costs, world):
    """Contiguous sector ranges [(m0, m1), ...] (one per rank) balanced by
    cost: the cut before rank r sits at the prefix sum closest to r/world of
    the total, so no rank exceeds total/world by more than the largest
    sector cost.  Ranks past the sector count get empty ranges."""
    costs = np.asarray(costs, np.float64)
    if world < 1:
        raise ValueError("world size must be positive")
    if np.any(costs < 0):
        raise ValueError("sector costs must be non-negative")
    n = costs.size
    cum = np.concatenate([[0.0], np.cumsum(costs)])
    total = cum[-1]
    cuts = [0]
    for r in range(1, world):
        target = total * r / world
        i = min(int(np.searchsorted(cum, target)), n)  # first prefix >= target
        if i > 0 and abs(cum[i - 1] - target) <= abs(cum[i] - target):
            i -= 1
        cuts.append(max(i, cuts[-1]))
    cuts.append(n)
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


class ShardLayout:
    """This rank's share of the theta layout: sectors m0:m1, elements lo:hi
    of each plane; `spans` lists every rank's (lo, hi)."""

    def __init__(self, offsets, costs, world, rank):
        self.offsets = np.asarray(offsets, np.int64)
        nsec = self.offsets.size - 1
        if np.asarray(costs).size != nsec:
            raise ValueError("one cost per sector")
        if np.any(np.diff(self.offsets) < 0):
            raise ValueError("sector offsets must be non-decreasing")
        self.world, self.rank = world, rank
        self.ranges = partition_sectors(costs, world)
        self.spans = [(int(self.offsets[a]), int(self.offsets[b])) for a, b in self.ranges]
        self.m0, self.m1 = self.ranges[rank]
        self.lo, self.hi = self.spans[rank]
        self.total = int(self.offsets[-1])
        self.width = max(1, max(h - l for l, h in self.spans))
        self.owned = np.zeros(nsec, bool)
        self.owned[self.m0:self.m1] = True

    @property
    def n_local(self):
        return self.hi - self.lo


def torch_stream_handle():
    """torch's current CUDA stream as a stream argument of the library.  On
    torch's default stream this is the legacy default stream (handle 1):
    handle 0 would select the library's own non-blocking stream, which is not
    ordered with torch's work."""
    h = torch.cuda.current_stream().cuda_stream
    return h if h else 1


def _world(group):
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(group)
    return 1


def allreduce_sum(t, group=None):
    """In-place sum over the ranks of `group` (a no-op on one rank)."""
    if _world(group) > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t


class ShardedOperator:
    """y_local = (H x)[lo:hi] from x_local = x[lo:hi].

    apply_full(x_full, y_full) must write the owned sectors of H x_full into
    y_full ((2, total) tensors); it may leave the other sectors unwritten.
    The input is re-assembled with one all-gather of equal-width slices."""

    def __init__(self, layout, apply_full, device, group=None):
        self.layout = layout
        self.apply_full = apply_full
        self.group = group
        self.world = _world(group)
        if self.world != layout.world:
            raise ValueError("layout and process group have different sizes")
        kw = dict(dtype=torch.float64, device=device)
        self.xfull = torch.zeros(2, layout.total, **kw)
        self.yfull = torch.zeros(2, layout.total, **kw)
        if self.world > 1:
            self.send = torch.zeros(2, layout.width, **kw)
            self.recv = [torch.zeros(2, layout.width, **kw) for _ in range(self.world)]
        self.matvecs = 0

    def gather(self, x_local):
        L = self.layout
        if self.world == 1:
            self.xfull[:, L.lo:L.hi].copy_(x_local)
            return self.xfull
        self.send[:, :L.n_local].copy_(x_local)
        dist.all_gather(self.recv, self.send, group=self.group)
        for r, (lo, hi) in enumerate(L.spans):
            self.xfull[:, lo:hi].copy_(self.recv[r][:, :hi - lo])
        return self.xfull

    def __call__(self, x_local):
        self.gather(x_local)
        self.apply_full(self.xfull, self.yfull)
        self.matvecs += 1
        return self.yfull[:, self.layout.lo:self.layout.hi].clone()


def _coeffs(V, w):
    """<V_i | w> for the rows of V ((k, 2, n) planar) -> (2, k): re, im."""
    re = torch.einsum("kn,n->k", V[:, 0], w[0]) + torch.einsum("kn,n->k", V[:, 1], w[1])
    im = torch.einsum("kn,n->k", V[:, 0], w[1]) - torch.einsum("kn,n->k", V[:, 1], w[0])
    return torch.stack([re, im])


def _subtract(w, V, c):
    """w -= sum_i c_i V_i (complex c given as (2, k))."""
    w[0] -= torch.einsum("k,kn->n", c[0], V[:, 0]) - torch.einsum("k,kn->n", c[1], V[:, 1])
    w[1] -= torch.einsum("k,kn->n", c[0], V[:, 1]) + torch.einsum("k,kn->n", c[1], V[:, 0])


def _norm(x, group):
    s = (x * x).sum().reshape(1)
    return float(allreduce_sum(s, group).sqrt().item())


def lanczos_lowest(op, x0_local, group=None, tol=1e-10, krylov_dim=24, max_restarts=50):
    """Lowest eigenpair of the Hermitian operator `op` on sharded vectors:
    restarted Lanczos with full re-orthogonalisation (two classical
    Gram-Schmidt passes) from x0_local, converged when the residual norm
    beta_k |y_k| <= tol |theta|.  Returns (theta, x_local normalised over all
    ranks, matvec count, converged)."""
    x = x0_local.clone()
    nrm = _norm(x, group)
    if nrm == 0.0:
        raise ValueError("zero start vector")
    kdim = max(2, int(krylov_dim))
    dev = x.device
    mv = 0
    theta = float("nan")
    converged = False
    for _ in range(max(1, int(max_restarts))):
        V = torch.zeros(kdim + 1, 2, x.shape[1], dtype=torch.float64, device=dev)
        V[0] = x / nrm
        alpha, beta = [], []
        y = np.ones(1)
        for j in range(kdim):
            w = op(V[j])
            mv += 1
            a = None
            for p in range(2):
                c = allreduce_sum(_coeffs(V[:j + 1], w), group)
                if p == 0:
                    a = float(c[0, j].item())
                _subtract(w, V[:j + 1], c)
            b = _norm(w, group)
            alpha.append(a)
            T = np.diag(alpha) + np.diag(beta, 1) + np.diag(beta, -1)
            ev, evec = np.linalg.eigh(T)
            theta, y = float(ev[0]), evec[:, 0]
            if b * abs(y[-1]) <= tol * max(abs(theta), 1e-300) or b <= 1e-300:
                converged = True
                break
            if j + 1 < kdim:
                beta.append(b)
                V[j + 1] = w / b
        k = len(alpha)
        yt = torch.as_tensor(y, dtype=torch.float64, device=dev)
        x = torch.einsum("k,kcn->cn", yt, V[:k])
        nrm = _norm(x, group)
        if converged:
            break
    return theta, x / nrm, mv, converged


class ShardedTwoVertex:
    """A TwoVertexComponents handle sharded over the ranks of `group`: this
    rank computes the output sectors of its share (cmps_heff_set_owned) and
    the solver works on its slice of the theta layout.  Library calls run on
    torch's current stream."""

    def __init__(self, heff, group=None):
        world = _world(group)
        rank = dist.get_rank(group) if world > 1 else 0
        offsets, flops = heff.sector_table()
        self.heff = heff
        self.group = group
        self.layout = ShardLayout(offsets, flops, world, rank)
        if world > 1:
            heff.set_owned(self.layout.owned)

        def apply_full(xin, yout):
            heff.multiply_theta_device(xin.data_ptr(), yout.data_ptr(), torch_stream_handle())

        self.op = ShardedOperator(self.layout, apply_full, "cuda", group)

    def local_from_arpack(self, x):
        """This rank's slice of a whole vector given in ARPACK order (host or
        device, n_allowed complex)."""
        xa = x if torch.is_tensor(x) else torch.as_tensor(np.asarray(x, np.complex128))
        xa = torch.view_as_real(xa.to("cuda", torch.complex128).contiguous()).contiguous()
        th = torch.empty(2, self.layout.total, dtype=torch.float64, device="cuda")
        self.heff.theta_from_arpack_device(xa.data_ptr(), th.data_ptr(), torch_stream_handle())
        return th[:, self.layout.lo:self.layout.hi].clone()

    def lowest(self, guess=None, tol=1e-10, krylov_dim=24, max_restarts=50):
        """Lowest eigenvalue of H_eff; returns (energy, local eigenvector
        slice, matvecs, converged).  guess: whole vector in ARPACK order, or
        None for a seeded start vector identical on every rank."""
        if guess is None:
            g = np.random.default_rng(12345).standard_normal((2, self.heff.n))
            guess = g[0] + 1j * g[1]
        x0 = self.local_from_arpack(guess)
        return lanczos_lowest(self.op, x0, self.group, tol, krylov_dim, max_restarts)
