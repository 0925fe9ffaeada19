"""The H_eff matvec and its Lanczos solver sharded across GPUs by output
charge sector.

The reference applies H_eff on one host: ARPACK calls the matvec
(``TwoVertexMPOMPSMultiply``, DMRG_routines.cpp:898-974) with the whole
vector.  Across GPUs the work splits by output sector of the theta layout
(one dense block per middle charge m).  Sectors are dealt to ranks as
contiguous ranges balanced by the executed flops of each output sector, so
each rank's slice of the theta layout is one contiguous range of each plane.
Every rank holds the environments and the MPO (small next to the vectors)
and computes the output sectors it owns.

No rank holds a whole vector.  A rank keeps its owned slice of every Krylov
vector and, per matvec, an input window: the input sectors its owned outputs
read (the library reports them, cmps_heff_input_sectors), packed in
increasing sector order.  The windows are filled by one all-to-all per
matvec in which each rank sends every other rank the owned sectors that rank
reads.  The library reads the window and writes the owned slice directly
(cmps_heff_set_windows).

The Krylov solver works on the owned slices.  Its scalars are all-reduced:
per Lanczos step one all-reduce of the re-orthogonalisation coefficients
(alpha among them) per Gram-Schmidt pass and one of the new norm.  Every rank
therefore sees the same tridiagonal matrix and takes the same decisions.
The eigenvector is post-processed as HED does (DMRG_routines.cpp:870-889):
the phase of its largest entry over all ranks, the drop of entries at or
below eps times that entry, and FixComplexPrecision.

Vectors are (2, len) float64 tensors: the real plane, then the imaginary
plane, as in the theta layout.  The code runs on any torch device and any
``torch.distributed`` backend: NCCL between GPUs, gloo for the host-side
tests.
"""
import numpy as np
import torch
import torch.distributed as dist

EPS = np.finfo(np.float64).eps


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

        # windows (set_needs); by default the whole theta layout
        nsec = self.offsets.size - 1
        self.in_base = self.offsets[:-1].copy()
        self.in_len = self.total
        self.out_base = self.offsets[:-1].copy()
        self.out_len = self.total
        self.needs = None

    @property
    def n_local(self):
        return self.hi - self.lo

    def set_needs(self, needs):
        """Windows from every rank's input sectors: needs is a (world,
        n_sectors) boolean array, row q the sectors rank q's owned outputs
        read.  This rank's input window packs its own row's sectors in
        increasing order; its output window is its owned slice.  Also the
        exchange plan: what this rank sends to and receives from each rank."""
        needs = np.asarray(needs, bool)
        nsec = self.offsets.size - 1
        if needs.shape != (self.world, nsec):
            raise ValueError("one row of input sectors per rank")
        size = np.diff(self.offsets)
        self.needs = needs
        mine = needs[self.rank]
        self.in_base = np.full(nsec, -1, np.int64)
        pos = 0
        for m in range(nsec):
            if mine[m]:
                self.in_base[m] = pos
                pos += int(size[m])
        self.in_len = pos
        self.out_base = np.full(nsec, -1, np.int64)
        self.out_base[self.m0:self.m1] = self.offsets[self.m0:self.m1] - self.lo
        self.out_len = self.n_local
        # send to q: my owned sectors that q reads (local element indices);
        # receive from p: p's owned sectors that I read, which arrive in
        # increasing sector order, i.e. in my window's order
        self.send_idx, self.send_counts, self.recv_counts = [], [], []
        for q in range(self.world):
            idx = [np.arange(self.offsets[m] - self.lo, self.offsets[m + 1] - self.lo)
                   for m in range(self.m0, self.m1) if needs[q, m]]
            idx = np.concatenate(idx) if idx else np.zeros(0, np.int64)
            self.send_idx.append(idx)
            self.send_counts.append(int(idx.size))
        for p, (a, b) in enumerate(self.ranges):
            self.recv_counts.append(int(sum(size[m] for m in range(a, b) if mine[m])))
        if sum(self.recv_counts) != self.in_len:
            raise ValueError("exchange plan does not fill the input window")


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


def gather_needs(need, group=None, device="cpu"):
    """Every rank's input-sector mask, (world, n_sectors) bool, from this
    rank's own (one all-gather at setup)."""
    need = torch.as_tensor(np.asarray(need, np.float64), device=device)
    world = _world(group)
    if world == 1:
        return need.cpu().numpy()[None, :] > 0
    out = [torch.zeros_like(need) for _ in range(world)]
    dist.all_gather(out, need, group=group)
    return np.stack([o.cpu().numpy() for o in out]) > 0


class ShardedOperator:
    """y_local = (H x)[lo:hi] from x_local = x[lo:hi].

    apply_window(xwin, yloc) must write the owned sectors of H x into yloc
    ((2, out_len)) from the input window xwin ((2, in_len)), both laid out as
    the layout's windows say.  On one rank the windows are the whole theta
    layout.  With several ranks the window is filled by one all-to-all of the
    sectors each rank reads (ShardLayout.set_needs must have been called)."""

    def __init__(self, layout, apply_window, device, group=None):
        self.layout = layout
        self.apply_window = apply_window
        self.group = group
        self.world = _world(group)
        if self.world != layout.world:
            raise ValueError("layout and process group have different sizes")
        kw = dict(dtype=torch.float64, device=device)
        self.xwin = torch.zeros(2, max(1, layout.in_len), **kw)
        self.yloc = torch.zeros(2, max(1, layout.out_len), **kw)
        if self.world > 1:
            if layout.needs is None:
                raise ValueError("several ranks: set the layout's input sectors first (set_needs)")
            idx = np.concatenate(layout.send_idx) if layout.send_idx else np.zeros(0, np.int64)
            self.send_idx = torch.as_tensor(idx, dtype=torch.long, device=device)
            self.send = torch.zeros(max(1, idx.size), 2, **kw)
            self.recv = torch.zeros(max(1, layout.in_len), 2, **kw)
        self.matvecs = 0

    def exchange(self, x_local):
        """Fill the input window from the ranks' owned slices."""
        L = self.layout
        if self.world == 1:
            self.xwin[:, :L.in_len].copy_(x_local)
            return self.xwin
        ns = int(self.send_idx.numel())
        if ns:
            self.send[:ns].copy_(x_local.index_select(1, self.send_idx).t())
        dist.all_to_all_single(self.recv[:L.in_len], self.send[:ns], output_split_sizes=L.recv_counts,
                               input_split_sizes=L.send_counts, group=self.group)
        self.xwin[:, :L.in_len].copy_(self.recv[:L.in_len].t())
        return self.xwin

    def __call__(self, x_local):
        self.exchange(x_local)
        self.apply_window(self.xwin, self.yloc)
        self.matvecs += 1
        return self.yloc[:, :self.layout.out_len].clone()


def postprocess(x_local, group=None):
    """HED's eigenvector post-processing (DMRG_routines.cpp:870-889) on a
    sharded vector: the largest-|x| entry over all ranks (ties: the lowest
    rank, then the lowest position) made real positive, entries at or below
    eps times its magnitude dropped, then FixComplexPrecision
    (sparse_interface.cpp:28-32): a part far below the other is zeroed."""
    re, im = x_local[0], x_local[1]
    mag2 = re * re + im * im
    world = _world(group)
    rank = dist.get_rank(group) if world > 1 else 0
    if mag2.numel():
        k = int(torch.argmax(mag2).item())
        cand = torch.tensor([float(mag2[k].item()), float(re[k].item()), float(im[k].item()), float(rank), float(k)],
                            dtype=torch.float64, device=x_local.device)
    else:
        cand = torch.tensor([-1.0, 0.0, 0.0, float(rank), 0.0], dtype=torch.float64, device=x_local.device)
    if world > 1:
        allc = [torch.zeros_like(cand) for _ in range(world)]
        dist.all_gather(allc, cand, group=group)
        rows = [c.cpu().numpy() for c in allc]
    else:
        rows = [cand.cpu().numpy()]
    best = max(rows, key=lambda r: (r[0], -r[3], -r[4]))
    mx2, mr, mi = float(best[0]), float(best[1]), float(best[2])
    out = x_local.clone()
    if mx2 <= 0.0:
        return out
    a = np.sqrt(mx2)
    pr, pi = mr / a, -mi / a  # |mx| / mx
    xr = re * pr - im * pi
    xi = re * pi + im * pr
    keep = torch.sqrt(xr * xr + xi * xi) > EPS * a
    small_im = torch.abs(xi / xr) < EPS  # x / 0 gives inf or nan: not small
    small_re = torch.abs(xr / xi) < EPS
    xi = torch.where(small_im, torch.zeros_like(xi), xi)
    xr = torch.where(~small_im & small_re, torch.zeros_like(xr), xr)
    out[0] = torch.where(keep, xr, torch.zeros_like(xr))
    out[1] = torch.where(keep, xi, torch.zeros_like(xi))
    return out


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
    rank computes the output sectors of its share (cmps_heff_set_owned) from
    the input sectors they read (cmps_heff_set_windows), and the solver works
    on its slice of the theta layout.  Library calls run on torch's current
    stream."""

    def __init__(self, heff, group=None):
        world = _world(group)
        rank = dist.get_rank(group) if world > 1 else 0
        offsets, flops = heff.sector_table()
        self.heff = heff
        self.group = group
        self.layout = ShardLayout(offsets, flops, world, rank)
        if world > 1:
            heff.set_owned(self.layout.owned)
            self.layout.set_needs(gather_needs(heff.input_sectors(), group, "cuda"))
            heff.set_windows(self.layout.in_base, self.layout.in_len, self.layout.out_base, self.layout.out_len)

        def apply_window(xin, yout):
            heff.multiply_theta_device(xin.data_ptr(), yout.data_ptr(), torch_stream_handle())

        self.op = ShardedOperator(self.layout, apply_window, "cuda", group)

    def local_from_arpack(self, x):
        """This rank's slice of a whole vector given in ARPACK order (host or
        device, n_allowed complex): the ARPACK-order vector is placed in the
        theta layout once (setup), then sliced."""
        xa = x if torch.is_tensor(x) else torch.as_tensor(np.asarray(x, np.complex128))
        xa = torch.view_as_real(xa.to("cuda", torch.complex128).contiguous()).contiguous()
        th = torch.empty(2, self.layout.total, dtype=torch.float64, device="cuda")
        self.heff.theta_from_arpack_device(xa.data_ptr(), th.data_ptr(), torch_stream_handle())
        return th[:, self.layout.lo:self.layout.hi].clone()

    def lowest(self, guess=None, tol=1e-10, krylov_dim=24, max_restarts=50):
        """Lowest eigenvalue of H_eff; returns (energy, local eigenvector
        slice after HED's post-processing, matvecs, converged).  guess: whole
        vector in ARPACK order, or None for a seeded start vector identical on
        every rank."""
        if guess is None:
            g = np.random.default_rng(12345).standard_normal((2, self.heff.n))
            guess = g[0] + 1j * g[1]
        x0 = self.local_from_arpack(guess)
        e, x, mv, conv = lanczos_lowest(self.op, x0, self.group, tol, krylov_dim, max_restarts)
        return e, postprocess(x, self.group), mv, conv
