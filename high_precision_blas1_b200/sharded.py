"""Compensated reductions over a vector sharded across GPUs (one process
per GPU, ``torch.distributed`` over NCCL).

The vector of global length n is split in contiguous slices, rank r owning
``partition(n, world, r)``.  Element-wise operations need no exchange: each
rank runs the single-GPU kernels on its slice.  A reduction takes one
exchange step:

1. the rank reduces its slice with the single-GPU kernel (``hpb_dot2_*``,
   ``hpb_sum2_*``, ``hpb_asum2_*``), leaving one (hi, lo) result -- 2
   doubles, 4 for a complex result -- in device memory;
2. ``all_gather_into_tensor`` collects the world's results (16 or 32 bytes
   per rank over NVLink) on every rank, in rank order;
3. ``hpb_shard_merge`` merges them in rank order with the compensated
   recurrence of the reference's second reduction pass, one device thread,
   on the same stream.

Every rank ends with the same bits, whatever order the ranks finish in;
the result stays within the Ogita-Rump-Oishi bound of the whole-vector Dot2
(the merge adds world-1 compensated additions to the single-GPU combine).
An all-reduce(sum) would drop the error terms and has no specified order.

The reference runs on one GPU and has no sharded reductions; the
single-GPU entry points replaced are ``gpu_reduction_ogita<T>::dot / sum /
asum / norm`` (common/ogita/gpu_reduction_ogita.h:74-96).

There is no CPU compute path: the reductions and the merge run in
libhpblas1.so on the GPU.  ``merge_gathered_cpu`` (the host build of the
same merge, ``hpb_shard_merge_cpu``) serves callers whose exchange gathers
to host memory, e.g. a gloo process group.
"""
from __future__ import annotations

import numpy as np

from . import Context, load

_RED = {  # (name, complex result)
    ("dot", "f32"): ("hpb_dot2_f32", False), ("dot", "f64"): ("hpb_dot2_f64", False),
    ("dot", "c64"): ("hpb_dot2_c64", True), ("dot", "c128"): ("hpb_dot2_c128", True),
    ("sum", "f32"): ("hpb_sum2_f32", False), ("sum", "f64"): ("hpb_sum2_f64", False),
    ("sum", "c64"): ("hpb_sum2_c64", True), ("sum", "c128"): ("hpb_sum2_c128", True),
    ("asum", "f32"): ("hpb_asum2_f32", False), ("asum", "f64"): ("hpb_asum2_f64", False),
    ("asum", "c64"): ("hpb_asum2_c64", False), ("asum", "c128"): ("hpb_asum2_c128", False),
}


def partition(n: int, world: int, rank: int) -> tuple[int, int]:
    """[lo, hi) of rank's contiguous slice: the first n % world ranks hold
    one element more than the others."""
    if n < 0 or world < 1 or not 0 <= rank < world:
        raise ValueError("partition: need n >= 0, world >= 1, 0 <= rank < world")
    q, r = divmod(n, world)
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)


def merge_gathered_cpu(parts: np.ndarray, is_complex: bool) -> np.ndarray:
    """Merge gathered results (count x 2, or count x 4 complex, float64, in
    rank order) on the host with hpb_shard_merge_cpu."""
    L = load().lib
    comps = 2 if is_complex else 1
    a = np.ascontiguousarray(parts, dtype=np.float64).reshape(-1)
    if a.size == 0 or a.size % (2 * comps):
        raise ValueError("merge_gathered_cpu: need count >= 1 results of 2 (real) or 4 (complex) doubles")
    out = np.empty(2 * comps)
    st = L.hpb_shard_merge_cpu(a.size // (2 * comps), int(is_complex), a.ctypes.data, out.ctypes.data)
    if st != 0:
        raise load().HpbError(st, "hpb_shard_merge_cpu")
    return out


def value_of(res, is_complex: bool):
    """hi of a merged result (the rounded compensated value, as the
    reference's reductions return it)."""
    r = [float(v) for v in res]
    return complex(r[0], r[1]) if is_complex else r[0]


class ShardedReductions:
    """Dot2 / Sum2 / asum2 / norm of vectors sharded over the ranks of
    ``group`` (NCCL), one GPU per rank.  ``x`` and ``y`` are this rank's
    slices: CUDA tensors of the element type (float32, float64, complex64,
    complex128), contiguous, on this rank's device.  Calls are ordered on
    torch's current stream and return host scalars (like the reference's
    by-value reductions, gpu_vector_operations.h:257-340)."""

    def __init__(self, device: int, group=None):
        import torch
        import torch.distributed as dist
        self._torch, self._dist = torch, dist
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.device = torch.device("cuda", device)
        self.stream = torch.cuda.current_stream(self.device)
        self.ctx = Context(device, self.stream.cuda_stream)
        self.L = load().lib
        self._local = torch.zeros(4, dtype=torch.float64, device=self.device)
        self._gathered = torch.zeros(4 * self.world, dtype=torch.float64, device=self.device)
        self._out = torch.zeros(4, dtype=torch.float64, device=self.device)

    @staticmethod
    def _type(t) -> str:
        import torch
        m = {torch.float32: "f32", torch.float64: "f64", torch.complex64: "c64", torch.complex128: "c128"}
        if t.dtype not in m:
            raise TypeError(f"unsupported element type {t.dtype}")
        return m[t.dtype]

    def _check(self, *ts):
        for t in ts:
            if not t.is_cuda or t.device != self.device or not t.is_contiguous():
                raise ValueError("sharded reductions take contiguous CUDA tensors on this rank's device")
        if len(ts) == 2 and (ts[0].numel() != ts[1].numel() or ts[0].dtype != ts[1].dtype):
            raise ValueError("x and y differ in length or element type")

    def _reduce(self, op: str, x, y=None):
        self._check(*((x,) if y is None else (x, y)))
        t = self._type(x)
        name, cplx = _RED[(op, t)]
        width = 4 if cplx else 2
        f = getattr(self.L, name)
        check_stream_and_device(self)
        args = (self.ctx.h, x.numel(), x.data_ptr()) + (() if y is None else (y.data_ptr(),))
        self.ctx.check(f(*args, self._local.data_ptr()), name)
        local = self._local[:width]
        gathered = self._gathered[:width * self.world]
        if self._dist.is_initialized():
            self._dist.all_gather_into_tensor(gathered, local, group=self.group)
        else:
            gathered.copy_(local)
        self.ctx.check(self.L.hpb_shard_merge(self.ctx.h, self.world, int(cplx), gathered.data_ptr(),
                                              self._out.data_ptr()), "hpb_shard_merge")
        return self._out[:width].cpu().numpy(), cplx

    def dot(self, x, y):
        """sum_i conj(x_i) y_i over the whole vector (Dot2)."""
        res, cplx = self._reduce("dot", x, y)
        return value_of(res, cplx)

    def sum(self, x):
        """sum_i x_i (Sum2)."""
        res, cplx = self._reduce("sum", x)
        return value_of(res, cplx)

    def asum(self, x):
        """sum_i |x_i| (real), sum_i |re_i| + |im_i| (complex), compensated."""
        res, cplx = self._reduce("asum", x)
        return value_of(res, cplx)

    def norm(self, x):
        """sqrt(Re Dot2(x, x)) over the whole vector."""
        res, cplx = self._reduce("dot", x, x)
        return float(np.sqrt(res[0]))

    def result(self, op: str, x, y=None) -> np.ndarray:
        """The merged (hi, lo) result itself (2 doubles; 4 for complex)."""
        return self._reduce(op, x, y)[0]

    def close(self):
        self.ctx.close()


def torch_stream_changed(obj) -> bool:
    return obj._torch.cuda.current_stream(obj.device).cuda_stream != obj.stream.cuda_stream


def check_stream_and_device(obj) -> None:
    """The library's kernels run on the stream saved at construction, and the
    NCCL collectives on torch's current stream of the current device: the two
    are ordered only while they are the same stream."""
    if obj._torch.cuda.current_device() != obj.device.index:
        raise RuntimeError("torch's current device differs from the one this object was made on")
    if torch_stream_changed(obj):
        raise RuntimeError("torch's current stream changed since this object was made")


# --------------------------------------------------------------- sparse operator
def owner_of(cols: np.ndarray, n: int, world: int) -> np.ndarray:
    """Rank owning each global index under partition(n, world, .)."""
    starts = np.array([partition(n, world, r)[0] for r in range(world)] + [n], dtype=np.int64)
    return np.searchsorted(starts, np.asarray(cols, dtype=np.int64), side="right") - 1


class HaloPlan:
    """Row block of a square CSR operator split like the vectors: rank r owns
    rows and x entries partition(n, world, r).  Each stored column index is
    renumbered into this rank's extended vector x_ext = [own slice | halo]:
    an own column c becomes c - lo, a column owned by another rank becomes
    n_own + its position in ``halo`` (the needed remote indices, sorted by
    owner and then by index, so each owner's entries arrive as one
    contiguous segment).  Entries keep their order inside a row, so the
    row sums run in the same order as on one GPU.

    ``send_index`` / ``send_counts`` say which own entries (local indices,
    grouped by destination rank in rank order) this rank sends to the others
    at every product; they are known once every rank's ``requests`` have been
    exchanged (``finish``)."""

    def __init__(self, row_ptr, col_ind, n: int, world: int, rank: int):
        self.n, self.world, self.rank = n, world, rank
        self.lo, self.hi = partition(n, world, rank)
        self.rows = self.hi - self.lo
        rp = np.asarray(row_ptr, dtype=np.int64)
        ci = np.asarray(col_ind, dtype=np.int64)
        if rp.shape[0] != self.rows + 1 or rp[0] != 0 or rp[-1] != ci.shape[0]:
            raise ValueError("HaloPlan: row_ptr must hold this rank's rows, starting at 0")
        if ci.size and (ci.min() < 0 or ci.max() >= n):
            raise ValueError("HaloPlan: column index out of range")
        own = (ci >= self.lo) & (ci < self.hi)
        remote = np.unique(ci[~own])  # sorted by index, hence by owner
        self.halo = remote
        self.recv_counts = np.bincount(owner_of(remote, n, world), minlength=world).astype(np.int64) \
            if remote.size else np.zeros(world, dtype=np.int64)
        loc = np.empty_like(ci)
        loc[own] = ci[own] - self.lo
        loc[~own] = self.rows + np.searchsorted(remote, ci[~own])
        self.row_ptr = rp.astype(np.int32)
        self.col_ind = loc.astype(np.int32)
        self.cols = self.rows + int(remote.size)
        owners = owner_of(remote, n, world) if remote.size else np.zeros(0, dtype=np.int64)
        # requests[s]: the global indices this rank needs from rank s
        self.requests = [remote[owners == s] for s in range(world)]
        self.send_index = None
        self.send_counts = None

    def finish(self, requests_to_me):
        """requests_to_me[s]: the global indices rank s needs from this rank."""
        parts = []
        for s, req in enumerate(requests_to_me):
            req = np.asarray(req, dtype=np.int64)
            if req.size and (req.min() < self.lo or req.max() >= self.hi):
                raise ValueError(f"HaloPlan: rank {s} requests indices this rank does not own")
            if s == self.rank and req.size:
                raise ValueError("HaloPlan: a rank requested its own entries")
            parts.append(req - self.lo)
        self.send_counts = np.array([p.size for p in parts], dtype=np.int64)
        self.send_index = (np.concatenate(parts) if parts else np.zeros(0, dtype=np.int64)).astype(np.int32)
        return self

    def exchange_requests(self, group=None):
        """All ranks' requests through torch.distributed (once per operator)."""
        import torch.distributed as dist
        everyone = [None] * self.world
        dist.all_gather_object(everyone, [r.tolist() for r in self.requests], group=group)
        return self.finish([everyone[s][self.rank] for s in range(self.world)])


class ShardedCSR:
    """y = A x for a square CSR operator whose rows and vectors are split
    over the ranks (one GPU each) as ``partition`` says.  Per product: the
    entries other ranks need are gathered on the device (hpb_gather_*), one
    ``all_to_all_single`` over NCCL moves them into the halo of the extended
    vector, the own slice is copied in front of the halo (hpb_copy), and the
    row block's SpMV (hpb_csr_spmv_*) runs on the extended vector.  The
    result equals the single-GPU SpMV's rows bit for bit.

    The reference has no sharded operator; the single-GPU operator replaced
    is csr::gpu_matrix::axpy (common/csr/gpu_matrix.h:322-375).

    Construction without a ``plan`` exchanges the halo requests with
    ``all_gather_object``, which NCCL runs on the current CUDA device: call
    ``torch.cuda.set_device(device)`` on every rank first."""

    _T = {"float32": "f32", "float64": "f64", "complex64": "c64", "complex128": "c128"}

    def __init__(self, device: int, row_ptr, col_ind, val, n: int, group=None, plan: HaloPlan | None = None):
        import torch
        import torch.distributed as dist
        self._torch, self._dist, self.group = torch, dist, group
        world = dist.get_world_size(group) if dist.is_initialized() else 1
        rank = dist.get_rank(group) if dist.is_initialized() else 0
        if plan is None:
            plan = HaloPlan(row_ptr, col_ind, n, world, rank)
            plan = plan.exchange_requests(group) if world > 1 else plan.finish([np.zeros(0)] * world)
        self.plan = plan
        self.device = torch.device("cuda", device)
        self.stream = torch.cuda.current_stream(self.device)
        self.ctx = Context(device, self.stream.cuda_stream)
        self.L = load().lib
        v = np.ascontiguousarray(val)
        self.t = self._T[str(v.dtype)]
        self.elem = v.dtype.itemsize
        d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(self.device)
        self.rp, self.ci, self.val = d(plan.row_ptr), d(plan.col_ind), d(v)
        self.send_index = d(plan.send_index)
        tdt = getattr(torch, str(v.dtype))
        self.send_buf = torch.zeros(max(1, int(plan.send_counts.sum())), dtype=tdt, device=self.device)
        self.x_ext = torch.zeros(max(1, plan.cols), dtype=tdt, device=self.device)
        self._one = load().scalar(self.t, 1.0)
        self._zero = load().scalar(self.t, 0.0)

    def gather_send(self, x_local):
        n_send = int(self.plan.send_counts.sum())
        if n_send:
            f = getattr(self.L, f"hpb_gather_{self.t}")
            self.ctx.check(f(self.ctx.h, n_send, self.send_index.data_ptr(), x_local.data_ptr(),
                             self.send_buf.data_ptr()), "hpb_gather")

    def exchange(self):
        p = self.plan
        check_stream_and_device(self)
        if p.world > 1:
            self._dist.all_to_all_single(self.x_ext[p.rows:p.cols], self.send_buf[:int(p.send_counts.sum())],
                                         output_split_sizes=p.recv_counts.tolist(),
                                         input_split_sizes=p.send_counts.tolist(), group=self.group)

    def local_spmv(self, x_local, y_local):
        p = self.plan
        if p.rows:
            self.ctx.check(self.L.hpb_copy(self.ctx.h, p.rows, self.elem, x_local.data_ptr(), self.x_ext.data_ptr()),
                           "hpb_copy")
        f = getattr(self.L, f"hpb_csr_spmv_{self.t}")
        self.ctx.check(f(self.ctx.h, p.rows, p.cols, int(p.col_ind.size), self.rp.data_ptr(), self.ci.data_ptr(),
                         self.val.data_ptr(), self._one, self.x_ext.data_ptr(), self._zero, y_local.data_ptr()),
                       "hpb_csr_spmv")

    def apply(self, x_local, y_local):
        """y_local = (A x) on this rank's rows; x_local, y_local: this rank's
        slices (contiguous CUDA tensors of the operator's element type)."""
        for t in (x_local, y_local):
            if not t.is_cuda or t.device != self.device or not t.is_contiguous() or t.numel() != self.plan.rows:
                raise ValueError("ShardedCSR.apply takes this rank's contiguous slices on its device")
        check_stream_and_device(self)
        self.gather_send(x_local)
        self.exchange()
        self.local_spmv(x_local, y_local)

    def close(self):
        self.ctx.close()


# ----------------------------------------------------------------- solver
class ShardedVectorOps:
    """Vector operations on this rank's float64 slices for ``bicgstabl``:
    element-wise work in the library's kernels (hpb_axpby_f64, hpb_copy,
    hpb_fill_f64), dot products and norms through ``ShardedReductions``
    (identical on every rank).  The operations mirror the reference's
    vector-operations concept (add_mul, assign, assign_scalar, scalar_prod,
    norm; common/gpu_vector_operations.h:257-462)."""

    def __init__(self, reductions: ShardedReductions, n_local: int):
        self.red, self.n = reductions, n_local
        self.ctx, self.L = reductions.ctx, reductions.L
        self._torch = reductions._torch

    def new(self):
        return self._torch.zeros(self.n, dtype=self._torch.float64, device=self.red.device)

    def dot(self, x, y) -> float:
        return self.red.dot(x, y)

    def norm(self, x) -> float:
        return self.red.norm(x)

    def axpby(self, a: float, x, b: float, y):
        """y := a x + b y"""
        self.ctx.check(self.L.hpb_axpby_f64(self.ctx.h, self.n, a, x.data_ptr(), b, y.data_ptr()), "hpb_axpby_f64")

    def copy(self, x, y):
        self.ctx.check(self.L.hpb_copy(self.ctx.h, self.n, 8, x.data_ptr(), y.data_ptr()), "hpb_copy")

    def fill(self, y, v: float):
        self.ctx.check(self.L.hpb_fill_f64(self.ctx.h, self.n, v, y.data_ptr()), "hpb_fill_f64")


def bicgstabl(ops, A, b, x, L: int = 2, rel_tol: float = 1e-10, max_iters: int = 10000):
    """BiCGStab(l) on vectors split across ranks: the Sleijpen-Fokkema
    recurrences of the reference's numerical_algos/lin_solvers/bicgstabl.h
    (cycle :196-265: BiCG part :198-222, MR part with modified Gram-Schmidt
    :223-258) with
    its monitor's test ||r_0|| <= rel_tol ||b|| once per cycle
    (default_monitor.h:202-226), unpreconditioned.  ``ops`` supplies new,
    dot, norm, axpby (y := a x + b y), copy and fill on this rank's slices;
    ``A.apply(x, y)`` the row block of y = A x.  With complex vectors
    ops.dot(x, y) = sum conj(x_i) y_i, and every inner product puts the
    conjugated vector on the left (rho = (rt, r_j), (rt, u_{j+1}),
    tau = (r_i, r_j), gamma' = (r_j, r_0)), as the library's solvers do:
    the reference's order (bicgstabl.h:207, :216, :226, :230) conjugates
    these scalars, which breaks the complex iteration; on real data both
    orders give the same bits.  Every scalar comes from a
    reduction that every rank holds bit for bit, so all ranks take the same
    branches.  x holds the initial guess and receives the solution.
    Returns (converged, iterations, ||r_0|| / ||b||)."""
    if L < 1:
        raise ValueError("bicgstabl: basis size must be >= 1")
    r = [ops.new() for _ in range(L + 1)]
    u = [ops.new() for _ in range(L + 1)]
    rt = ops.new()
    bnorm = ops.norm(b)
    A.apply(x, r[0])
    ops.axpby(1.0, b, -1.0, r[0])  # r_0 = b - A x
    ops.copy(r[0], rt)
    ops.axpby(0.0, r[0], 1.0 / ops.norm(rt), rt)  # rt = r_0 / ||r_0||
    ops.fill(u[0], 0.0)
    sigma, gam, gam1, gam2 = ([0.0] * (L + 1) for _ in range(4))
    tau = [[0.0] * (L + 1) for _ in range(L + 1)]
    rho, alpha, omega = 1.0, 0.0, 1.0
    it = 0
    rnorm = ops.norm(r[0])
    while True:
        if not np.isfinite(rnorm):
            return False, it, float("nan")
        if rnorm <= rel_tol * bnorm:
            return True, it, rnorm / bnorm
        if it >= max_iters:
            return False, it, rnorm / bnorm
        rho = -omega * rho
        for j in range(L):
            if rho == 0.0:
                return False, it, rnorm / bnorm  # breakdown
            rho1 = ops.dot(rt, r[j])
            beta = alpha * rho1 / rho
            rho = rho1
            for i in range(j + 1):
                ops.axpby(1.0, r[i], -beta, u[i])  # u_i = r_i - beta u_i
            A.apply(u[j], u[j + 1])
            alpha = rho / ops.dot(rt, u[j + 1])
            for i in range(j + 1):
                ops.axpby(-alpha, u[i + 1], 1.0, r[i])  # r_i -= alpha u_{i+1}
            A.apply(r[j], r[j + 1])
            ops.axpby(alpha, u[0], 1.0, x)
        for j in range(1, L + 1):
            for i in range(1, j):
                tau[i][j] = ops.dot(r[i], r[j]) / sigma[i]
                ops.axpby(-tau[i][j], r[i], 1.0, r[j])
            sigma[j] = ops.dot(r[j], r[j])
            gam1[j] = ops.dot(r[j], r[0]) / sigma[j]
        gam[L] = gam1[L]
        omega = gam[L]
        for j in range(L - 1, 0, -1):
            g = gam1[j]
            for i in range(j + 1, L + 1):
                g -= tau[j][i] * gam[i]
            gam[j] = g
        for j in range(1, L):
            g = gam[j + 1]
            for i in range(j + 1, L):
                g += tau[j][i] * gam[i + 1]
            gam2[j] = g
        ops.axpby(gam[1], r[0], 1.0, x)
        ops.axpby(-gam1[L], r[L], 1.0, r[0])
        ops.axpby(-gam[L], u[L], 1.0, u[0])
        for j in range(1, L):
            ops.axpby(gam2[j], r[j], 1.0, x)
            ops.axpby(-gam1[j], r[j], 1.0, r[0])
            ops.axpby(-gam[j], u[j], 1.0, u[0])
        it += L
        rnorm = ops.norm(r[0])


def _make_rotation(dx: float, dy: float):
    if dy == 0.0:
        return 1.0, 0.0
    if abs(dy) > abs(dx):
        t = dx / dy
        sn = 1.0 / np.sqrt(1.0 + t * t)
        return t * sn, sn
    t = dy / dx
    cs = 1.0 / np.sqrt(1.0 + t * t)
    return cs, t * cs


def _rotate(dx: float, dy: float, cs: float, sn: float):
    return cs * dx + sn * dy, -sn * dx + cs * dy


def gmres(ops, A, b, x, m: int = 30, rel_tol: float = 1e-10, max_iters: int = 10000, reorthogonalize: bool = False):
    """Restarted GMRES(m) on vectors split across ranks, real binary64: the
    reference's numerical_algos/lin_solvers/gmres.h (restart loop :412-484;
    modified Gram-Schmidt with optional reorthogonalisation :426-452; Givens
    rotations :224-273, applied on the host to the rank-identical Hessenberg
    entries), unpreconditioned, with the monitor's test
    ||b - A x|| <= rel_tol ||b|| at every restart (default_monitor.h:202-226).
    ``ops`` and ``A`` as for ``bicgstabl``.  Returns (converged, iterations,
    ||b - A x|| / ||b||).

    ``reorthogonalize`` applies ONE correction per basis vector (classical
    "twice is enough" re-orthogonalisation).  The reference's loop
    (gmres.h:431-447) repeats the correction while |alpha| > 1e-10 sqrt(N), up
    to 11 times, but tests the accumulated coefficient alpha rather than the
    correction c, so it runs all 11 corrections whenever the projection
    itself is not tiny; the single pass is the intended method."""
    if m < 1:
        raise ValueError("gmres: basis size must be >= 1")
    V = [ops.new() for _ in range(m + 1)]
    r = ops.new()
    bnorm = ops.norm(b)

    def residual():
        A.apply(x, r)
        ops.axpby(1.0, b, -1.0, r)  # r = b - A x
        return ops.norm(r)

    it = 0
    rnorm = residual()
    while True:
        if not np.isfinite(rnorm):
            return False, it, float("nan")
        if rnorm <= rel_tol * bnorm:
            return True, it, rnorm / bnorm
        if it >= max_iters:
            return False, it, rnorm / bnorm
        ops.copy(r, V[0])
        ops.axpby(0.0, r, 1.0 / rnorm, V[0])  # V_0 = r / ||r||
        H = np.zeros((m + 1, m))
        s = np.zeros(m + 1)
        cs = np.zeros(m)
        sn = np.zeros(m)
        s[0] = rnorm
        i = -1
        while i + 1 < m:
            i += 1
            it += 1
            A.apply(V[i], V[i + 1])
            for k in range(i + 1):  # modified Gram-Schmidt
                a = ops.dot(V[k], V[i + 1])
                ops.axpby(-a, V[k], 1.0, V[i + 1])
                if reorthogonalize:
                    c = ops.dot(V[k], V[i + 1])
                    ops.axpby(-c, V[k], 1.0, V[i + 1])
                    a += c
                H[k, i] = a
            hn = ops.norm(V[i + 1])
            H[i + 1, i] = hn
            if hn > 0.0:
                ops.axpby(0.0, V[i + 1], 1.0 / hn, V[i + 1])
            for k in range(i):
                H[k, i], H[k + 1, i] = _rotate(H[k, i], H[k + 1, i], cs[k], sn[k])
            cs[i], sn[i] = _make_rotation(H[i, i], H[i + 1, i])
            H[i, i], H[i + 1, i] = _rotate(H[i, i], H[i + 1, i], cs[i], sn[i])
            H[i + 1, i] = 0.0
            s[i], s[i + 1] = _rotate(s[i], s[i + 1], cs[i], sn[i])
            if hn == 0.0:  # happy breakdown: the Krylov space is invariant
                break
        y = s.copy()
        for j in range(i, -1, -1):
            y[j] /= H[j, j]
            for k in range(j - 1, -1, -1):
                y[k] -= H[k, j] * y[j]
        for j in range(i + 1):
            ops.axpby(float(y[j]), V[j], 1.0, x)
        rnorm = residual()
