"""Independent FMM work split over ranks (one process per GPU).

The reference has no distributed code and solves one problem per object.
Two of its workloads split with no exchange between ranks:

* a list of independent problems -- the batched Stokes workload, one FMM per
  problem (flexmm/kifmm2d/vector/stokes_fmm.py:598-858): the problems are
  partitioned by cost (points) over the ranks, each rank runs its share;
* the charge columns of a multi-RHS build -- kifmm2d's tau[k, N]
  (flexmm/kifmm2d/scalar/fmm.py:73-124): every rank builds the same tree
  (the tree depends on the sources only) and forms and evaluates its own
  block of columns.

Each rank computes alone; one all-gather at the end hands every rank all
results in the caller's order (NCCL over NVLink between GPUs, gloo between
CPU processes).  The all-gather carries float64 results only: the partition
is a pure function of the problem sizes and the world size, so every rank
knows every piece's length without exchanging it.  Every rank takes the same
collective steps in the same order.
"""
import numpy as np


def partition_by_cost(costs, world):
    """Problem indices per rank: longest-processing-time greedy on ``costs``
    (the largest problem first, each to the currently least loaded rank, ties
    to the lower rank), each rank's list in ascending index order.
    Deterministic, so every rank computes the same partition."""
    costs = np.asarray(costs, dtype=np.float64)
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(costs.size), key=lambda i: (-costs[i], i))
    load = np.zeros(world)
    parts = [[] for _ in range(world)]
    for i in order:
        r = int(np.argmin(load))   # first minimum: the lower rank on ties
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def column_blocks(k, world):
    """Contiguous column ranges [lo, hi) per rank, sizes differing by at most one."""
    base, extra = divmod(int(k), int(world))
    out, lo = [], 0
    for r in range(world):
        hi = lo + base + (1 if r < extra else 0)
        out.append((lo, hi))
        lo = hi
    return out


def _dist():
    import torch.distributed as dist
    return dist


def world_and_rank(group=None):
    dist = _dist()
    if not dist.is_available() or not dist.is_initialized():
        return 1, 0
    return dist.get_world_size(group), dist.get_rank(group)


def all_gather_pieces(local, lengths, parts, group=None):
    """All-gather float64 pieces whose lengths every rank knows.

    ``parts[r]`` lists the piece ids rank r owns (in its send order),
    ``lengths[i]`` is piece i's length, ``local`` is this rank's pieces in
    ``parts[rank]`` order (tensors or arrays of shape [lengths[i]]).
    Returns every piece, by id, as a CPU float64 numpy array.  One
    all_gather of equal-sized padded buffers (on the GPU for NCCL)."""
    import torch
    world, rank = world_and_rank(group)
    lengths = [int(v) for v in lengths]
    tot = [sum(lengths[i] for i in p) for p in parts]
    if world == 1:
        return {i: np.asarray(_cpu(t), dtype=np.float64).reshape(-1) for i, t in zip(parts[0], local)}
    dist = _dist()
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
        else torch.device("cpu")
    width = max(max(tot), 1)
    send = torch.zeros(width, dtype=torch.float64, device=dev)
    at = 0
    for i, t in zip(parts[rank], local):
        v = torch.as_tensor(t, dtype=torch.float64).reshape(-1).to(dev)
        if v.numel() != lengths[i]:
            raise ValueError(f"piece {i}: {v.numel()} values, expected {lengths[i]}")
        send[at:at + v.numel()] = v
        at += v.numel()
    recv = torch.empty(world * width, dtype=torch.float64, device=dev)
    dist.all_gather_into_tensor(recv, send, group=group)
    host = recv.cpu().numpy()
    out = {}
    for r in range(world):
        at = r * width
        for i in parts[r]:
            out[i] = host[at:at + lengths[i]].copy()
            at += lengths[i]
    return out


def _cpu(t):
    try:
        import torch
        if isinstance(t, torch.Tensor):
            return t.detach().cpu().numpy()
    except ImportError:
        pass
    return t


def run_sharded(costs, compute, pieces_of, lengths_of, group=None):
    """Partition items by ``costs`` over the ranks, run ``compute(indices)`` on
    this rank's items (it returns one result per item), flatten each result
    into pieces with ``pieces_of(result)`` (a list of 1-D arrays, their
    lengths ``lengths_of(i)`` for item i), and all-gather.  Returns, for every
    item in the caller's order, the list of its pieces."""
    world, rank = world_and_rank(group)
    parts = partition_by_cost(costs, world)
    mine = parts[rank]
    results = compute(mine) if mine else []
    n_per = [len(lengths_of(i)) for i in range(len(costs))]
    # piece ids: item i's j-th piece is sum(n_per[:i]) + j
    first = np.concatenate([[0], np.cumsum(n_per)]).astype(int)
    lengths = [ln for i in range(len(costs)) for ln in lengths_of(i)]
    piece_parts = [[int(first[i]) + j for i in p for j in range(n_per[i])] for p in parts]
    local = [pc for res in results for pc in pieces_of(res)]
    got = all_gather_pieces(local, lengths, piece_parts, group)
    return [[got[int(first[i]) + j] for j in range(n_per[i])] for i in range(len(costs))]


class ShardedStokesBatch:
    """``StokesBatch`` over all ranks: problem k runs on the rank
    ``partition_by_cost`` gives it (cost = its point count), and forward /
    adjoint return every problem's results on every rank (numpy arrays)."""

    def __init__(self, problems, Nequiv=32, Ncutoff=64, n_streams=8, group=None, **kw):
        from .batch import StokesBatch
        self.group = group
        self.world, self.rank = world_and_rank(group)
        self.sizes = [int(np.asarray(x).size) for x, _ in problems]
        self.parts = partition_by_cost(self.sizes, self.world)
        self.mine = self.parts[self.rank]
        self.local = StokesBatch([problems[i] for i in self.mine], Nequiv=Nequiv, Ncutoff=Ncutoff,
                                 n_streams=n_streams, **kw) if self.mine else None

    def _gather(self, local_outs, n_rows):
        lengths = [n for n in self.sizes for _ in range(n_rows)]
        parts = [[n_rows * i + r for i in p for r in range(n_rows)] for p in self.parts]
        flat = [row for tup in local_outs for row in tup]
        got = all_gather_pieces(flat, lengths, parts, self.group)
        return [tuple(got[n_rows * i + r] for r in range(n_rows)) for i in range(len(self.sizes))]

    def forward(self, forces):
        """(u, v, p) of every problem, on every rank."""
        outs = self.local.forward([forces[i] for i in self.mine]) if self.mine else []
        return self._gather(outs, 3)

    def adjoint(self, cotangents):
        """(dfx, dfy) of every problem, on every rank."""
        outs = self.local.adjoint([cotangents[i] for i in self.mine]) if self.mine else []
        return self._gather(outs, 2)


def sharded_multi_rhs(make_fmm, tau, targets=(), sources=True, group=None):
    """Multi-RHS evaluation with the charge columns split over the ranks.

    ``make_fmm()`` builds this rank's FMM object on the (shared) sources;
    ``tau`` is [k, N].  Rank r forms the expansions of its column block and
    evaluates them at the sources (``source_evaluation``, when ``sources``)
    and at each (x, y) of ``targets`` (``target_evaluation``).  Returns the
    list of full [k, M] results (sources first) on every rank."""
    world, rank = world_and_rank(group)
    tau = np.asarray(_cpu(tau), dtype=np.float64)
    if tau.ndim != 2:
        raise ValueError("tau must be [k, N]")
    k, n = tau.shape
    blocks = column_blocks(k, world)
    lo, hi = blocks[rank]
    F = make_fmm() if hi > lo else None
    evals = []
    if hi > lo:
        F.build_expansions(tau[lo:hi])
        if sources:
            evals.append(np.asarray(_cpu(F.source_evaluation(F._x, F._y))).reshape(hi - lo, -1))
        for tx, ty in targets:
            evals.append(np.asarray(_cpu(F.target_evaluation(tx, ty))).reshape(hi - lo, -1))
    sizes = ([n] if sources else []) + [int(np.asarray(_cpu(tx)).size) for tx, _ in targets]
    # pieces: (evaluation e, column c) -> id e * k + c
    lengths = [m for m in sizes for _ in range(k)]
    parts = [[e * k + c for c in range(b0, b1) for e in range(len(sizes))] for b0, b1 in blocks]
    local = [evals[e][c - lo] for c in range(lo, hi) for e in range(len(sizes))]
    got = all_gather_pieces(local, lengths, parts, group)
    return [np.stack([got[e * k + c] for c in range(k)]) for e in range(len(sizes))]
