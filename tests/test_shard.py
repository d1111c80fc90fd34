"""Work split over ranks (flexmm_b200.shard): partition, gather, and the two
splits of the path that need no exchange -- independent problems and
multi-RHS charge columns -- on world-size-2 gloo process groups (CPU).

The per-rank compute here is the oracle's FP64 direct sum standing in for
the FMM (the GPU FMM itself is covered by the other tests); what is under
test is that every rank ends with every result, in the caller's order,
equal to a single-process run."""
import os
import socket

import numpy as np
import pytest

from flexmm_b200.shard import column_blocks, partition_by_cost


def test_partition_by_cost_is_balanced_and_complete():
    rng = np.random.default_rng(4)
    sizes = np.round(np.exp(rng.uniform(np.log(2000), np.log(200000), 256))).astype(int)
    for world in (1, 2, 3, 4, 8):
        parts = partition_by_cost(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(sizes.size))
        assert all(p == sorted(p) for p in parts)
        loads = [sizes[p].sum() for p in parts]
        # LPT: no rank above the mean by more than the largest single item
        assert max(loads) - sizes.sum() / world <= sizes.max()
        assert parts == partition_by_cost(sizes, world)   # deterministic
    assert partition_by_cost([5, 5, 5], 4)[3] == []


def test_column_blocks():
    assert column_blocks(64, 8) == [(8 * r, 8 * r + 8) for r in range(8)]
    b = column_blocks(10, 4)
    assert b == [(0, 3), (3, 6), (6, 8), (8, 10)]
    assert column_blocks(1, 2) == [(0, 1), (1, 1)]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


class _DirectFMM:
    """A CPU stand-in with KI_FMM's multi-RHS surface (direct sums)."""

    def __init__(self, x, y):
        self._x, self._y = x, y

    def build_expansions(self, tau):
        self.tau = np.atleast_2d(tau)

    def source_evaluation(self, x, y):
        from oracle.direct import direct_laplace
        return np.stack([direct_laplace(self._x, self._y, t, x, y, True) for t in self.tau])

    def target_evaluation(self, x, y):
        from oracle.direct import direct_laplace
        return np.stack([direct_laplace(self._x, self._y, t, x, y, False) for t in self.tau])


def _problems():
    rng = np.random.default_rng(9)
    sizes = [300, 40, 900, 120, 700, 60, 510]
    probs = [(rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)) for n in sizes]
    forces = [(rng.standard_normal(n), rng.standard_normal(n)) for n in sizes]
    return sizes, probs, forces


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from flexmm_b200.shard import run_sharded, sharded_multi_rhs
        from oracle.direct import direct_stokes
        sizes, probs, forces = _problems()

        def compute(idx):
            return [direct_stokes(probs[i][0], probs[i][1], forces[i][0], forces[i][1],
                                  probs[i][0], probs[i][1], True) for i in idx]
        res = run_sharded(sizes, compute, lambda r: [r[0], r[1], r[2]], lambda i: [sizes[i]] * 3)
        np.savez(os.path.join(out_dir, f"batch_{rank}.npz"),
                 **{f"p{i}_{j}": res[i][j] for i in range(len(sizes)) for j in range(3)})
        rng = np.random.default_rng(2)
        n, k = 500, 5
        x, y = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
        tau = rng.standard_normal((k, n))
        tx, ty = rng.uniform(-1, 1, 77), rng.uniform(-1, 1, 77)
        us, ut = sharded_multi_rhs(lambda: _DirectFMM(x, y), tau, targets=[(tx, ty)])
        np.savez(os.path.join(out_dir, f"multi_{rank}.npz"), us=us, ut=ut)
    finally:
        dist.destroy_process_group()


def test_sharded_problems_and_columns_on_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    from oracle.direct import direct_laplace, direct_stokes
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    sizes, probs, forces = _problems()
    for rank in range(world):
        g = np.load(tmp_path / f"batch_{rank}.npz")
        for i in range(len(sizes)):
            want = direct_stokes(probs[i][0], probs[i][1], forces[i][0], forces[i][1],
                                 probs[i][0], probs[i][1], True)
            for j in range(3):
                np.testing.assert_array_equal(g[f"p{i}_{j}"], want[j])
    rng = np.random.default_rng(2)
    n, k = 500, 5
    x, y = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    tau = rng.standard_normal((k, n))
    tx, ty = rng.uniform(-1, 1, 77), rng.uniform(-1, 1, 77)
    for rank in range(world):
        m = np.load(tmp_path / f"multi_{rank}.npz")
        for c in range(k):
            np.testing.assert_array_equal(m["us"][c], direct_laplace(x, y, tau[c], x, y, True))
            np.testing.assert_array_equal(m["ut"][c], direct_laplace(x, y, tau[c], tx, ty, False))


@pytest.mark.gpu
def test_sharded_stokes_batch_single_rank_equals_batch(built_lib):
    """On one rank the sharded batch is the batch itself (the multi-rank
    split is the gloo test above)."""
    import torch
    from flexmm_b200.batch import StokesBatch
    from flexmm_b200.shard import ShardedStokesBatch
    sizes, probs, forces = _problems()
    S = ShardedStokesBatch(probs, Nequiv=16, Ncutoff=32, n_streams=2)
    B = StokesBatch(probs, Nequiv=16, Ncutoff=32, n_streams=2)
    a = S.forward(forces)
    b = B.forward(forces)
    torch.cuda.synchronize()
    for i in range(len(sizes)):
        for j in range(3):
            np.testing.assert_allclose(a[i][j], b[i][j].cpu().numpy(), rtol=0, atol=0)
