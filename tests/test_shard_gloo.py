"""Multi-rank sharding of the batched workloads, on CPU with two gloo ranks.

Each rank evaluates its share of a QAOA batch (on the oracle here; on its own GPU in
production) and the per-instance energies meet on rank 0 in one gather; the result
must equal the single-process evaluation in instance order.  Trajectory ranges must
cover every trajectory exactly once.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from statecraft_b200 import shard as S


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_path):
    import datetime

    import torch.distributed as dist

    from oracle import oracle as O
    from statecraft_b200 import workloads as W

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    b = W.qaoa_instances(13, 2, 31, n_min=3, n_max=8)
    parts = S.partition_by_cost(S.qaoa_costs(b.n_qubits), world)
    mine = parts[rank]
    local = np.array([O.qaoa_ring_energy(int(b.n_qubits[i]), b.gammas[i], b.betas[i]) for i in mine])
    full = S.gather_by_index(local, mine, b.instances)
    if rank == 0:
        np.save(out_path, full)
    dist.barrier()
    dist.destroy_process_group()


def test_partition_covers_and_balances():
    costs = S.qaoa_costs([10, 22, 14, 22, 13, 20, 11, 18])
    parts = S.partition_by_cost(costs, 3)
    allidx = np.sort(np.concatenate(parts))
    assert allidx.tolist() == list(range(8))
    loads = [costs[p].sum() for p in parts]
    # greedy largest-first: no rank exceeds another by more than one item
    assert max(loads) - min(loads) <= costs.max()
    many = S.qaoa_costs(np.random.default_rng(0).integers(10, 23, 4096))
    loads = [many[p].sum() for p in S.partition_by_cost(many, 8)]
    assert max(loads) <= 1.01 * min(loads)
    ranges = [S.contiguous_range(1024, r, 3) for r in range(3)]
    assert ranges[0][0] == 0 and ranges[-1][1] == 1024
    assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
    assert max(b - a for a, b in ranges) - min(b - a for a, b in ranges) <= 1


def test_two_rank_qaoa_gather_matches_serial(tmp_path):
    from oracle import oracle as O
    from statecraft_b200 import workloads as W

    out = str(tmp_path / "energies.npy")
    mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True,
                       start_method="spawn")
    got = np.load(out)
    b = W.qaoa_instances(13, 2, 31, n_min=3, n_max=8)
    want = np.array([O.qaoa_ring_energy(int(n), b.gammas[i], b.betas[i])
                     for i, n in enumerate(b.n_qubits)])
    np.testing.assert_array_equal(got, want)
