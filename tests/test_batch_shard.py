"""The 48-cell batch spread over ranks by cell (qxmd_b200.batch), on the CPU:
the partition covers every cell once and balances the cost estimate, and two
gloo ranks that each evaluate their own cells (the oracle's kinetic energy of
the reference's LCG start, a stand-in for the device SCF) and gather the
results reproduce the one-process results cell by cell."""
import os
import socket

import numpy as np
import pytest

from qxmd_b200 import batch, cell

NCELLS = 48


def _cells():
    return [cell.batch_cell(i) for i in range(NCELLS)]


def _costs(cells):
    return [batch.cell_cost(s.nband, s.gs.grid, s.gs.nplwex) for s in cells]


def _result(s):
    import oracle
    c = cell.random_wavefunctions(s.gs.nplwex, s.nband)
    e, _ = oracle.Ham(s, 1).ekinetic(c, s.occ)
    return float(e)


@pytest.mark.parametrize("nranks", [1, 2, 3, 4, 8])
def test_partition_covers_every_cell_once_and_balances(nranks):
    costs = _costs(_cells())
    parts = batch.partition(costs, nranks)
    assert len(parts) == nranks
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(NCELLS))
    loads = [sum(costs[i] for i in p) for p in parts]
    # longest-first greedy: no rank exceeds the mean by more than the largest cell
    assert max(loads) <= sum(costs) / nranks + max(costs)
    # the same assignment on every call (every rank computes it alone)
    assert batch.partition(costs, nranks) == parts


def _worker(rank, world, port, out_path):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        cells = _cells()
        mine = batch.partition(_costs(cells), world)[rank]
        local = {i: _result(cells[i]) for i in mine}
        merged = batch.gather_results(local, world)
        if rank == 0:
            np.save(out_path, np.array([merged[i] for i in range(NCELLS)]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_the_batch(tmp_path):
    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    out = str(tmp_path / "merged.npy")
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    want = np.array([_result(s) for s in _cells()])
    np.testing.assert_array_equal(got, want)
