"""CPU test of bench.py's multi-rank plumbing on two gloo ranks: each rank is an independent
replica (its own batch and case draws, no data-path collective); the timed region is bracketed by
barriers and the device time reported is the maximum over ranks, the work the sum."""
import os
import socket

import torch.distributed as dist
import torch.multiprocessing as mp


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR='127.0.0.1',
                      MASTER_PORT=str(port))
    import bench
    r, w, local = bench.dist_setup(world)
    assert (r, w, local) == (rank, world, rank)
    bench.dist_barrier(w)
    t = bench.dist_max(1.5 + rank, w)
    total = bench.dist_sum(10 * (rank + 1), w)
    draws = [spec.mach for spec in bench.workloads.batched_sa_specs(4, seed=bench.rank_seed(rank))]  # the replica's own cases
    with open(f'{out}.{rank}', 'w') as f:
        f.write(' '.join(repr(m) for m in draws))
    if rank == 0:
        with open(out, 'w') as f:
            f.write(f'{t} {total}')
    bench.dist_barrier(w)
    dist.destroy_process_group()


def test_two_rank_max_and_sum(tmp_path):
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        port = s.getsockname()[1]
    out = tmp_path / 'r.txt'
    mp.start_processes(_rank, args=(2, port, str(out)), nprocs=2, start_method='spawn', join=True)
    t, total = out.read_text().split()
    assert float(t) == 2.5 and float(total) == 30.0
    assert (tmp_path / 'r.txt.0').read_text() != (tmp_path / 'r.txt.1').read_text()
