"""CPU tests of the serving loop's host logic (serve.Server) against a fake batch: FIFO
admission while the arena has room, retirement as converged / capped / failed, latency
accounting on a simulated clock, and the replica sharding across two gloo ranks."""
import os
import socket
import types

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import _abi, serve


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += max(dt, 1e-4)


class FakeBatch:
    """Cases of n cells; each advance costs 1 ms per live case on the fake clock and adds
    `trials` steps; a case converges at its `need` steps (checked by check()), hits the cap, or
    fails with status 4 when need < 0."""

    def __init__(self, clock, capacity_cells, needs):
        self.clock, self.capacity, self.needs = clock, capacity_cells, needs
        self.cases, self.next_slot, self.used = {}, 0, 0

    def admit(self, mesh, params, u0, control):
        if self.used + mesh.n_cells > self.capacity:
            return None
        s = self.next_slot
        self.next_slot += 1
        self.used += mesh.n_cells
        self.cases[s] = dict(cells=mesh.n_cells, steps=0, cap=control.maxsteps, need=self.needs[mesh.rid],
                             status=0, converged=False)
        return s

    def advance(self, trials):
        self.clock.t += 1e-3 * len(self.cases)
        for c in self.cases.values():
            if c['status'] or c['converged']:
                continue
            if c['need'] < 0:
                c['status'] = 4
                continue
            c['steps'] = min(c['cap'], c['steps'] + trials)
            if c['steps'] >= c['cap'] and c['steps'] < c['need']:
                c['status'] = _abi.STATUS_MAXSTEPS

    def check(self):
        for c in self.cases.values():
            if not c['status'] and c['steps'] >= c['need']:
                c['converged'] = True

    def status(self, s):
        c = self.cases[s]
        return dict(steps=c['steps'], status=c['status'], finished=int(c['converged'] or c['status'] != 0),
                    converged=int(c['converged']), cl=0.1, cd=0.01, cm=0.0)

    def release(self, s):
        self.used -= self.cases.pop(s)['cells']


def fake_build(req):
    return types.SimpleNamespace(n_cells=1000 + 10 * req.id, nv=4, rid=req.id)


def run_fake(requests, needs, capacity, max_steps=200, clock=None):
    clock = clock or FakeClock()
    batch = FakeBatch(clock, capacity, needs)
    server = serve.Server(batch, max_steps=max_steps, trials=32, builder_threads=2, build=fake_build,
                          clock=clock, sleep=clock.sleep)
    return server.run(requests), server


def requests_euler(n, rate=100.0, seed=3):
    return serve.poisson_requests(n, rate, seed, physics='euler')


def test_poisson_requests_are_seeded_and_ordered():
    a, b = requests_euler(50), requests_euler(50)
    assert [r.arrival for r in a] == [r.arrival for r in b]
    assert all(x.arrival < y.arrival for x, y in zip(a, a[1:]))
    gaps = np.diff([0.0] + [r.arrival for r in serve.poisson_requests(4000, 50.0, 11, physics='euler')])
    assert abs(gaps.mean() - 1 / 50.0) < 0.1 / 50.0
    assert [r.spec.profile for r in a[:4]] == ['LF1', 'LF2', 'LF1', 'LF2']


def test_outcomes_and_latency_accounting():
    reqs = requests_euler(12)
    needs = {r.id: (64 if r.id % 3 == 0 else (10 ** 6 if r.id % 3 == 1 else -1)) for r in reqs}
    results, server = run_fake(reqs, needs, capacity=10 ** 9)
    by = {r.id: r for r in results}
    for r in reqs:
        res = by[r.id]
        assert res.outcome == ('converged' if r.id % 3 == 0 else 'capped' if r.id % 3 == 1 else 'failed')
        assert res.finished >= res.admitted >= r.arrival and res.latency > 0
        if res.outcome == 'capped':
            assert res.steps == 200
        if res.outcome == 'failed':
            assert res.error == 'status 4'
    s = serve.summarize(results, server.wall_seconds, server.cell_steps)
    assert s['outcomes'] == {'capped': 4, 'converged': 4, 'failed': 4}
    assert s['latency']['converged']['count'] == 4 and s['latency']['converged']['p99'] >= s['latency']['converged']['p50']


def test_admission_waits_for_room_fifo():
    reqs = requests_euler(8, rate=1e6)  # everything arrives at once
    needs = {r.id: 96 for r in reqs}
    results, _ = run_fake(reqs, needs, capacity=2100)  # room for two cases at a time
    admitted = sorted(results, key=lambda r: r.admitted)
    assert [r.id for r in admitted] == sorted(r.id for r in reqs)  # first come, first served
    # never more than two live at once: each admission after the second waits for a retirement
    for i in range(2, len(admitted)):
        finished_before = sum(1 for r in results if r.finished <= admitted[i].admitted)
        assert finished_before >= i - 1


class FakeDevice:
    """Device memory for arenas of `arena_bytes` each: free = total - arenas * arena_bytes."""

    def __init__(self, total, arena_bytes):
        self.total, self.arena_bytes, self.arenas = total, arena_bytes, 0
        self.peak = 0

    def memory(self):
        return self.total - self.arenas * self.arena_bytes, self.total


def test_arenas_grow_by_free_memory_and_are_returned():
    """Admission by free device memory: a request that fits no arena opens a new one while the
    device's free memory, less the reserve, covers one more; emptied arenas beyond the first are
    destroyed (their memory returned)."""
    clock = FakeClock()
    reqs = requests_euler(12, rate=1e6)  # everything arrives at once
    needs = {r.id: 96 for r in reqs}
    dev = FakeDevice(total=1000, arena_bytes=100)
    made, destroyed = [], []

    def make_arena():
        b = FakeBatch(clock, 2100, needs)  # two cases per arena
        b.device_bytes = dev.arena_bytes
        dev.arenas += 1
        dev.peak = max(dev.peak, dev.arenas)

        def destroy(b=b):
            destroyed.append(b)
            dev.arenas -= 1
        b.destroy = destroy
        made.append(b)
        return b

    # reserve 650: free - reserve >= 100 holds for 0, 1 and 2 existing arenas, so at most 3
    server = serve.Server(make_arena, max_steps=200, trials=32, builder_threads=2, build=fake_build, clock=clock,
                          sleep=clock.sleep, memory=dev.memory, hbm_reserve=650)
    results = server.run(reqs)
    assert all(r.outcome == 'converged' for r in results)
    assert server.peak_arenas == 3 and dev.peak == 3 and len(made) >= 3
    assert server.peak_live_cells <= 3 * 2100
    # at most six live at once: the seventh admission waited for a retirement
    admitted = sorted(results, key=lambda r: r.admitted)
    assert sum(1 for r in results if r.finished <= admitted[6].admitted) >= 1
    assert len(server.arenas) == 1 and len(destroyed) == len(made) - 1


def test_live_cell_cap_and_unplaceable_request():
    clock = FakeClock()
    reqs = requests_euler(6, rate=1e6)
    needs = {r.id: 64 for r in reqs}
    server = serve.Server(lambda: FakeBatch(clock, 10 ** 9, needs), max_steps=200, trials=32, builder_threads=2,
                          build=fake_build, clock=clock, sleep=clock.sleep, memory=lambda: (10 ** 12, 10 ** 12),
                          max_live_cells=2100)
    results = server.run(reqs)
    assert all(r.outcome == 'converged' for r in results) and server.peak_live_cells <= 2100
    # a request larger than an empty arena fails instead of waiting forever
    big = serve.Server(lambda: FakeBatch(clock, 500, needs), max_steps=200, trials=32, builder_threads=2,
                       build=fake_build, clock=clock, sleep=clock.sleep, memory=lambda: (10 ** 12, 10 ** 12))
    out = big.run(reqs[:2])
    assert [r.outcome for r in out] == ['failed', 'failed'] and out[0].error == 'no room'
    assert big.arenas_created == 2 and big.arenas == []  # each trial arena was given back


def _rank_main(rank, world, port, out_path):
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    reqs = requests_euler(10)
    mine = serve.shard(reqs, rank, world)
    needs = {r.id: 64 for r in reqs}
    results, _ = run_fake(mine, needs, capacity=10 ** 9)
    merged = serve.gather_results(results, world)
    if rank == 0:
        with open(out_path, 'w') as f:
            f.write(','.join(f'{r.id}:{r.outcome}' for r in merged))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_shards_cover_every_request_once(tmp_path):
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        port = s.getsockname()[1]
    out = tmp_path / 'merged.txt'
    mp.start_processes(_rank_main, args=(2, port, str(out)), nprocs=2, start_method='spawn', join=True)
    ids = [tuple(x.split(':')) for x in out.read_text().split(',')]
    assert [int(i) for i, _ in ids] == list(range(10))
    assert all(o == 'converged' for _, o in ids)
