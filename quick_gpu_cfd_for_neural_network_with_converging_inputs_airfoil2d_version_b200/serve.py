"""Serving loop over the batched engine.

Requests (one airfoil + flow condition each) arrive as a Poisson process.  Each request's mesh
is built on a pool of host threads (the native builder, amr_mesh_build) as soon as it
arrives; built requests are admitted first come first served while the device arena has room
(amr_batch_admit answers "no room" with 3); the batch advances a fixed number of trials per
poll; the reference driver's steady rule (src/quick_airfoil.cpp:75-92), evaluated on the
device, retires converged cases, and the step cap retires the rest as capped.  A request's
latency runs from its arrival to the poll that retires it.

    reqs = poisson_requests(2000, rate=50.0, seed=20261203)
    server = Server(Batch(precision=32, max_cases=512), max_steps=30000)
    results = server.run(reqs)
    print(summarize(results, server.wall_seconds))

With several GPUs each rank serves its own shard of the request stream (shard()), one batch
per GPU; the ranks exchange nothing but the final results (gather_results).
"""
import concurrent.futures
import dataclasses
import time

import numpy as np

from . import _abi, airfoils, cases

STATUS_MAXSTEPS = _abi.STATUS_MAXSTEPS


@dataclasses.dataclass
class Request:
    id: int
    arrival: float          # seconds after the start of the run
    spec: cases.CaseSpec


@dataclasses.dataclass
class Result:
    id: int
    arrival: float
    admitted: float = float('nan')
    finished: float = float('nan')
    outcome: str = ''       # 'converged' | 'capped' | 'failed'
    steps: int = 0
    cells: int = 0
    cl: float = float('nan')
    cd: float = float('nan')
    cm: float = float('nan')
    error: str = ''

    @property
    def latency(self):
        return self.finished - self.arrival


def poisson_requests(n, rate, seed, profiles=('LF1', 'LF2'), physics='sa', mach=(1.2, 2.0), aoa=(-3.0, 5.0)):
    """n requests with exponential inter-arrival times of mean 1/rate, alternating profiles, and
    seeded NACA 4-digit shapes, Mach numbers and angles of attack."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += float(rng.exponential(1.0 / rate))
        naca = airfoils.seeded_naca(rng)
        spec = cases.CaseSpec(naca=naca, profile=profiles[i % len(profiles)], physics=physics,
                              mach=float(rng.uniform(*mach)), aoa=float(rng.uniform(*aoa)))
        out.append(Request(i, t, spec))
    return out


def shard(requests, rank, world):
    """The requests rank `rank` of `world` serves: every world-th one, arrival times kept."""
    return requests[rank::world]


def build_request_mesh(req):
    from . import builder
    x, y, pt = airfoils.naca4(*req.spec.naca)
    return builder.build_mesh(req.spec, x, y, pt)


class Server:
    """Runs one batch.  `batch` is a batch.Batch (or an object with the same admit / advance /
    check / status / release methods); `build` maps a Request to its MeshArrays."""

    def __init__(self, batch, max_steps=30000, trials=32, builder_threads=0, build=build_request_mesh, steady=None,
                 clock=time.perf_counter, sleep=time.sleep):
        self.batch = batch
        self.max_steps = int(max_steps)
        self.trials = int(trials)
        self.build = build
        self.steady = dict(cases.STEADY, **(steady or {}))
        self.clock = clock
        self.sleep = sleep
        self.threads = builder_threads if builder_threads > 0 else None
        self.wall_seconds = 0.0
        self.polls = 0
        self.cell_steps = 0

    def _control(self, spec):
        from .batch import case_control
        return case_control(1e30, self.max_steps, steady=True, mach=spec.mach, aoa=spec.aoa, **self.steady)

    def run(self, requests):
        requests = sorted(requests, key=lambda r: r.arrival)
        results = {r.id: Result(r.id, r.arrival) for r in requests}
        pending = list(requests)          # not yet arrived
        building = {}                     # future -> request
        ready = []                        # (request, mesh) built, waiting for room
        live = {}                         # slot -> (request, cells)
        t0 = self.clock()
        pool = concurrent.futures.ThreadPoolExecutor(max_workers=self.threads)
        try:
            while pending or building or ready or live:
                now = self.clock() - t0
                while pending and pending[0].arrival <= now:
                    r = pending.pop(0)
                    building[pool.submit(self.build, r)] = r
                for fut in [f for f in building if f.done()]:
                    r = building.pop(fut)
                    try:
                        ready.append((r, fut.result()))
                    except Exception as e:  # a mesh the builder rejects fails the request
                        res = results[r.id]
                        res.outcome, res.error, res.finished = 'failed', str(e), self.clock() - t0
                ready.sort(key=lambda item: item[0].arrival)
                while ready:
                    r, mesh = ready[0]
                    u0 = cases.initial_state(mesh, r.spec.initial_primitive())
                    slot = self.batch.admit(mesh, r.spec.params(), u0, self._control(r.spec))
                    if slot is None:
                        break                 # no room: admit again after a retirement
                    ready.pop(0)
                    live[slot] = (r, mesh.n_cells)
                    results[r.id].admitted = self.clock() - t0
                    results[r.id].cells = mesh.n_cells
                if not live:
                    # idle: wait for the next arrival or build
                    waits = [pending[0].arrival - (self.clock() - t0)] if pending else []
                    if building:
                        waits.append(0.002)
                    if waits:
                        self.sleep(max(0.0, min(waits)))
                    continue
                before = {s: self.batch.status(s)['steps'] for s in live}
                self.batch.advance(self.trials)
                self.batch.check()
                self.polls += 1
                done_at = self.clock() - t0
                for s in list(live):
                    st = self.batch.status(s)
                    r, cells = live[s]
                    self.cell_steps += (st['steps'] - before[s]) * cells
                    if not (st['finished'] or st['status']):
                        continue
                    res = results[r.id]
                    res.finished, res.steps = done_at, st['steps']
                    res.cl, res.cd, res.cm = st['cl'], st['cd'], st['cm']
                    if st['converged']:
                        res.outcome = 'converged'
                    elif st['status'] == STATUS_MAXSTEPS:
                        res.outcome = 'capped'
                    else:
                        res.outcome, res.error = 'failed', f"status {st['status']}"
                    self.batch.release(s)
                    del live[s]
        finally:
            pool.shutdown(wait=True)
        self.wall_seconds = self.clock() - t0
        return [results[r.id] for r in requests]


def _percentiles(values):
    if not values:
        return dict(count=0, p50=None, p99=None, mean=None)
    v = np.asarray(values, dtype=np.float64)
    return dict(count=len(v), p50=float(np.percentile(v, 50)), p99=float(np.percentile(v, 99)), mean=float(v.mean()))


def summarize(results, wall_seconds, cell_steps=None):
    """Latency percentiles per outcome, completed solves per second (converged and capped are
    reported apart), and the request count per outcome."""
    by = {}
    for r in results:
        by.setdefault(r.outcome or 'unfinished', []).append(r)
    out = dict(requests=len(results), wall_seconds=wall_seconds,
               outcomes={k: len(v) for k, v in sorted(by.items())},
               latency={k: _percentiles([r.latency for r in v]) for k, v in sorted(by.items()) if k != 'unfinished'},
               converged_per_s=len(by.get('converged', [])) / wall_seconds if wall_seconds > 0 else 0.0,
               completed_per_s=(len(by.get('converged', [])) + len(by.get('capped', []))) / wall_seconds
               if wall_seconds > 0 else 0.0)
    if cell_steps is not None:
        out['cell_steps_per_s'] = cell_steps / wall_seconds if wall_seconds > 0 else 0.0
    return out


def gather_results(results, world):
    """All ranks' results on every rank (torch.distributed, any backend)."""
    if world == 1:
        return results
    import torch.distributed as dist
    parts = [None] * world
    dist.all_gather_object(parts, [dataclasses.asdict(r) for r in results])
    merged = [Result(**d) for part in parts for d in part]
    merged.sort(key=lambda r: r.id)
    return merged
