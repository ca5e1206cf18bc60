"""Serving loop over the batched engine.

Requests (one airfoil + flow condition each) arrive as a Poisson process.  Each request's mesh
is built on a pool of host threads (the native builder, amr_mesh_build) as soon as it
arrives; built requests are admitted first come first served into device arenas (batches): the
first arena with room takes it (amr_batch_admit answers "no room" with 3), and when none has
room a new arena is created if the device's free memory (cudaMemGetInfo) still holds one beside
a reserve.  Every poll enqueues a fixed number of trials on every arena with live cases, then
waits; the reference driver's steady rule (src/quick_airfoil.cpp:75-92), evaluated on the
device, retires converged cases, and the step cap retires the rest as capped.  A request's
latency runs from its arrival to the poll that retires it.

    reqs = poisson_requests(2000, rate=50.0, seed=20261203)
    server = Server(lambda: Batch(precision=32, max_cases=64, max_cells=64 * 9800), max_steps=30000)
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
UNPLACEABLE = ('unplaceable',)  # _admit: the request does not fit even an empty arena


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
    u: object = None        # final state, with Server(keep_states=True)

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
    """Runs the serving loop over one or more arenas (batches).

    `arena` is either one batch (a fixed arena: requests are admitted while it has room) or a
    callable that creates one (arenas on demand, admission by free device memory): a built request
    goes into the first arena with room for it; when none has room, a new arena is created if the
    device's free memory, less `hbm_reserve` bytes, still covers one arena of the size the first
    one took (`memory` returns (free, total) bytes; by default cudaMemGetInfo of `device`), and
    otherwise the request waits for a retirement.  Arenas that empty, beyond the first, are
    destroyed and their memory returned.  `max_live_cells` optionally caps the live cells (the
    point past which more concurrent cases add latency but no throughput).  Every poll enqueues
    `trials` trials on every arena with live cases before waiting for any, so the arenas' kernels
    overlap on the device.  `build` maps a Request to its MeshArrays; with keep_states each
    result carries its final state."""

    def __init__(self, arena, max_steps=30000, trials=32, builder_threads=0, build=build_request_mesh, steady=None,
                 clock=time.perf_counter, sleep=time.sleep, memory=None, device=0, hbm_reserve=2 << 30,
                 max_live_cells=None, keep_states=False, max_arenas=256):
        if callable(arena) and not hasattr(arena, 'admit'):
            self.make_arena, self.arenas = arena, []
        else:
            self.make_arena, self.arenas = None, [arena]
        self.max_steps = int(max_steps)
        self.trials = int(trials)
        self.build = build
        self.steady = dict(cases.STEADY, **(steady or {}))
        self.clock = clock
        self.sleep = sleep
        self.threads = builder_threads if builder_threads > 0 else None
        self.device = device
        self.memory = memory
        self.hbm_reserve = int(hbm_reserve)
        self.max_live_cells = max_live_cells
        self.keep_states = keep_states
        self.max_arenas = max_arenas
        self.arena_bytes = None
        self.wall_seconds = 0.0
        self.polls = 0
        self.cell_steps = 0
        self.live_cells = 0
        self.peak_live_cells = 0
        self.peak_arenas = len(self.arenas)
        self.arenas_created = 0

    def _control(self, spec):
        from .batch import case_control
        return case_control(1e30, self.max_steps, steady=True, mach=spec.mach, aoa=spec.aoa, **self.steady)

    def _free_memory(self):
        if self.memory is not None:
            return self.memory()[0]
        from .batch import device_memory
        return device_memory(self.device)[0]

    def _grow(self):
        """A new arena when the device's free memory allows one more; None otherwise."""
        if self.make_arena is None or len(self.arenas) >= self.max_arenas:
            return None
        if self.arena_bytes is not None and self._free_memory() - self.hbm_reserve < self.arena_bytes:
            return None
        a = self.make_arena()
        if self.arena_bytes is None:
            self.arena_bytes = int(getattr(a, 'device_bytes', 0))
        self.arenas.append(a)
        self.arenas_created += 1
        self.peak_arenas = max(self.peak_arenas, len(self.arenas))
        return a

    def _admit(self, r, mesh):
        """(arena, slot) of the admitted request, or None when no arena has room for it now."""
        if self.max_live_cells is not None and self.live and self.live_cells + mesh.n_cells > self.max_live_cells:
            return None
        u0 = cases.uniform_state(mesh, r.spec.initial_primitive())  # the device fills the cells
        ctl = self._control(r.spec)
        for a in self.arenas:
            slot = a.admit(mesh, r.spec.params(), u0, ctl)
            if slot is not None:
                return a, slot
        a = self._grow()
        if a is not None:
            slot = a.admit(mesh, r.spec.params(), u0, ctl)
            if slot is not None:
                return a, slot
            # not even an empty arena holds it: give the arena back and fail the request
            self.arenas.remove(a)
            if hasattr(a, 'destroy'):
                a.destroy()
            return UNPLACEABLE
        return None

    def _advance(self, arenas):
        if all(hasattr(a, 'advance_async') for a in arenas):
            for a in arenas:
                a.advance_async(self.trials)
            for a in arenas:
                a.wait()
        else:
            for a in arenas:
                a.advance(self.trials)
        for a in arenas:
            a.check()

    def run(self, requests):
        requests = sorted(requests, key=lambda r: r.arrival)
        results = {r.id: Result(r.id, r.arrival) for r in requests}
        pending = list(requests)          # not yet arrived
        building = {}                     # future -> request
        ready = []                        # (request, mesh) built, waiting for room
        self.live = {}                    # (arena id, slot) -> (arena, slot, request, cells)
        live = self.live
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
                # first come, first served: never ahead of an earlier request whose mesh is building
                oldest_building = min((b.arrival for b in building.values()), default=float('inf'))
                while ready and ready[0][0].arrival < oldest_building:
                    r, mesh = ready[0]
                    placed = self._admit(r, mesh)
                    if placed is UNPLACEABLE or (placed is None and not live):
                        # nothing live will free room: the request does not fit an empty arena, or
                        # the device has no memory for one
                        ready.pop(0)
                        res = results[r.id]
                        res.outcome, res.error, res.finished = 'failed', 'no room', self.clock() - t0
                        continue
                    if placed is None:
                        break                 # no room: admit again after a retirement
                    a, slot = placed
                    ready.pop(0)
                    live[(id(a), slot)] = (a, slot, r, mesh.n_cells)
                    self.live_cells += mesh.n_cells
                    self.peak_live_cells = max(self.peak_live_cells, self.live_cells)
                    results[r.id].admitted = self.clock() - t0
                    results[r.id].cells = mesh.n_cells
                if not live:
                    # idle: wait for the next arrival or build
                    waits = [pending[0].arrival - (self.clock() - t0)] if pending else []
                    if building or ready:
                        waits.append(0.002)
                    if waits:
                        self.sleep(max(0.0, min(waits)))
                    continue
                before = {key: a.status(slot)['steps'] for key, (a, slot, _, _) in live.items()}
                active = []
                for a, _, _, _ in live.values():
                    if all(a is not b for b in active):
                        active.append(a)
                self._advance(active)
                self.polls += 1
                done_at = self.clock() - t0
                for key in list(live):
                    a, slot, r, cells = live[key]
                    st = a.status(slot)
                    self.cell_steps += (st['steps'] - before[key]) * cells
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
                    if self.keep_states:
                        res.u = a.download(slot)
                    a.release(slot)
                    self.live_cells -= cells
                    del live[key]
                # arenas that emptied, beyond the first, give their memory back
                for a in self.arenas[1:]:
                    if self.make_arena is not None and all(v[0] is not a for v in live.values()):
                        self.arenas.remove(a)
                        if hasattr(a, 'destroy'):
                            a.destroy()
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
