"""Benchmark of the static-AMR explicit time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload batched|plain]

One step = one SSP-RK3 step (one trial) of every case in the batch.  Workload `batched` (the
default): 256 SA-neg/Sutherland cases, HLLC, FP32 state (FP64 dt/norms/loads), half LF1 and half
LF2 meshes, each case with its own seeded Mach ~ U[1.2, 2.0] and AoA ~ U[-3, 5] deg.  `value` is
whole-job accepted cell-steps per second timed with CUDA events on the engine's launch stream;
`e2e` is the same work through the C ABI from host buffers (mesh + state upload, the steps, state
download) timed on the host clock.  Beside it: the plain FP64 session on the same meshes and the
reference CPU core (oracle/_ref, all host threads) on a bounded sample.
"""
import argparse
import json
import math
import os
import pathlib
import select
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import _abi, cases  # noqa: E402
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.batch import Batch, case_control  # noqa: E402
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.mesh import MeshArrays  # noqa: E402
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.session import StaticAmrGpu, default_options  # noqa: E402

METRIC = 'solves/s & cell-steps/s at |ΔCL|,|ΔCD|≤1e-4 vs plain FP64; p50/p99 latency'
GOLDEN = ROOT / 'tests' / 'golden'
MESHES = {'LF1': GOLDEN / 'mesh_naca2412_lf1_sa.npz', 'LF2': GOLDEN / 'mesh_naca2412_lf2_sa.npz'}
SOLVE_STEPS = 5000  # steps per solve of the batched workload
# DRAM bytes (read + write) of one split-mode trial of the 256-case workload, summed over its
# kernels from one ncu capture (profiles/split_trial_f32_sa_256cases.md; cold cache, so an upper
# bound of a warm trial).  Reported as roofline.traffic when the run matches that configuration.
SPLIT_256_TRAFFIC_PER_STEP = 2.7783e9


def peaks():
    p = ROOT / 'MEASURED_PEAKS.json'
    if p.exists():
        d = json.loads(p.read_text())
        return d['hbm_gbs'], 'measured'
    return 6650.0, 'fallback'


def algorithmic_bytes(mesh, s=4, sg=4):
    """Compulsory HBM bytes of one accepted step of one case (intermediates count 0):
    8*nv*s*n state traffic + 3*[n*c_cell + nf*c_face + nw*c_wall + T*c_term + S_srd]."""
    n, nf, nw, nv = mesh.n_cells, mesh.n_faces, mesh.n_walls, mesh.nv
    viscous = mesh.laminar
    T = int(mesh.visc_offsets[-1]) if viscous else 0
    c_cell = 8 + 4 + ((sg + 4) if viscous else 0)
    c_face = 8 + 4 + 8 + sg + (5 * sg if viscous else 0)
    c_wall = 4 + 3 * sg + ((4 + sg) if viscous else 0)
    c_term = 4 + 2 * sg
    srd = 0
    if mesh.small_cells:
        for k in range(n):
            size = int(mesh.group_offsets[k + 1] - mesh.group_offsets[k])
            if size > 1:
                srd += 16 * size
    return 8 * nv * s * n + 3 * (n * c_cell + nf * c_face + nw * c_wall + T * c_term + srd)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every `interval_ms` while entered (the
    batched bench enters it for the warm-up and timed loop only, so idle set-up time, when the
    GPU drops its clocks, does not count)."""
    FIELDS = 'index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,' \
             'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap'

    def __init__(self, device, interval_ms=200):
        self.device = device
        self.interval_ms = int(interval_ms)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.device), '--query-gpu=' + self.FIELDS,
                                          '--format=csv,noheader,nounits', '-lms', str(self.interval_ms)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        # wait (at most 5 s) for nvidia-smi's first sample, taken before the sampled work starts,
        # and drop it, so that every kept sample falls inside the sampled region
        if self.proc:
            if select.select([self.proc.stdout], [], [], 5.0)[0]:
                self.proc.stdout.readline()
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for line in getattr(self, 'lines', []):
            parts = [p.strip() for p in line.split(',')]
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except (ValueError, IndexError):
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == 'active':
                    reasons.add(name)
        return dict(sm_mhz=statistics.median(sm) if sm else None, sm_max_mhz=mx, reasons=sorted(reasons),
                    samples=len(sm))


def batched_cases(ncases, seed=20261203):
    rng = np.random.default_rng(seed)
    meshes = {k: MeshArrays.load(v) for k, v in MESHES.items()}
    out = []
    for i in range(ncases):
        profile = 'LF1' if i % 2 == 0 else 'LF2'
        mach, aoa = float(rng.uniform(1.2, 2.0)), float(rng.uniform(-3.0, 5.0))
        spec = cases.CaseSpec(naca=(0.02, 0.4, 0.12), profile=profile, physics='sa', mach=mach, aoa=aoa)
        mesh = meshes[profile].with_physics(boundaries=spec.boundary_records())
        out.append((spec, mesh))
    return out


def parse_launch(cfg):
    """(block, grid, launch_mode) of a launch_config() string."""
    block = int(cfg.split('block=')[1].split()[0])
    grid = int(cfg.split('grid=')[1].split()[0])
    mode = (_abi.LAUNCH_PHASES if 'mode=phases' in cfg else _abi.LAUNCH_SPLIT if 'mode=split' in cfg
            else _abi.LAUNCH_TILED if 'mode=tiled' in cfg else _abi.LAUNCH_PERSISTENT)
    return block, grid, mode


def run_batched(case_list, precision, steps, warmup, device=0, trials=32, block=0, grid=0, tune=True, clock=None):
    """Admit every case, autotune, warm up, then time `steps` trials with CUDA events on the
    engine stream.  Accepted cell-steps are counted per case from the device counters.  `clock`
    (a ClockSampler) samples the warm-up and timed loop."""
    total_cells = sum(m.n_cells for _, m in case_list)
    b = Batch(precision=precision, model=_abi.MODEL_LAMINAR, sa=True, max_cases=len(case_list),
              max_cells=total_cells + 64, device=device, block_threads=block, grid_blocks=grid)
    slots = []
    for spec, mesh in case_list:
        u0 = cases.initial_state(mesh, spec.initial_primitive())
        s = b.admit(mesh, spec.params(), u0, case_control(1e30, 10 ** 9, steady=False, mach=spec.mach, aoa=spec.aoa))
        assert s is not None, 'arena too small'
        slots.append(s)
    if tune:
        b.autotune(4)
    if clock is not None:
        clock.__enter__()
    done = 0
    while done < warmup:
        k = min(trials, warmup - done)
        b.advance(k)
        done += k
    before = [b.status(s)['steps'] for s in slots]
    launches0 = b.kernel_launches
    dev_seconds, adv, advances = 0.0, 0, 0
    while adv < steps:
        k = min(trials, steps - adv)
        b.advance(k)
        dev_seconds += b.last_advance_seconds
        adv += k
        advances += 1
    if clock is not None:
        clock.__exit__(None, None, None)
    status = [b.status(s) for s in slots]
    cell_steps = sum(m.n_cells * (st['steps'] - b0) for (_, m), st, b0 in zip(case_list, status, before))
    return dict(batch=b, slots=slots, dev_seconds=dev_seconds, launches=b.kernel_launches - launches0,
                cell_steps=cell_steps, status=status, config=b.launch_config(), advances=advances)


def run_e2e(case_list, precision, steps, device=0, trials=32, block=0, grid=0, mode=0):
    """The same work end to end through the C ABI from host buffers: batch creation, mesh and
    state upload of every case (one bulk admission), `steps` trials with a control read-back per launch, and the
    download of every final state; host wall clock."""
    t0 = time.perf_counter()
    total_cells = sum(m.n_cells for _, m in case_list)
    b = Batch(precision=precision, model=_abi.MODEL_LAMINAR, sa=True, max_cases=len(case_list),
              max_cells=total_cells + 64, device=device, block_threads=block, grid_blocks=grid, launch_mode=mode)
    t_create = time.perf_counter()
    items, h2d = [], 0
    for spec, mesh in case_list:
        u0 = cases.initial_state(mesh, spec.initial_primitive())
        items.append((mesh, spec.params(), u0, case_control(1e30, 10 ** 9, steady=False)))
        h2d += mesh_bytes(mesh, precision) + u0.nbytes * precision // 64
    t_items = time.perf_counter()
    slots = b.admit_many(items)
    t_admit = time.perf_counter()
    adv, advances = 0, 0
    while adv < steps:
        k = min(trials, steps - adv)
        b.advance(k)
        adv += k
        advances += 1
    t_advance = time.perf_counter()
    d2h = 0
    cell_steps = 0
    for (_, mesh), s in zip(case_list, slots):
        u = b.download(s)
        d2h += u.nbytes * precision // 64
        cell_steps += mesh.n_cells * b.status(s)['steps']
    t_end = time.perf_counter()
    seconds = t_end - t0
    d2h += advances * 96 * len(slots)  # per-launch control read-back
    b.destroy()
    return dict(value=cell_steps / seconds, seconds=seconds, h2d=h2d, d2h=d2h,
                phases=dict(create=t_create - t0, admit=t_admit - t_create, advance=t_advance - t_admit,
                            download=t_end - t_advance, admit_host_inputs=t_items - t_create))


def mesh_bytes(mesh, precision):
    """Bytes of engine tables uploaded for one mesh."""
    s = precision // 8
    n, ns, nw = mesh.n_cells + 1, int(mesh.face_offsets[-1]), mesh.n_walls
    T = int(mesh.visc_offsets[-1]) if mesh.laminar else 0
    cells = n * (4 + 8 * 5 + 1 + 4 * 3 + (s if mesh.nv == 5 else 0))
    slots = ns * (12 + s + (6 * s if mesh.laminar else 0))
    walls = nw * (4 * s + 4 + 16)
    terms = T * (8 + 2 * s)
    return cells + slots + walls + terms


def plain_fp64(case_list, steps):
    """The plain FP64 session on one case of each profile: accepted cell-steps per device second.
    A first session warms up (graph capture, autotune); the timed session runs `steps` steps."""
    res = {}
    for profile in ('LF1', 'LF2'):
        spec, mesh = [c for c in case_list if c[0].profile == profile][0]
        u0 = cases.initial_state(mesh, spec.initial_primitive())
        w = StaticAmrGpu.create(mesh, spec.params(), u0)
        w.advance(1e30, 64)
        cfg = w.launch_config()
        w.destroy()
        block, grid, mode = parse_launch(cfg)
        s = StaticAmrGpu.create(mesh, spec.params(), u0,
                                options=default_options(block_threads=block, grid_blocks=grid, launch_mode=mode))
        s.advance(1e30, steps)
        st = s.stats()
        sec = st['advance_event_seconds']
        res[profile] = dict(cells=mesh.n_cells, steps=s.steps, seconds=sec, us_per_step=1e6 * sec / s.steps,
                            cell_steps_per_s=mesh.n_cells * s.steps / sec, config=cfg, polls=st['status_polls'])
        s.destroy()
    return res


def cpu_reference(case_list, steps_lf1, steps_lf2, threads):
    """Reference CPU core (oracle/_ref, OpenMP) on one case of each profile, in a subprocess so the
    OpenMP thread count is fixed before the runtime loads."""
    code = f'''
import json, sys
sys.path.insert(0, {str(ROOT)!r})
from bench import batched_cases
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import cases
from oracle.oracle import RefCase
cl = batched_cases(2)
out = {{}}
for (spec, mesh), n in zip(cl, ({steps_lf1}, {steps_lf2})):
    rc = RefCase.from_mesh(mesh, spec.params(), kind='omp')
    u0 = cases.initial_state(mesh, spec.initial_primitive())
    sec, r = rc.run_timed(u0, 1e30, n)
    out[spec.profile] = dict(cells=mesh.n_cells, steps=r['steps'], seconds=sec)
print(json.dumps(out))
'''
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND='false')
    r = subprocess.run([sys.executable, '-c', code], capture_output=True, text=True, env=env, cwd=str(ROOT))
    if r.returncode:
        raise RuntimeError(r.stderr[-2000:])
    d = json.loads(r.stdout.strip().splitlines()[-1])
    cell_steps = sum(v['cells'] * v['steps'] for v in d.values())
    seconds = sum(v['seconds'] for v in d.values())
    return cell_steps / seconds, d


def cpu_model():
    try:
        for line in open('/proc/cpuinfo'):
            if line.startswith('model name'):
                return line.split(':', 1)[1].strip()
    except OSError:
        pass
    return 'unknown'


def dist_setup(n_gpus):
    rank = int(os.environ.get('RANK', '0'))
    world = int(os.environ.get('WORLD_SIZE', '1'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group('gloo', timeout=datetime.timedelta(seconds=600))
    return rank, world, local


def dist_max(value, world):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def reference_arm(args, rank, world):
    """--impl reference: the reference CPU implementation (oracle/_ref with all host threads) on
    the same workload, each step a bounded sample (one LF1 + one LF2 case)."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    case_list = batched_cases(2)
    n_lf1, n_lf2 = 40, 20
    values = []
    for _ in range(max(1, args.warmup)):
        cpu_reference(case_list, 4, 2, threads)
    for _ in range(args.steps):
        v, detail = cpu_reference(case_list, n_lf1, n_lf2, threads)
        values.append(v)
    value = statistics.median(values)
    line = dict(metric=METRIC, impl='reference', value=value, unit='cell-steps/s', n_gpus=args.gpus,
                steps=args.steps, warmup=args.warmup, higher_is_better=True, scaling='weak', vs_baseline=None,
                dtype='f64', data='synthetic',
                config=dict(workload='batched-sa-fp32-256', sample=f'1 LF1 x {n_lf1} + 1 LF2 x {n_lf2} steps per step'),
                cpu_baseline=dict(value=value, unit='cell-steps/s', cores=threads, kind='reference',
                                  sample=f'1 LF1 ({detail["LF1"]["cells"]} cells) x {n_lf1} steps + 1 LF2 '
                                         f'({detail["LF2"]["cells"]} cells) x {n_lf2} steps', cpu=cpu_model()),
                e2e=dict(value=value, unit='cell-steps/s', h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)


def run_serving(args, rank, world, local):
    """--serve: the served form.  Poisson request arrivals (seeded), host mesh builds on a thread
    pool, admission while the arena has room, device steady-rule retirement or the step cap.
    Each rank serves its shard on its own GPU; rank 0 prints one JSON line."""
    from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import serve
    reqs = serve.poisson_requests(args.requests, args.rate, args.seed)
    mine = serve.shard(reqs, rank, world)
    batch = Batch(precision=32, model=_abi.MODEL_LAMINAR, sa=True, max_cases=args.serve_cases,
                  max_cells=args.serve_cases * 9800, device=local, launch_mode=_abi.LAUNCH_SPLIT, block_threads=128)
    server = serve.Server(batch, max_steps=args.max_steps, trials=32, builder_threads=max(1, (os.cpu_count() or 2) - 1))
    dist_barrier(world)
    with ClockSampler(local) as clk:
        results = server.run(mine)
    wall = dist_max(server.wall_seconds, world)
    cell_steps = dist_sum(server.cell_steps, world)
    merged = serve.gather_results(results, world)
    if rank == 0:
        summary = serve.summarize(merged, wall, cell_steps)
        line = dict(metric='served solves/s and p50/p99 latency (converged and capped apart)', impl='ours',
                    value=summary['completed_per_s'], unit='solves/s', n_gpus=world, higher_is_better=True,
                    scaling='weak', dtype='f32', data='synthetic',
                    config=dict(workload='served-sa-fp32', requests=args.requests, rate_per_s=args.rate, seed=args.seed,
                                max_steps=args.max_steps, profiles='LF1:LF2 1:1', arena_cases=args.serve_cases,
                                meshes='native host builder, seeded NACA 4-digit draws'),
                    serving=summary, polls=server.polls, clocks=clk.summary())
        print(json.dumps(line), flush=True)
    dist_barrier(world)


def dist_sum(value, world):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=320)
    ap.add_argument('--warmup', type=int, default=64)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--cases', type=int, default=256)
    ap.add_argument('--no-cpu', action='store_true')
    ap.add_argument('--profile', choices=['persistent', 'phases', 'split', 'tiled'], default=None,
                    help='only the timed batched loop, with this launch mode and --block (for ncu)')
    ap.add_argument('--block', type=int, default=128)
    ap.add_argument('--precision', type=int, default=32, choices=[32, 64])
    ap.add_argument('--serve', action='store_true', help='the served form: Poisson arrivals, p50/p99 latency')
    ap.add_argument('--requests', type=int, default=200)
    ap.add_argument('--rate', type=float, default=50.0)
    ap.add_argument('--max-steps', type=int, default=3000)
    ap.add_argument('--serve-cases', type=int, default=512)
    ap.add_argument('--seed', type=int, default=20261203)
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    rank, world, local = dist_setup(args.gpus)
    if args.impl == 'reference':
        reference_arm(args, rank, world)
        return
    if args.serve:
        run_serving(args, rank, world, local)
        return
    case_list = batched_cases(args.cases, seed=20261203 + rank)
    if args.profile:
        mode = {'phases': _abi.LAUNCH_PHASES, 'split': _abi.LAUNCH_SPLIT,
                'tiled': _abi.LAUNCH_TILED}.get(args.profile, _abi.LAUNCH_PERSISTENT)
        b = Batch(precision=args.precision, model=_abi.MODEL_LAMINAR, sa=True, max_cases=len(case_list),
                  max_cells=sum(m.n_cells for _, m in case_list) + 64, device=local, block_threads=args.block,
                  launch_mode=mode)
        for spec, mesh in case_list:
            b.admit(mesh, spec.params(), cases.initial_state(mesh, spec.initial_primitive()),
                    case_control(1e30, 10 ** 9, steady=False))
        done = 0
        while done < args.warmup:
            k = min(32, args.warmup - done)
            b.advance(k)
            done += k
        done, sec = 0, 0.0
        while done < args.steps:
            k = min(32, args.steps - done)
            b.advance(k)
            sec += b.last_advance_seconds
            done += k
        print(json.dumps(dict(profile=args.profile, cases=len(case_list), precision=args.precision, block=args.block,
                              launch=b.launch_config(), ms_per_step=1e3 * sec / max(1, args.steps))))
        return
    hbm, peak_kind = peaks()
    dist_barrier(world)
    clk = ClockSampler(local, interval_ms=50)
    r = run_batched(case_list, 32, args.steps, args.warmup, device=local, clock=clk)
    dev_seconds = dist_max(r['dev_seconds'], world)
    cell_steps = r['cell_steps']
    value = cell_steps * world / dev_seconds
    cfg = r['config']
    block, grid, mode = parse_launch(cfg)
    # the device-timed batch is freed after the end-to-end run, so that its teardown in the driver
    # does not overlap (and slow) the end-to-end run's own batch creation
    e2e = run_e2e(case_list, 32, args.steps, device=local, block=block, grid=grid, mode=mode)
    r.pop('batch').destroy()
    e2e_value = e2e['value'] * world
    # roofline of the persistent kernel: algorithmic bytes per launch / launch duration
    bytes_per_step = sum(algorithmic_bytes(m) for _, m in case_list)
    per_launch = r['dev_seconds'] / r['advances']
    achieved = bytes_per_step * (args.steps / r['advances']) / per_launch / 1e9
    mean_cells = sum(m.n_cells for _, m in case_list) / len(case_list)
    line = dict(metric=METRIC, value=value, unit='cell-steps/s', n_gpus=world, steps=args.steps, warmup=args.warmup,
                ms_per_step=1e3 * dev_seconds / args.steps, higher_is_better=True, scaling='weak', vs_baseline=None,
                dtype='f32', data='synthetic',
                config=dict(workload='batched-sa-fp32-256', cases=args.cases * world,
                            meshes='NACA 2412 LF1 (%d cells) / LF2 (%d cells), 1:1, replicated with seeded M~U[1.2,2], '
                                   'AoA~U[-3,5]' % (case_list[0][1].n_cells, case_list[1][1].n_cells),
                            cells=sum(m.n_cells for _, m in case_list), solve_steps=SOLVE_STEPS,
                            solves_per_s=value / mean_cells / SOLVE_STEPS,
                            l2='working set > L2 (no flush needed)', launch=cfg, parallelism='replicas'),
                roofline=dict(bound='hbm', achieved=achieved, peak=hbm, unit='GB/s', frac=achieved / hbm,
                              peak_kind=peak_kind,
                              traffic=(SPLIT_256_TRAFFIC_PER_STEP * args.steps / r['advances']
                                       if 'mode=split' in cfg and args.cases == 256 else None),
                              traffic_scope='DRAM bytes per launch (a graph of steps_per_launch steps), ncu, cold cache',
                              bytes_per_step=bytes_per_step,
                              launch_ms=1e3 * per_launch, steps_per_launch=args.steps / r['advances']),
                e2e=dict(value=e2e_value, unit='cell-steps/s', h2d_bytes_per_step=e2e['h2d'] / args.steps,
                         d2h_bytes_per_step=e2e['d2h'] / args.steps, seconds=e2e['seconds'],
                         phases_seconds=e2e['phases']),
                gpu_launches=r['launches'], clocks=clk.summary(),
                rejected=sum(st['rejected'] for st in r['status']))
    if rank == 0:
        plain = plain_fp64(case_list, 256)
        pv = sum(p['cells'] * p['steps'] for p in plain.values()) / sum(p['seconds'] for p in plain.values())
        line['plain_fp64'] = dict(cell_steps_per_s=pv, per_profile=plain, batched_over_plain=value / world / pv)
        if not args.no_cpu:
            threads = os.cpu_count() or 1
            cv, detail = cpu_reference(case_list, 400, 200, threads)
            line['cpu_baseline'] = dict(value=cv, unit='cell-steps/s', cores=threads, kind='reference',
                                        sample='1 LF1 x 400 steps + 1 LF2 x 200 steps of the workload (reference CPU '
                                               'core, OpenMP)', cpu=cpu_model(), detail=detail)
        print(json.dumps(line), flush=True)
    dist_barrier(world)


if __name__ == '__main__':
    main()
