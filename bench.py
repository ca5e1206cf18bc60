"""Benchmark of the static-AMR explicit time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload batched|accuracy|time-accurate|serve]

One step = one SSP-RK3 step (one trial) of every case in the batch.

Workload `batched` (the default): 256 seeded NACA 4-digit airfoils (m~U[0,0.06], p~U[0.2,0.6],
t~U[0.08,0.15]; a draw the mesh builder rejects is redrawn and counted), half on LF1 and half on
LF2 meshes, SA-neg with Sutherland viscosity, HLLC, M~U[1.2,2.0], AoA~U[-3,5] deg, FP32 state with
FP64 dt, norms and loads, in one arena (batch); with --arenas N the cases are dealt into N batches
whose trials are in flight together (amr_batch_group_advance).  `value` is whole-job accepted
cell-steps per second over exactly K timed steps, CUDA events from one start event to the last
arena's end; `e2e` is the same work through the C ABI from host buffers (arena creation, mesh and
state upload, the K steps, download of every state) on the host clock.  Beside it: a measured 5000-step solve of the same cases (solves/s), the plain FP64
session on the same meshes, the plain FP64 inviscid Euler+SRD NACA 0012 LF1 case (200 steps) with
the reference CPU core at 1 thread and at all host threads, and the reference CPU core on a
bounded sample of the workload.

Workload `accuracy`: NACA 2412 on LF2, SA, run to the steady criteria or 20000 steps in FP64 and in
FP32, with the CL/CD/CM and per-field errors of the FP32 form.  `time-accurate`: 128 seeded LF2
cases, laminar with constant viscosity, AUSM+-up, pressure outlet on xmax, integrated to t*=1 in
FP32 and FP64, with the per-cell errors of rho, u, v, p.  `serve`: the served form (Poisson
arrivals, continuous batching, p50/p99 latency).
"""
import argparse
import ctypes
import json
import math
import os
import pathlib
import select
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import _abi, cases, runs, workloads  # noqa: E402
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.batch import (  # noqa: E402
    Batch, case_control, group_advance)
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.mesh import MeshArrays  # noqa: E402
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.session import StaticAmrGpu, default_options  # noqa: E402

METRIC = 'solves/s & cell-steps/s at |ΔCL|,|ΔCD|≤1e-4 vs plain FP64; p50/p99 latency'
GOLDEN = ROOT / 'tests' / 'golden'
SOLVE_STEPS = 5000  # steps per solve of the batched workload
# DRAM bytes (read + write) of one step of the default workload (256 cases, split launch mode): the
# nine split-kernel launches of one trial captured with ncu (dram__bytes_read.sum +
# dram__bytes_write.sum, caches flushed before every launch) on the first 64 draws of the same
# stream (614.0 MB for 454,622 cells), scaled by cells to the 256-case workload (1,818,201 cells).
# It comes from that separate capture, not from the timed run.
SPLIT_256_TRAFFIC_PER_STEP = 2.412e9
TRAFFIC_SOURCE = ('separate ncu capture (dram__bytes_read.sum + dram__bytes_write.sum, cold cache) of the nine '
                  'split-kernel launches of one trial of `bench.py --profile split --cases 64 --lanes 1`, scaled by cells to '
                  'the 256-case workload')


def peaks():
    p = ROOT / 'MEASURED_PEAKS.json'
    if p.exists():
        d = json.loads(p.read_text())
        return d['hbm_gbs'], 'measured'
    return 6650.0, 'fallback'


def algorithmic_bytes(mesh, s=4, sg=4):
    """Compulsory HBM bytes of one accepted step of one case (intermediates count 0):
    8*nv*s*n state traffic + 3*[n*c_cell + nf*c_face + nw*c_wall + T*c_term + S_srd], plus, for the
    FP32 form's two-word accepted state, the read and write of the trailing word in the final stage
    (2*nv*4*n)."""
    n, nf, nw, nv = mesh.n_cells, mesh.n_faces, mesh.n_walls, mesh.nv
    viscous = mesh.laminar
    T = int(mesh.visc_offsets[-1]) if viscous else 0
    c_cell = 8 + 4 + ((sg + 4) if viscous else 0)
    c_face = 8 + 4 + 8 + sg + (5 * sg if viscous else 0)
    c_wall = 4 + 3 * sg + ((4 + sg) if viscous else 0)
    c_term = 4 + 2 * sg
    srd = 0
    if mesh.small_cells:
        sizes = np.diff(mesh.group_offsets.astype(np.int64))
        srd = 16 * int(sizes[sizes > 1].sum())
    trailing = 2 * nv * 4 * n if s == 4 else 0
    return 8 * nv * s * n + trailing + 3 * (n * c_cell + nf * c_face + nw * c_wall + T * c_term + srd)


def _cuda_pci_bus_id(device):
    try:
        rt = ctypes.CDLL('libcudart.so.12')
        buf = ctypes.create_string_buffer(64)
        if rt.cudaDeviceGetPCIBusId(buf, 64, int(device)) == 0:
            return buf.value.decode()
    except OSError:
        pass
    return None


class NvmlSampler:
    """SM clock and clock-event reasons read through NVML every `interval_s` while entered.  It is
    entered around the timed region itself, which at the driver's step counts lasts only tens of
    milliseconds (too short for nvidia-smi's sampling)."""
    REASONS = {8: 'hw_slowdown', 64: 'hw_thermal_slowdown', 32: 'sw_thermal_slowdown', 4: 'sw_power_cap',
               128: 'hw_power_brake_slowdown'}

    def __init__(self, device, interval_s=0.0005):
        self.device = device
        self.interval_s = interval_s
        self.samples = []
        self.max_mhz = None
        self._stop = threading.Event()
        self._thread = None
        self._h = None

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            bus = _cuda_pci_bus_id(self.device)
            self._h = (pynvml.nvmlDeviceGetHandleByPciBusId(bus) if bus else pynvml.nvmlDeviceGetHandleByIndex(self.device))
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM))
            self._nvml = pynvml
            self._thread = threading.Thread(target=self._loop, daemon=True)
            self._thread.start()
        except Exception:
            self._h = None
        return self

    def _loop(self):
        nv = self._nvml
        while not self._stop.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM)
                reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                self.samples.append((float(mhz), int(reasons)))
            except Exception:
                break
            time.sleep(self.interval_s)

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread:
            self._thread.join(timeout=5)

    def summary(self):
        sm = [s for s, _ in self.samples]
        reasons = set()
        for _, bits in self.samples:
            for bit, name in self.REASONS.items():
                if bits & bit:
                    reasons.add(name)
        return dict(sm_mhz=statistics.median(sm) if sm else None, sm_max_mhz=self.max_mhz, reasons=sorted(reasons),
                    samples=len(sm), source='NVML, timed region only')


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every `interval_ms` while entered (used
    around the longer legs: warm-up, timed loop and the full solve)."""
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
                    samples=len(sm), source='nvidia-smi, warm-up + timed loop + full solve')


def parse_launch(cfg):
    """(block, grid, launch_mode) of a launch_config() string."""
    block = int(cfg.split('block=')[1].split()[0])
    grid = int(cfg.split('grid=')[1].split()[0])
    mode = (_abi.LAUNCH_PHASES if 'mode=phases' in cfg else _abi.LAUNCH_SPLIT if 'mode=split' in cfg
            else _abi.LAUNCH_TILED if 'mode=tiled' in cfg else _abi.LAUNCH_PERSISTENT)
    return block, grid, mode


LANES = 0  # --lanes: split-mode lanes of the batched and profile legs (0: the engine's default)


def new_batch(case_list, precision, device=0, block=0, grid=0, mode=0):
    kw = workloads.batch_kwargs(case_list)
    b = Batch(precision=precision, device=device, block_threads=block, grid_blocks=grid, launch_mode=mode, **kw)
    if LANES:
        b.set_lanes(LANES)
    return b


def admit_all(b, case_list, steps_cap=10 ** 9):
    items = [(m, s.params(), cases.uniform_state(m, s.initial_primitive()),
              case_control(1e30, steps_cap, steady=False, mach=s.mach, aoa=s.aoa)) for s, m in case_list]
    slots = b.admit_many(items)
    assert all(s is not None for s in slots), 'arena too small'
    return slots


def arena_parts(case_list, arenas):
    """The workload's cases dealt round-robin into `arenas` batches (LF1 and LF2 stay 1:1 in each)."""
    return [case_list[i::arenas] for i in range(arenas)]


def run_batched(case_list, precision, steps, warmup, device=0, trials=32, arenas=1):
    """Admit every case into `arenas` batches, autotune each, warm up, then time exactly `steps`
    trials of all of them with their work in flight together (amr_batch_group_advance: CUDA events
    from one start event to the last batch's end).  Accepted cell-steps are counted per case from
    the device counters.  The NVML sampler covers the timed loop alone."""
    parts = arena_parts(case_list, arenas)
    bs = [new_batch(part, precision, device) for part in parts]
    slots = [admit_all(b, part) for b, part in zip(bs, parts)]
    for b in bs:
        b.autotune(4)
    done = 0
    while done < warmup:
        k = min(trials, warmup - done)
        group_advance(bs, k)
        done += k
    before = [[b.status(x)['steps'] for x in sl] for b, sl in zip(bs, slots)]
    launches0 = sum(b.kernel_launches for b in bs)
    dev_seconds, adv, advances = 0.0, 0, 0
    with NvmlSampler(device) as nvml:
        while adv < steps:
            k = min(trials, steps - adv)
            dev_seconds += group_advance(bs, k)
            adv += k
            advances += 1
    status = [[b.status(x) for x in sl] for b, sl in zip(bs, slots)]
    cell_steps = sum(m.n_cells * (st['steps'] - b0) for part, sts, bef in zip(parts, status, before)
                     for (_, m), st, b0 in zip(part, sts, bef))
    return dict(batches=bs, dev_seconds=dev_seconds, launches=sum(b.kernel_launches for b in bs) - launches0,
                cell_steps=cell_steps, status=[x for sts in status for x in sts], config=bs[0].launch_config(),
                advances=advances, nvml=nvml.summary(), arenas=arenas)


def run_solve(case_list, nsteps, device, block, grid, mode, trials=32, arenas=1):
    """A full solve of the workload: every case from its freestream start to `nsteps` accepted
    steps, its arenas advanced together, device time from CUDA events; solves/s = cases / that
    time (measured, not extrapolated)."""
    parts = arena_parts(case_list, arenas)
    bs = []
    try:
        for part in parts:
            bs.append(new_batch(part, 32, device, block, grid, mode))
        slots = [admit_all(b, part, nsteps) for b, part in zip(bs, parts)]
        t0 = time.perf_counter()
        dev = 0.0
        polls = 0
        while True:
            dev += group_advance(bs, trials)
            polls += 1
            st = [b.status(x) for b, sl in zip(bs, slots) for x in sl]
            if all(x['status'] == _abi.STATUS_MAXSTEPS for x in st) or polls > nsteps:
                break
        wall = time.perf_counter() - t0
        steps = [x['steps'] for x in st]
        cells = [m.n_cells for part in parts for _, m in part]
        cell_steps = sum(c * x for c, x in zip(cells, steps))
        return dict(steps_per_solve=nsteps, cases=len(case_list), arenas=arenas, device_seconds=dev, host_seconds=wall,
                    solves_per_s=len(case_list) / dev, cell_steps_per_s=cell_steps / dev,
                    all_cases_completed=all(x == nsteps for x in steps), rejected=sum(x['rejected'] for x in st))
    finally:
        for b in bs:
            b.destroy()


def run_e2e(case_list, precision, steps, device=0, trials=32, block=0, grid=0, mode=0, arenas=1):
    """The same work end to end through the C ABI from host buffers: creation of the arenas, mesh
    and state upload of every case (one bulk admission per arena), `steps` trials of all arenas
    together with a control read-back per launch, and the download of every final state (one bulk
    download per arena); host wall clock."""
    parts = arena_parts(case_list, arenas)
    t0 = time.perf_counter()
    bs = [new_batch(part, precision, device, block, grid, mode) for part in parts]
    t_create = time.perf_counter()
    items, h2d = [[] for _ in parts], 0
    for lst, part in zip(items, parts):
        for spec, mesh in part:
            u0 = cases.uniform_state(mesh, spec.initial_primitive())  # filled on the device
            lst.append((mesh, spec.params(), u0, case_control(1e30, 10 ** 9, steady=False)))
            h2d += mesh_bytes(mesh, precision) + u0.nbytes
    t_items = time.perf_counter()
    slots = [b.admit_many(lst) for b, lst in zip(bs, items)]
    t_admit = time.perf_counter()
    adv, advances = 0, 0
    while adv < steps:
        k = min(trials, steps - adv)
        group_advance(bs, k)
        adv += k
        advances += 1
    t_advance = time.perf_counter()
    d2h = 0
    cell_steps = 0
    for b, part, sl in zip(bs, parts, slots):
        states = b.download_many(sl)  # one staged copy, one synchronisation
        for (_, mesh), x, u in zip(part, sl, states):
            d2h += u.nbytes * precision // 64 * 2  # leading and trailing FP32 words
            cell_steps += mesh.n_cells * b.status(x)['steps']
    t_end = time.perf_counter()
    seconds = t_end - t0
    d2h += advances * 96 * len(case_list)  # per-launch control read-back
    for b in bs:
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


def time_plain(spec, mesh, steps):
    """The plain FP64 session on one case: a first session warms up (graph capture, autotune); a
    second, with the chosen launch, runs `steps` steps timed by CUDA events."""
    u0 = cases.initial_state(mesh, spec.initial_primitive())
    w = StaticAmrGpu.create(mesh, spec.params(), u0)
    w.advance(1e30, 64)
    cfg = w.launch_config()
    w.destroy()
    block, grid, mode = parse_launch(cfg)
    s = StaticAmrGpu.create(mesh, spec.params(), u0, options=default_options(block_threads=block, grid_blocks=grid,
                                                                             launch_mode=mode))
    s.advance(1e30, steps)
    st = s.stats()
    sec = st['advance_event_seconds']
    out = dict(cells=mesh.n_cells, steps=s.steps, seconds=sec, us_per_step=1e6 * sec / s.steps,
               cell_steps_per_s=mesh.n_cells * s.steps / sec, config=cfg, polls=st['status_polls'])
    s.destroy()
    return out


def plain_fp64(case_list, steps):
    """The plain FP64 session on the first case of each profile of the workload."""
    res = {}
    for profile in ('LF1', 'LF2'):
        spec, mesh = [c for c in case_list if c[0].profile == profile][0]
        res[profile] = time_plain(spec, mesh, steps)
    return res


def _ref_subprocess(code, threads):
    """Runs `code` in a fresh interpreter with the OpenMP thread count fixed before the runtime loads;
    returns the JSON object of its last output line."""
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND='false')
    r = subprocess.run([sys.executable, '-c', code], capture_output=True, text=True, env=env, cwd=str(ROOT))
    if r.returncode:
        raise RuntimeError(r.stderr[-2000:])
    return json.loads(r.stdout.strip().splitlines()[-1])


def cpu_reference(steps_lf1, steps_lf2, threads, seed):
    """The reference CPU core (oracle/_ref, OpenMP build) on the first LF1 and the first LF2 case of
    the workload's draws, meshes built by the reference builder; cell-steps per second."""
    code = f'''
import json, sys
sys.path.insert(0, {str(ROOT)!r})
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import airfoils, cases, workloads
from oracle.oracle import RefCase
out = {{}}
for spec, n in zip(workloads.batched_sa_specs(2, {seed}), ({steps_lf1}, {steps_lf2})):
    x, y, pt = airfoils.naca4(*spec.naca)
    rc = RefCase.build(spec, x, y, pt, kind='omp')
    u0 = rc.initial(spec.initial_primitive())
    sec, r = rc.run_timed(u0, 1e30, n)
    out[spec.profile] = dict(cells=rc.counts['n'], steps=r['steps'], seconds=sec)
print(json.dumps(out))
'''
    d = _ref_subprocess(code, threads)
    cell_steps = sum(v['cells'] * v['steps'] for v in d.values())
    seconds = sum(v['seconds'] for v in d.values())
    return cell_steps / seconds, d


def config1_leg(steps=200):
    """Plain FP64 inviscid Euler + SRD, NACA 0012 LF1 (the reference's CPU-runnable case), 200 steps:
    the FP64 session on the GPU beside the reference CPU core at 1 thread (the reference driver's
    default, OMP_NUM_THREADS=1) and at every host thread."""
    mesh = MeshArrays.load(GOLDEN / 'mesh_naca0012_lf1_euler_srd.npz')
    spec = cases.CaseSpec(physics='euler', profile='LF1', mach=1.65, aoa=1.5)
    gpu = time_plain(spec, mesh, steps)
    code = f'''
import json, sys
sys.path.insert(0, {str(ROOT)!r})
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import cases
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.mesh import MeshArrays
from oracle.oracle import RefCase
mesh = MeshArrays.load({str(GOLDEN / 'mesh_naca0012_lf1_euler_srd.npz')!r})
spec = cases.CaseSpec(physics='euler', profile='LF1', mach=1.65, aoa=1.5)
rc = RefCase.from_mesh(mesh, spec.params(), kind=sys.argv[1] if len(sys.argv) > 1 else 'KIND')
u0 = cases.initial_state(mesh, spec.initial_primitive())
rc.run_timed(u0, 1e30, 5)
sec, r = rc.run_timed(u0, 1e30, {steps})
print(json.dumps(dict(cells=mesh.n_cells, steps=r['steps'], seconds=sec)))
'''
    threads = os.cpu_count() or 1
    one = _ref_subprocess(code.replace("'KIND'", "'serial'"), 1)
    allc = _ref_subprocess(code.replace("'KIND'", "'omp'"), threads)
    cpu = {}
    for name, d, t in (('1_thread', one, 1), ('all_threads', allc, threads)):
        cpu[name] = dict(threads=t, ms_per_step=1e3 * d['seconds'] / d['steps'],
                         cell_steps_per_s=d['cells'] * d['steps'] / d['seconds'])
    return dict(workload='plain-fp64-euler-srd-naca0012-lf1', cells=mesh.n_cells, steps=steps,
                gpu=dict(us_per_step=gpu['us_per_step'], cell_steps_per_s=gpu['cell_steps_per_s'], launch=gpu['config']),
                cpu_reference=cpu, cpu=cpu_model(),
                gpu_over_cpu_1_thread=gpu['cell_steps_per_s'] / cpu['1_thread']['cell_steps_per_s'],
                gpu_over_cpu_all_threads=gpu['cell_steps_per_s'] / cpu['all_threads']['cell_steps_per_s'])


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


def dist_sum(value, world):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def dist_barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def rank_seed(rank):
    return workloads.SEED + 1000 * rank


def reference_arm(args, rank, world):
    """--impl reference: the reference CPU implementation (oracle/_ref with all host threads) on
    the same workload, each step a bounded sample (the first LF1 and LF2 cases of the draws)."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    n_lf1, n_lf2 = 40, 20
    values = []
    for _ in range(max(1, args.warmup)):
        cpu_reference(4, 2, threads, rank_seed(0))
    for _ in range(args.steps):
        v, detail = cpu_reference(n_lf1, n_lf2, threads, rank_seed(0))
        values.append(v)
    value = statistics.median(values)
    line = dict(metric=METRIC, impl='reference', value=value, unit='cell-steps/s', n_gpus=args.gpus,
                steps=args.steps, warmup=args.warmup, higher_is_better=True, scaling='weak', vs_baseline=None,
                dtype='f64', data='synthetic',
                config=dict(workload='batched-sa-fp32-%d' % args.cases,
                            sample=f'1 LF1 x {n_lf1} + 1 LF2 x {n_lf2} steps per step (first draws of the workload)'),
                cpu_baseline=dict(value=value, unit='cell-steps/s', cores=threads, kind='reference',
                                  sample=f'1 LF1 ({detail["LF1"]["cells"]} cells) x {n_lf1} steps + 1 LF2 '
                                         f'({detail["LF2"]["cells"]} cells) x {n_lf2} steps', cpu=cpu_model()),
                e2e=dict(value=value, unit='cell-steps/s', h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)


def serving_arena(args, device):
    """Factory of one serving arena: FP32 SA batch of args.arena_cases cases (9800 cells each)."""
    return lambda: Batch(precision=32, model=_abi.MODEL_LAMINAR, sa=True, max_cases=args.arena_cases,
                         max_cells=args.arena_cases * 9800, device=device, launch_mode=_abi.LAUNCH_SPLIT,
                         block_threads=128)


def plain_fp64_solves(items, max_steps):
    """The plain FP64 path on (spec, mesh) items, one case at a time to the steady criteria or the
    step cap (the FP64 batch of one case is bit for bit the single-case FP64 session); host wall
    time per case, polls and checks included."""
    out = []
    for spec, mesh in items:
        t0 = time.perf_counter()
        (r,), dev = runs.solve([(spec, mesh)], 64, runs.steady_control(max_steps=max_steps), download=False)
        out.append(dict(r, wall=time.perf_counter() - t0, device_seconds=dev))
    return out


def run_serving(args, rank, world, local):
    """--workload serve: the served form.  Poisson request arrivals (seeded), host mesh builds on a
    thread pool, admission into arenas by free device memory (and an optional live-cell cap),
    device steady-rule retirement or the step cap; then the loads of a sample of the requests
    against the plain FP64 path at the same cap.  Each rank serves its shard on its own GPU; rank 0
    prints one JSON line."""
    from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import serve
    reqs = serve.poisson_requests(args.requests, args.rate, args.seed)
    mine = serve.shard(reqs, rank, world)
    server = serve.Server(serving_arena(args, local), max_steps=args.max_steps, trials=32, device=local,
                          builder_threads=max(1, (os.cpu_count() or 2) - 1), hbm_reserve=args.hbm_reserve,
                          max_live_cells=args.max_live_cells or None)
    dist_barrier(world)
    with ClockSampler(local) as clk:
        results = server.run(mine)
    wall = dist_max(server.wall_seconds, world)
    cell_steps = dist_sum(server.cell_steps, world)
    merged = serve.gather_results(results, world)
    if rank == 0:
        summary = serve.summarize(merged, wall, cell_steps)
        # loads against the plain FP64 path on a sample (first LF1 and LF2 requests), same cap
        sample = [r for r in reqs if r.spec.profile == 'LF1'][:args.plain_sample // 2] + \
                 [r for r in reqs if r.spec.profile == 'LF2'][:args.plain_sample // 2]
        plain = plain_fp64_solves([(r.spec, serve.build_request_mesh(r)) for r in sample], args.max_steps)
        by_id = {r.id: r for r in merged}
        errs = [dict(id=q.id, profile=q.spec.profile, steps32=by_id[q.id].steps, steps64=p['steps'],
                     dcl=abs(by_id[q.id].cl - p['cl']), dcd=abs(by_id[q.id].cd - p['cd']), dcm=abs(by_id[q.id].cm - p['cm']))
                for q, p in zip(sample, plain)]
        line = dict(metric='served solves/s and p50/p99 latency (converged and capped apart)', impl='ours',
                    value=summary['completed_per_s'], unit='solves/s', n_gpus=world, higher_is_better=True,
                    scaling='weak', dtype='f32', data='synthetic',
                    config=dict(workload='served-sa-fp32', requests=args.requests, rate_per_s=args.rate, seed=args.seed,
                                max_steps=args.max_steps, profiles='LF1:LF2 1:1', arena_cases=args.arena_cases,
                                hbm_reserve=args.hbm_reserve, max_live_cells=args.max_live_cells or None,
                                meshes='native host builder, seeded NACA 4-digit draws'),
                    serving=summary, polls=server.polls, arenas=dict(peak=server.peak_arenas, created=server.arenas_created,
                                                                      bytes_each=server.arena_bytes),
                    peak_live_cells=server.peak_live_cells,
                    loads_vs_plain_fp64=dict(sample=errs, max_dcl=max(e['dcl'] for e in errs),
                                             max_dcd=max(e['dcd'] for e in errs), max_dcm=max(e['dcm'] for e in errs)),
                    clocks=clk.summary())
        print(json.dumps(line), flush=True)
    dist_barrier(world)


def converged_leg(args):
    """--workload converged: converged solves per second of the served FP32 form against the plain
    FP64 path on the same request mix.  args.requests requests of the served distribution arrive
    at once and run to the steady criteria (cap args.max_steps); the plain FP64 path solves a
    sample of the same requests one at a time; both converged-solve rates, their ratio, and the
    loads of the sampled requests against each other."""
    from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import serve
    reqs = serve.poisson_requests(args.requests, 1e9, args.seed)
    server = serve.Server(serving_arena(args, 0), max_steps=args.max_steps, trials=32,
                          builder_threads=max(1, (os.cpu_count() or 2) - 1), hbm_reserve=args.hbm_reserve)
    with ClockSampler(0) as clk:
        results = server.run(reqs)
    summary = serve.summarize(results, server.wall_seconds, server.cell_steps)
    sample = [r for r in reqs if r.spec.profile == 'LF1'][:args.plain_sample // 2] + \
             [r for r in reqs if r.spec.profile == 'LF2'][:args.plain_sample // 2]
    plain = plain_fp64_solves([(r.spec, serve.build_request_mesh(r)) for r in sample], args.max_steps)
    plain_wall = sum(p['wall'] for p in plain)
    plain_conv = sum(1 for p in plain if p['converged'])
    by_id = {r.id: r for r in results}
    errs = [dict(id=q.id, profile=q.spec.profile, converged32=by_id[q.id].outcome == 'converged',
                 converged64=bool(p['converged']), steps32=by_id[q.id].steps, steps64=p['steps'],
                 dcl=abs(by_id[q.id].cl - p['cl']), dcd=abs(by_id[q.id].cd - p['cd']), dcm=abs(by_id[q.id].cm - p['cm']))
            for q, p in zip(sample, plain)]
    fp32_rate = summary['converged_per_s']
    fp64_rate = plain_conv / plain_wall if plain_wall > 0 else 0.0
    line = dict(workload='converged-solves-fp32-served-vs-plain-fp64', requests=args.requests, max_steps=args.max_steps,
                seed=args.seed, arena_cases=args.arena_cases,
                fp32_served=dict(converged_per_s=fp32_rate, wall_seconds=server.wall_seconds,
                                 outcomes=summary['outcomes'], cell_steps_per_s=summary.get('cell_steps_per_s'),
                                 peak_arenas=server.peak_arenas, latency=summary['latency']),
                plain_fp64=dict(converged_per_s=fp64_rate, sample=len(sample), converged=plain_conv, wall_seconds=plain_wall,
                                note='one case at a time; rate from a sample of the same requests'),
                ratio=fp32_rate / fp64_rate if fp64_rate > 0 else None,
                loads_sample=errs, max_dcl=max(e['dcl'] for e in errs), max_dcd=max(e['dcd'] for e in errs),
                clocks=clk.summary())
    print(json.dumps(line), flush=True)


def g0001_items():
    """The reference's example G0001 on LF1 and LF2 with the reference pipeline's default settings
    (tests/golden: the settings text and the contour prepared by the reference's own pipeline);
    meshes from the native builder (bit-identical tables to the reference builder's)."""
    from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import builder, settings
    ka = json.loads((GOLDEN / 'known_answers.json').read_text())
    z = np.load(GOLDEN / 'examples.npz')
    i = list(z['names']).index('G0001')
    a, b = z['offsets'][i], z['offsets'][i + 1]
    items = []
    for profile in ('LF1', 'LF2'):
        s, boxes = settings.parse_settings(ka['settings']['default_' + profile])
        spec = settings.SettingsSpec(s, boxes, profile)
        items.append((spec, builder.build_mesh(spec, z['x'][a:b], z['y'][a:b], z['patches'][a:b])))
    return items, ka['full_steady']


def g0001_steady(args):
    """G0001 LF1 and LF2 to the steady criteria in FP64 and FP32 (two-word state), with the
    residual norms and loads of every check, against the reference's published FP64 solve."""
    items, published = g0001_items()
    ctl = runs.steady_control(stop_time=100.0)
    r64, s64 = runs.solve(items, 64, ctl, history=True)
    r32, s32 = runs.solve(items, 32, ctl, history=True)
    out = {}
    for (spec, mesh), a, b in zip(items, r32, r64):
        pub = published[spec.profile]
        same_t = a['time'] == b['time']
        out[spec.profile] = dict(
            cells=mesh.n_cells, published=pub,
            fp64=dict(converged=b['converged'], steps=b['steps'], time=b['time'], cl=b['cl'], cd=b['cd'], cm=b['cm'],
                      dcl_published=b['cl'] - pub['Cl'], dcd_published=b['cd'] - pub['Cd'],
                      dcm_published=b['cm'] - pub['Cm'], history=b['history']),
            fp32=dict(converged=a['converged'], steps=a['steps'], time=a['time'], cl=a['cl'], cd=a['cd'], cm=a['cm'],
                      history=a['history']),
            load_error=runs.load_errors(a, b),
            field_error_at_common_time=runs.field_errors(a['u'], b['u'], mesh.nv) if same_t else None)
    return dict(device_seconds=dict(fp64=s64, fp32=s32), cases=out)


def accuracy_leg(args):
    """NACA 2412 LF2 SA to the steady criteria or 20000 steps, FP64 and FP32: loads at every check
    and of the final states, and the per-field error of the FP32 final state; and G0001 LF1/LF2 to
    the steady criteria in FP64 and FP32 with their convergence histories."""
    w = workloads.naca2412_lf2_sa()
    spec, mesh = w.items[0]
    ctl = runs.steady_control(max_steps=args.accuracy_steps)
    out = {}
    for prec in (64, 32):
        res, sec = runs.solve(w.items, prec, ctl)
        r = res[0]
        out[prec] = dict(status=r['status'], steps=r['steps'], time=r['time'], converged=r['converged'],
                         checks=r['checks'], last_check=dict(cl=r['cl'], cd=r['cd'], cm=r['cm']),
                         final_state_loads=runs.loads_of_state(spec, mesh, r['u']), device_seconds=sec, u=r['u'])
    e_check = runs.load_errors(out[32]['last_check'], out[64]['last_check'])
    e_final = runs.load_errors(out[32]['final_state_loads'], out[64]['final_state_loads'])
    fields = runs.field_errors(out[32]['u'], out[64]['u'], mesh.nv)
    for p in out.values():
        p.pop('u')
    line = dict(workload='accuracy-naca2412-lf2-sa', cells=mesh.n_cells, max_steps=args.accuracy_steps,
                fp64=out[64], fp32=out[32], load_error_last_check=e_check, load_error_final_state=e_final,
                field_error_final_state=fields,
                note='FP32 and FP64 end at the same step count; their final times differ by the dt history',
                g0001_steady=g0001_steady(args))
    print(json.dumps(line), flush=True)


def time_accurate_leg(args):
    """128 seeded LF2 laminar AUSM+-up cases with a pressure outlet, to t*=1, FP32 against FP64:
    per-cell errors of rho, u, v, p (largest over the cases of each measure)."""
    w = workloads.time_accurate_laminar(args.ta_cases)
    res32, s32 = runs.solve(w.items, 32, runs.fixed_time(1.0))
    res64, s64 = runs.solve(w.items, 64, runs.fixed_time(1.0))
    worst = {}
    per_case = []
    for (spec, mesh), a, b in zip(w.items, res32, res64):
        e = runs.field_errors(a['u'], b['u'], mesh.nv)
        per_case.append(dict(mach=spec.mach, aoa=spec.aoa, steps32=a['steps'], steps64=b['steps'],
                             time32=a['time'], time64=b['time'], max_rel=max(v['max_rel'] for v in e.values())))
        for name, v in e.items():
            cur = worst.setdefault(name, dict(max_abs=0.0, max_rel=0.0, rms_rel=0.0))
            for k in cur:
                cur[k] = max(cur[k], v[k])
    cs32 = sum(m.n_cells * r['steps'] for (_, m), r in zip(w.items, res32))
    cs64 = sum(m.n_cells * r['steps'] for (_, m), r in zip(w.items, res64))
    line = dict(w.describe(), tend=1.0,
                fp32=dict(device_seconds=s32, cell_steps_per_s=cs32 / s32,
                          all_finished=all(r['time'] == 1.0 for r in res32), rejected=sum(r['rejected'] for r in res32)),
                fp64=dict(device_seconds=s64, cell_steps_per_s=cs64 / s64,
                          all_finished=all(r['time'] == 1.0 for r in res64), rejected=sum(r['rejected'] for r in res64)),
                steps=dict(min=min(r['steps'] for r in res64), max=max(r['steps'] for r in res64)),
                field_error_worst_case=worst,
                worst_cases=sorted(per_case, key=lambda c: -c['max_rel'])[:3])
    print(json.dumps(line), flush=True)


def profile_leg(args, local):
    """--profile MODE: only the timed batched loop with a fixed launch mode (for ncu)."""
    case_list = workloads.batched_sa(args.cases, seed=rank_seed(0)).items
    mode = {'phases': _abi.LAUNCH_PHASES, 'split': _abi.LAUNCH_SPLIT,
            'tiled': _abi.LAUNCH_TILED}.get(args.profile, _abi.LAUNCH_PERSISTENT)
    b = new_batch(case_list, args.precision, local, args.block, 0, mode)
    admit_all(b, case_list)
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=320)
    ap.add_argument('--warmup', type=int, default=64)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--workload', default='batched', choices=['batched', 'accuracy', 'time-accurate', 'serve', 'converged'])
    ap.add_argument('--cases', type=int, default=256)
    ap.add_argument('--no-cpu', action='store_true')
    ap.add_argument('--no-solve', action='store_true', help='skip the measured full-solve leg')
    ap.add_argument('--arenas', type=int, default=1,
                    help='batched workload: arenas (batches) the cases are dealt into, advanced together')
    ap.add_argument('--lanes', type=int, default=0,
                    help='split-mode lanes (amr_batch_set_lanes) of the batched and profile legs; 0: default (3)')
    ap.add_argument('--profile', choices=['persistent', 'phases', 'split', 'tiled'], default=None,
                    help='only the timed batched loop, with this launch mode and --block (for ncu)')
    ap.add_argument('--block', type=int, default=128)
    ap.add_argument('--precision', type=int, default=32, choices=[32, 64])
    ap.add_argument('--serve', action='store_true', help='same as --workload serve')
    ap.add_argument('--requests', type=int, default=200)
    ap.add_argument('--rate', type=float, default=50.0)
    ap.add_argument('--max-steps', type=int, default=3000)
    ap.add_argument('--arena-cases', type=int, default=64, help='cases per serving arena')
    ap.add_argument('--hbm-reserve', type=int, default=4 << 30, help='device bytes kept free when opening an arena')
    ap.add_argument('--max-live-cells', type=int, default=0, help='live-cell cap of the served form (0: none)')
    ap.add_argument('--plain-sample', type=int, default=4, help='requests the plain FP64 path solves for comparison')
    ap.add_argument('--seed', type=int, default=workloads.SEED)
    ap.add_argument('--accuracy-steps', type=int, default=20000)
    ap.add_argument('--ta-cases', type=int, default=128)
    args = ap.parse_args()
    global LANES
    LANES = args.lanes
    args.warmup = max(3, args.warmup)
    rank, world, local = dist_setup(args.gpus)
    if args.impl == 'reference':
        reference_arm(args, rank, world)
        return
    if args.serve or args.workload == 'serve':
        run_serving(args, rank, world, local)
        return
    if args.workload == 'accuracy':
        if rank == 0:
            accuracy_leg(args)
        return
    if args.workload == 'converged':
        if rank == 0:
            converged_leg(args)
        return
    if args.workload == 'time-accurate':
        if rank == 0:
            time_accurate_leg(args)
        return
    if args.profile:
        profile_leg(args, local)
        return
    work = workloads.batched_sa(args.cases, seed=rank_seed(rank))
    case_list = work.items
    hbm, peak_kind = peaks()
    dist_barrier(world)
    clk = ClockSampler(local, interval_ms=100)
    clk.__enter__()
    r = run_batched(case_list, 32, args.steps, args.warmup, device=local, arenas=args.arenas)
    dev_seconds = dist_max(r['dev_seconds'], world)
    cell_steps = dist_sum(r['cell_steps'], world)
    value = cell_steps / dev_seconds
    cfg = r['config']
    block, grid, mode = parse_launch(cfg)
    # the end-to-end run comes before any batch is freed: a batch's teardown in the driver can take
    # up to a second and, overlapping the next batch's creation, slows that creation
    e2e = run_e2e(case_list, 32, args.steps, device=local, block=block, grid=grid, mode=mode, arenas=args.arenas)
    for b in r.pop('batches'):
        b.destroy()
    solve = None if args.no_solve else run_solve(case_list, SOLVE_STEPS, local, block, grid, mode,
                                                 arenas=args.arenas)
    if solve is not None:  # whole-job figures: every rank solves its own cases at the same time
        solve['solves_per_s'] = dist_sum(solve['solves_per_s'], world)
        solve['cell_steps_per_s'] = dist_sum(solve['cell_steps_per_s'], world)
        solve['cases'] *= world
    clk.__exit__(None, None, None)
    e2e_value = dist_sum(e2e['value'], world)
    # roofline of the step: algorithmic bytes per launch / launch duration (CUDA events)
    bytes_per_step = sum(algorithmic_bytes(m) for _, m in case_list)
    per_launch = r['dev_seconds'] / r['advances']
    steps_per_launch = args.steps / r['advances']
    achieved = bytes_per_step * steps_per_launch / per_launch / 1e9
    traffic = (SPLIT_256_TRAFFIC_PER_STEP * steps_per_launch
               if SPLIT_256_TRAFFIC_PER_STEP and 'mode=split' in cfg and args.cases == 256 else None)
    desc = work.describe()
    line = dict(metric=METRIC, value=value, unit='cell-steps/s', n_gpus=world, steps=args.steps, warmup=args.warmup,
                ms_per_step=1e3 * dev_seconds / args.steps, higher_is_better=True, scaling='weak', vs_baseline=None,
                dtype='f32', data='synthetic',
                config=dict(workload=desc['workload'], cases=args.cases * world, cells=desc['cells'],
                            profiles=desc['profiles'], seed=desc['seed'], redraws=desc['redraws'],
                            meshes='seeded NACA 4-digit draws m~U[0,0.06] p~U[0.2,0.6] t~U[0.08,0.15], LF1:LF2 1:1, '
                                   'M~U[1.2,2], AoA~U[-3,5], SA-neg + Sutherland, HLLC, native mesh builder',
                            solve_steps=SOLVE_STEPS,
                            l2='working set > L2 (no flush needed)', launch=cfg, arenas=args.arenas,
                            parallelism='replicas'),
                roofline=dict(bound='hbm', achieved=achieved, peak=hbm, unit='GB/s', frac=achieved / hbm,
                              peak_kind=peak_kind, traffic=traffic,
                              traffic_source=TRAFFIC_SOURCE if traffic else None,
                              bytes_per_step=bytes_per_step, launch_ms=1e3 * per_launch,
                              steps_per_launch=steps_per_launch),
                e2e=dict(value=e2e_value, unit='cell-steps/s', h2d_bytes_per_step=e2e['h2d'] / args.steps,
                         d2h_bytes_per_step=e2e['d2h'] / args.steps, seconds=e2e['seconds'],
                         phases_seconds=e2e['phases']),
                gpu_launches=r['launches'], clocks=r['nvml'], clocks_under_load=clk.summary(),
                rejected=sum(st['rejected'] for st in r['status']))
    if solve is not None:
        line['solve'] = dict(solve, note='measured: every case run from its freestream start to %d steps' % SOLVE_STEPS)
        line['config']['solves_per_s'] = solve['solves_per_s']
    if rank == 0:
        plain = plain_fp64(case_list, 256)
        pv = sum(p['cells'] * p['steps'] for p in plain.values()) / sum(p['seconds'] for p in plain.values())
        line['plain_fp64'] = dict(cell_steps_per_s=pv, per_profile=plain, batched_over_plain=value / world / pv)
        if not args.no_cpu:
            threads = os.cpu_count() or 1
            cv, detail = cpu_reference(400, 200, threads, rank_seed(0))
            line['cpu_baseline'] = dict(value=cv, unit='cell-steps/s', cores=threads, kind='reference',
                                        sample='first LF1 draw x 400 steps + first LF2 draw x 200 steps of the workload '
                                               '(reference CPU core, OpenMP)', cpu=cpu_model(), detail=detail)
            line['config1'] = config1_leg()
        print(json.dumps(line), flush=True)
    dist_barrier(world)


if __name__ == '__main__':
    main()
