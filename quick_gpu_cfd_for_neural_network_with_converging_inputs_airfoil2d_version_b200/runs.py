"""Run-to-completion drivers over the batched engine, and the error measures between two runs.

    res = solve(items, precision=32, control=steady_control())    # until every case retires
    res = solve(items, precision=64, control=fixed_steps(20000))
    res = solve(items, precision=32, control=fixed_time(1.0))
    err = field_errors(res32[i]['u'], res64[i]['u'], mesh.nv)

`items` is a list of (CaseSpec, MeshArrays); all cases share one batch, each with its own time,
dt, retries and steady rule (the reference driver's, src/quick_airfoil.cpp:75-92, evaluated on the
device in FP64 after every poll).  The FP64 batch is bit-for-bit the single-case FP64 session on
every case, so a precision-64 run is the plain FP64 path's answer.
"""
import numpy as np

from . import _abi, cases
from .batch import Batch, case_control
from .workloads import batch_kwargs


def steady_control(stop_time=100.0, max_steps=10 ** 9, **steady):
    """The driver's steady rule: checks at first_check then every check_period, retirement after
    `hold` consecutive checks within tolerance once time >= min_time; stop_time caps the run."""
    return lambda spec: case_control(stop_time, max_steps, steady=True, mach=spec.mach, aoa=spec.aoa, **steady)


def fixed_steps(n):
    """Exactly n accepted steps (the run ends with the maxsteps status, as in the reference)."""
    return lambda spec: case_control(1e30, n, steady=False, mach=spec.mach, aoa=spec.aoa)


def fixed_time(tend, max_steps=10 ** 9):
    """Time-accurate run to exactly tend (the last step is clipped onto it)."""
    return lambda spec: case_control(tend, max_steps, steady=False, mach=spec.mach, aoa=spec.aoa)


def solve(items, precision, control, trials=32, launch_mode=0, download=True, device=0, max_polls=10 ** 7,
          history=False):
    """Admits every case, advances `trials` trials per poll and applies the steady rule after each
    poll until every case has retired.  Returns (results, device_seconds): per case the status
    record (time, steps, rejected, status, converged, cl, cd, cm, ...) and, with download, its
    accepted state u (FP64 copy); with history, the record of every steady check as 'history'
    (time, steps, residual norms, loads, hold)."""
    b = Batch(precision=precision, launch_mode=launch_mode, device=device, **batch_kwargs(items))
    try:
        entries = [(m, s.params(), cases.uniform_state(m, s.initial_primitive()), control(s)) for s, m in items]
        slots = b.admit_many(entries)
        if any(s is None for s in slots):
            raise RuntimeError('batch arena too small for the workload')
        if launch_mode == 0:
            b.autotune(4)
        seconds = 0.0
        live = set(slots)
        hist = {s: [] for s in slots}
        for _ in range(max_polls):
            if not live:
                break
            b.advance(trials)
            seconds += b.last_advance_seconds
            b.check()
            for s in list(live):
                st = b.status(s)
                if history and st['checks'] > len(hist[s]):
                    hist[s].append({k: st[k] for k in ('time', 'steps', 'residual', 'cl', 'cd', 'cm', 'hold')})
                if st['finished']:
                    live.discard(s)
        out = []
        for s in slots:
            r = b.status(s)
            if download:
                r['u'] = b.download(s)
            if history:
                r['history'] = hist[s]
            out.append(r)
        return out, seconds
    finally:
        b.destroy()


def primitive(u, nv, gamma=1.4):
    """(rho, u, v, p) per cell from the SoA conserved state."""
    q = u.reshape(nv, -1)
    rho = q[0]
    vx, vy = q[1] / rho, q[2] / rho
    p = (gamma - 1) * (q[3] - 0.5 * rho * (vx * vx + vy * vy))
    return np.stack([rho, vx, vy, p])


def field_errors(u, ref, nv, gamma=1.4):
    """Per-cell error of rho, u, v, p (and the SA variable) of state u against state ref: the largest
    absolute difference, the same over the largest |ref| of that field (max-normalised), and the RMS
    difference over the RMS of ref."""
    a, b = primitive(u, nv, gamma), primitive(ref, nv, gamma)
    names = ['rho', 'u', 'v', 'p']
    if nv == 5:
        a = np.vstack([a, u.reshape(nv, -1)[4:5]])
        b = np.vstack([b, ref.reshape(nv, -1)[4:5]])
        names.append('rho_nutilde')
    out = {}
    for i, name in enumerate(names):
        d = a[i] - b[i]
        scale = max(np.abs(b[i]).max(), 1e-300)
        rms_ref = max(float(np.sqrt(np.mean(b[i] * b[i]))), 1e-300)
        out[name] = dict(max_abs=float(np.abs(d).max()), max_rel=float(np.abs(d).max() / scale),
                         rms_rel=float(np.sqrt(np.mean(d * d)) / rms_ref))
    return out


def load_errors(r, ref):
    """|dCL|, |dCD|, |dCM| between two status records."""
    return dict(cl=abs(r['cl'] - ref['cl']), cd=abs(r['cd'] - ref['cd']), cm=abs(r['cm'] - ref['cm']))


def loads_of_state(spec, mesh, u, precision=64):
    """CL, CD, CM of a given state, evaluated on the device in FP64 (one FP64 single-case session of
    the state, whose diagnostics are the driver's force and moment sums)."""
    from .session import StaticAmrGpu
    s = StaticAmrGpu.create(mesh, spec.params(), u)
    try:
        d = s.diagnostics(cases.STEADY['region'], (cases.STEADY['moment_x'], cases.STEADY['moment_y']))
    finally:
        s.destroy()
    a = spec.aoa * np.pi / 180
    q = 0.5 * spec.mach * spec.mach
    fx, fy, mz = d[5], d[6], d[7]
    return dict(cl=(-fx * np.sin(a) + fy * np.cos(a)) / q, cd=(fx * np.cos(a) + fy * np.sin(a)) / q, cm=mz / q)


STATUS_NAMES = {0: 'ok', _abi.STATUS_MAXSTEPS: 'maxsteps'}
