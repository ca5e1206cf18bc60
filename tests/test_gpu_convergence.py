"""Accuracy of the FP32 form where the headline metric is quoted: at convergence.

1. The plain FP64 session, driven by the reference's own driver (src/quick_airfoil.cpp linked against
   this engine), solves G0001 on LF1 and LF2 to the steady criteria; its step count, final time and
   loads are compared with the reference's published full-steady solve (validation/summary.json:36-71,
   FP64 on the reference CUDA kernels).  Those kernels round some expressions differently (energy
   and AUSM+-up operand order), so the loads are compared at a roundoff tolerance of 1e-11 (observed
   differences are ~4e-14); the accepted-step counts and final times must be equal.
2. The batched FP32 form solves the same two cases to the steady criteria beside the FP64 batch
   (bit-for-bit the plain FP64 session, tests/test_gpu_batch.py): it must converge, and
   |dCL|, |dCD| <= 1e-4 at retirement.  (With a one-word FP32 state it never converges: increments
   below half an ulp of the state are rounded away and the residual stalls above the tolerance.)
3. NACA 2412 on LF2 (SA), to the steady criteria or 20000 steps, FP64 and FP32: loads and fields.
4. Time-accurate laminar AUSM+-up with a pressure outlet to t*=1 on seeded LF2 cases, FP32 against
   FP64: per-cell errors of rho, u, v, p, each max-normalised, <= 1e-3 (observed <= 4e-4 over the
   full 128-case workload).
"""
import json

import numpy as np
import pytest

from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import runs, workloads
from oracle.oracle import RefCase
from tests.golden.make_golden import SettingsSpec, parse_settings
from tests.test_gpu_dropin import BIN, run as run_driver

pytestmark = pytest.mark.gpu

LOAD_TOL = 1e-4          # |dCL|, |dCD| of the FP32 form against FP64 (the headline metric's bound)
PUBLISHED_LOAD_TOL = 1e-11  # |d load| of this FP64 engine against the reference's published FP64 solve


def g0001(golden, profile):
    ka = json.loads((golden / 'known_answers.json').read_text())
    s, boxes = parse_settings(ka['settings']['default_' + profile])
    spec = SettingsSpec(s, boxes, profile)
    z = np.load(golden / 'examples.npz')
    i = list(z['names']).index('G0001')
    a, b = z['offsets'][i], z['offsets'][i + 1]
    mesh = RefCase.build(spec, z['x'][a:b], z['y'][a:b], z['patches'][a:b]).mesh()
    return spec, mesh, ka['full_steady'][profile]


@pytest.mark.parametrize('profile', ['LF1', 'LF2'])
def test_g0001_full_steady_plain_fp64_matches_published(golden, tmp_path, profile):
    if not BIN.exists():
        pytest.fail(f'{BIN} missing: make -C oracle dropin')
    ka = json.loads((golden / 'known_answers.json').read_text())
    pub = ka['full_steady'][profile]
    r = run_driver(golden, tmp_path, 'steady', 'cuda', profile=profile)
    print(f"G0001 {profile}: steps {r['steps']} (published {pub['steps']}), t {r['physical_time']} "
          f"(published {pub['t']}), Cl {r['Cl']!r} dCl {r['Cl'] - pub['Cl']:.3e}, "
          f"Cd {r['Cd']!r} dCd {r['Cd'] - pub['Cd']:.3e}, Cm {r['Cm']!r} dCm {r['Cm'] - pub['Cm']:.3e}")
    assert r['converged'] and not r['failed'] and r['fluid_control_volumes'] == pub['cells']
    assert r['physical_time'] == pub['t'] and r['steps'] == pub['steps'] and r['rejected'] == 0
    for key in ('Cl', 'Cd', 'Cm'):
        assert abs(r[key] - pub[key]) <= PUBLISHED_LOAD_TOL, (key, r[key], pub[key])


def test_g0001_fp32_steady_loads_against_fp64(golden):
    items = []
    for profile in ('LF1', 'LF2'):
        spec, mesh, _ = g0001(golden, profile)
        items.append((spec, mesh))
    ctl = runs.steady_control(stop_time=100.0)
    r64, _ = runs.solve(items, 64, ctl)
    r32, _ = runs.solve(items, 32, ctl)
    for (spec, mesh), a, b in zip(items, r32, r64):
        e = runs.load_errors(a, b)
        print(f"G0001 {spec.profile}: FP64 steps {b['steps']} t {b['time']} Cl {b['cl']!r} Cd {b['cd']!r} Cm {b['cm']!r}; "
              f"FP32 steps {a['steps']} t {a['time']}; |dCl| {e['cl']:.2e} |dCd| {e['cd']:.2e} |dCm| {e['cm']:.2e}")
        if a['time'] == b['time']:
            f = runs.field_errors(a['u'], b['u'], mesh.nv)
            print('  fields at the common retirement time:', {k: f'{v["max_rel"]:.2e}/{v["rms_rel"]:.2e}' for k, v in f.items()})
        assert a['converged'] and b['converged'], (a, b)
        assert e['cl'] <= LOAD_TOL and e['cd'] <= LOAD_TOL, e


def test_naca2412_lf2_fp32_against_fp64_20k_steps():
    """The single-case accuracy workload: steady criteria or 20000 steps (LF2 needs more than 20000
    steps to reach t >= 3, so both end at the step cap)."""
    w = workloads.naca2412_lf2_sa()
    spec, mesh = w.items[0]
    ctl = runs.steady_control(max_steps=20000)
    (r64,), _ = runs.solve(w.items, 64, ctl)
    (r32,), _ = runs.solve(w.items, 32, ctl)
    e_check = runs.load_errors(r32, r64)
    e_final = runs.load_errors(runs.loads_of_state(spec, mesh, r32['u']), runs.loads_of_state(spec, mesh, r64['u']))
    f = runs.field_errors(r32['u'], r64['u'], mesh.nv)
    print('NACA 2412 LF2 20k:', r64['steps'], r32['steps'], r64['time'], r32['time'], 'last check', e_check, 'final',
          e_final, {k: f'{v["max_rel"]:.2e}/{v["rms_rel"]:.2e}' for k, v in f.items()})
    assert r64['steps'] == r32['steps'] == 20000
    assert max(e_check['cl'], e_check['cd']) <= LOAD_TOL and max(e_final['cl'], e_final['cd']) <= LOAD_TOL


def test_time_accurate_laminar_fp32_against_fp64():
    """A reduced case count of the time-accurate workload (same distribution, 8 LF2 cases)."""
    w = workloads.time_accurate_laminar(8)
    r32, _ = runs.solve(w.items, 32, runs.fixed_time(1.0))
    r64, _ = runs.solve(w.items, 64, runs.fixed_time(1.0))
    worst = 0.0
    for (spec, mesh), a, b in zip(w.items, r32, r64):
        assert a['time'] == b['time'] == 1.0 and a['rejected'] == b['rejected'] == 0
        f = runs.field_errors(a['u'], b['u'], mesh.nv)
        print(f'M {spec.mach:.3f} AoA {spec.aoa:.2f} steps {a["steps"]}/{b["steps"]}:',
              {k: f'{v["max_rel"]:.2e}/{v["rms_rel"]:.2e}' for k, v in f.items()})
        worst = max(worst, max(v['max_rel'] for v in f.values()))
    assert worst <= 1e-3
