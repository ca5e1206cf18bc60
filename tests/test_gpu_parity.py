"""GPU parity of the plain FP64 session against the oracle (C restatement, pinned bit-exact to the
reference CPU core).  Tolerance: per variable, max_k |u_gpu - u_oracle| <= 1e-10 * max_k |u_oracle|
after N steps, with identical step/rejection counters and times."""
import json

import numpy as np
import pytest

from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import _abi, airfoils, cases
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.mesh import MeshArrays
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.session import StaticAmrGpu, default_options
from oracle.oracle import Oracle, RefCase
from tests.golden.make_golden import SettingsSpec, parse_settings

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel_err(a, b, nv):
    a = a.reshape(nv, -1)
    b = b.reshape(nv, -1)
    return max(np.abs(a[v] - b[v]).max() / max(np.abs(b[v]).max(), 1e-300) for v in range(nv))


def run_pair(mesh, spec, checkpoints, options=None):
    """Advance to each cumulative step count; the maxsteps status is sticky in a session (as in
    the reference), so each checkpoint continues in a new session created from the downloaded
    state and counters."""
    params = spec.params()
    u0 = cases.initial_state(mesh, spec.initial_primitive())
    orc = Oracle(mesh, params)
    u_ref, st_ref = u0, dict(steps=0, time=0.0, rejected=0)
    u_gpu, t_gpu, n_gpu, r_gpu = u0, 0.0, 0, 0
    errs = []
    s = None
    for n in checkpoints:
        out = orc.run(u_ref, 1e30, n, time=st_ref['time'], steps=st_ref['steps'], rejected=st_ref['rejected'])
        assert out['error'] == 'maxsteps reached before tend'
        u_ref, st_ref = out['u'], out
        s = StaticAmrGpu.create(mesh, params, u_gpu, time=t_gpu, steps=n_gpu, rejected=r_gpu, options=options)
        status = s.advance(1e30, n)
        assert status == 1 and 'status 3' in s.last_error, s.last_error
        assert s.advance(1e30, n + 5) == 1 and s.steps == n  # status 3 is sticky
        u_gpu, t_gpu, n_gpu, r_gpu = s.download(), s.time, s.steps, s.rejected
        assert (n_gpu, r_gpu) == (out['steps'], out['rejected'])
        assert t_gpu == out['time']
        errs.append(rel_err(u_gpu, u_ref, mesh.nv))
        assert errs[-1] <= TOL, (n, errs)
    return s, u_ref, errs


def test_euler_srd_lf1_1_10_200_steps(golden):
    """Plain FP64 inviscid Euler + SRD, NACA 0012 LF1, HLLC, CFL 0.15, farfield (the CPU workload)."""
    mesh = MeshArrays.load(golden / 'mesh_naca0012_lf1_euler_srd.npz')
    spec = cases.CaseSpec(physics='euler', profile='LF1', mach=1.65, aoa=1.5)
    s, u_ref, errs = run_pair(mesh, spec, [1, 10, 200])
    print('euler srd rel errors', errs)


def test_sa_lf1_parity(golden):
    mesh = MeshArrays.load(golden / 'mesh_naca2412_lf1_sa.npz')
    spec = cases.CaseSpec(physics='sa', profile='LF1', mach=1.65, aoa=1.5)
    s, u_ref, errs = run_pair(mesh, spec, [1, 10, 60])
    print('sa lf1 rel errors', errs)


def test_sa_lf2_parity(golden):
    mesh = MeshArrays.load(golden / 'mesh_naca2412_lf2_sa.npz')
    spec = cases.CaseSpec(physics='sa', profile='LF2', mach=1.65, aoa=1.5)
    run_pair(mesh, spec, [1, 20])


@pytest.mark.parametrize('law,flux,kinds', [
    ('constant', 'ausm', ('farfield', 'pressure-outlet', 'farfield', 'farfield')),
    ('sutherland', 'hllc', ('farfield', 'transmissive', 'reflect', 'reflect')),
])
def test_laminar_variants(law, flux, kinds):
    x, y, pt = airfoils.naca4(0.04, 0.3, 0.1)
    spec = cases.CaseSpec(naca=(0.04, .3, .1), profile='LF1', physics='laminar', law=law, flux=flux, kinds=kinds, mach=1.4,
                          aoa=2.0)
    mesh = RefCase.build(spec, x, y, pt).mesh()
    run_pair(mesh, spec, [1, 15])


def test_euler_ausm_agglomerated():
    x, y, pt = airfoils.naca4(0.0, 0.4, 0.09)
    spec = cases.CaseSpec(naca=(0.0, .4, .09), profile='LF1', physics='euler', flux='ausm', agglomerate=True, mach=1.8)
    mesh = RefCase.build(spec, x, y, pt).mesh()
    run_pair(mesh, spec, [1, 25])


def test_rejections_match_oracle(golden):
    """Oversize fixed dt: the device halves dt and retries exactly as the CPU does."""
    mesh = MeshArrays.load(golden / 'mesh_naca0012_lf1_euler_srd.npz')
    spec = cases.CaseSpec(physics='euler', profile='LF1', dt_fixed=0.02)
    params = spec.params()
    u0 = cases.initial_state(mesh, spec.initial_primitive())
    ref = Oracle(mesh, params).run(u0, 0.05, 10)
    s = StaticAmrGpu.create(mesh, params, u0)
    st = s.advance(0.05, 10)
    assert (st != 0) == (ref['status'] != 0)
    assert (s.steps, s.rejected, s.time) == (ref['steps'], ref['rejected'], ref['time'])
    assert ref['rejected'] > 0
    assert rel_err(s.download(), ref['u'], 4) <= TOL


def test_fatal_statuses(golden):
    mesh = MeshArrays.load(golden / 'mesh_naca0012_lf1_euler_srd.npz')
    spec = cases.CaseSpec(physics='euler', profile='LF1')
    u0 = cases.initial_state(mesh, spec.initial_primitive())
    # nonphysical base state -> status 2, state retained
    bad = u0.copy()
    bad[3 * mesh.n_cells + 17] = -1.0
    s = StaticAmrGpu.create(mesh, spec.params(), bad)
    assert s.advance(1.0, 5) == 1 and 'status 2' in s.last_error
    assert np.array_equal(s.download(), bad)
    # dt underflow (time + dt == time) -> status 4
    spec4 = cases.CaseSpec(physics='euler', profile='LF1', dt_fixed=1e-300)
    ref4 = Oracle(mesh, spec4.params()).run(u0, 2.0, 5, time=1.0)
    assert ref4['error'] == 'physical time step underflow'
    s = StaticAmrGpu.create(mesh, spec4.params(), u0, time=1.0)
    assert s.advance(2.0, 5) == 1 and 'status 4' in s.last_error
    # 21 rejections -> status 5
    spec5 = cases.CaseSpec(physics='euler', profile='LF1', dt_fixed=1e10)
    ref = Oracle(mesh, spec5.params()).run(u0, 1e12, 5)
    assert 'after 21 trials' in ref['error']
    s = StaticAmrGpu.create(mesh, spec5.params(), u0)
    assert s.advance(1e12, 5) == 1 and 'status 5' in s.last_error
    assert s.rejected == ref['rejected'] == 21
    assert np.array_equal(s.download(), u0)
    # invalid advance arguments
    s = StaticAmrGpu.create(mesh, spec.params(), u0)
    assert s.advance(-1.0, 5) == 1 and 'invalid' in s.last_error
    assert s.advance(1.0, 0) == 1


def test_exact_tend_and_resume(golden):
    """advance stops exactly at tend (dt clipping) and resumes across calls like one call."""
    mesh = MeshArrays.load(golden / 'mesh_naca0012_lf1_euler_srd.npz')
    spec = cases.CaseSpec(physics='euler', profile='LF1')
    u0 = cases.initial_state(mesh, spec.initial_primitive())
    ref = Oracle(mesh, spec.params()).run(u0, 0.003, 10 ** 6)
    s = StaticAmrGpu.create(mesh, spec.params(), u0)
    assert s.advance(0.001, 10 ** 6) == 0 and s.time == 0.001
    assert s.advance(0.003, 10 ** 6) == 0 and s.time == 0.003
    ref1 = Oracle(mesh, spec.params()).run(u0, 0.001, 10 ** 6)
    ref2 = Oracle(mesh, spec.params()).run(ref1['u'], 0.003, 10 ** 6, time=0.001, steps=ref1['steps'])
    assert s.steps == ref2['steps']
    assert rel_err(s.download(), ref2['u'], 4) <= TOL
    assert ref['time'] == 0.003


def test_residual_and_diagnostics_on_device(golden):
    mesh = MeshArrays.load(golden / 'mesh_naca2412_lf1_sa.npz')
    spec = cases.CaseSpec(physics='sa', profile='LF1')
    params = spec.params()
    u0 = cases.initial_state(mesh, spec.initial_primitive())
    orc = Oracle(mesh, params)
    ref = orc.run_steps(u0, 30)
    s = StaticAmrGpu.create(mesh, params, u0)
    s.advance(1e30, 30)
    r = s.residual()
    r_ref = orc.rhs(ref['u'])
    assert rel_err(r, r_ref, 5) <= 1e-9
    d = s.diagnostics()
    d_ref = orc.diagnostics(ref['u'])
    np.testing.assert_allclose(d, d_ref, rtol=1e-9, atol=1e-13)


def test_rest_state_preserved(golden):
    """Free-stream-at-rest known answer of the reference driver: L_inf drift <= 2e-11."""
    mesh = MeshArrays.load(golden / 'mesh_naca2412_lf1_sa.npz')
    spec = cases.CaseSpec(physics='sa', profile='LF1', mach=1.65)
    rest = np.array([1.0, 0.0, 0.0, 1 / 1.4])
    u0 = cases.initial_state(mesh, rest)
    b = mesh.boundaries.copy()
    for side in range(4):
        b[side]['reference'] = rest
    m = mesh.with_physics(boundaries=b)
    s = StaticAmrGpu.create(m, spec.params(), u0)
    assert s.advance(0.01, 10 ** 6) == 0
    u = s.download()
    assert np.abs(u[:4 * mesh.n_cells] - u0[:4 * mesh.n_cells]).max() <= 2e-11


@pytest.mark.parametrize('profile', ['LF1', 'LF2'])
def test_short_known_answer_g0001_on_gpu(golden, profile):
    """validation/ten_short_checks.json through the B200 path: cells and steps to t*=0.01."""
    ka = json.loads((golden / 'known_answers.json').read_text())
    s, boxes = parse_settings(ka['settings']['default_' + profile])
    spec = SettingsSpec(s, boxes, profile)
    z = np.load(golden / 'examples.npz')
    i = list(z['names']).index('G0001')
    a, b = z['offsets'][i], z['offsets'][i + 1]
    mesh = RefCase.build(spec, z['x'][a:b], z['y'][a:b], z['patches'][a:b]).mesh()
    expect = [c for c in ka['short_checks'] if c['case'] == 'G0001' and c['profile'] == profile][0]
    u0 = cases.initial_state(mesh, spec.initial_primitive())
    g = StaticAmrGpu.create(mesh, spec.params(), u0)
    assert g.advance(0.01, 50000000) == 0
    assert mesh.n_cells == expect['cells'] and g.steps == expect['steps'] and g.rejected == 0 and g.time == 0.01
    ref = Oracle(mesh, spec.params()).run(u0, 0.01, 50000000)
    assert rel_err(g.download(), ref['u'], 5) <= TOL


def test_graph_and_direct_launch_agree(golden):
    mesh = MeshArrays.load(golden / 'mesh_naca0012_lf1_euler_srd.npz')
    spec = cases.CaseSpec(physics='euler', profile='LF1')
    u0 = cases.initial_state(mesh, spec.initial_primitive())
    outs = []
    for graph, block in ((1, 128), (0, 256), (1, 256)):
        s = StaticAmrGpu.create(mesh, spec.params(), u0, options=default_options(graph=graph, block_threads=block))
        s.advance(1e30, 40)
        outs.append(s.download())
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[1], outs[2])


def test_total_inlet_parity():
    """Total-pressure inlet (the 64-step bisection of the inflow state) with a pressure outlet."""
    from tests.test_oracle import total_inlet_spec
    spec = total_inlet_spec()
    x, y, pt = airfoils.naca4(0.0, 0.4, 0.12)
    mesh = RefCase.build(spec, x, y, pt).mesh()
    run_pair(mesh, spec, [1, 20])


@pytest.mark.parametrize('control', ['fixed_dt', 'cpu_ausm', 'subsonic_outlet'])
def test_control_known_steps_on_gpu(golden, control):
    """validation/controls_checks.json through the B200 path: steps to t*=0.01 on G0001 LF2."""
    ka = json.loads((golden / 'known_answers.json').read_text())
    s, boxes = parse_settings(ka['settings']['control_' + control])
    spec = SettingsSpec(s, boxes, 'LF2')
    z = np.load(golden / 'examples.npz')
    i = list(z['names']).index('G0001')
    a, b = z['offsets'][i], z['offsets'][i + 1]
    mesh = RefCase.build(spec, z['x'][a:b], z['y'][a:b], z['patches'][a:b]).mesh()
    u0 = cases.initial_state(mesh, spec.initial_primitive())
    g = StaticAmrGpu.create(mesh, spec.params(), u0)
    assert g.advance(0.01, 50000000) == 0
    assert g.steps == ka['controls'][control] and g.rejected == 0 and g.time == 0.01


def srd_rate_spec():
    from tests.test_oracle import _with_stabilization
    spec = cases.CaseSpec(naca=(0.02, 0.4, 0.12), profile='LF1', physics='laminar', agglomerate=False, mach=1.4,
                          kinds=('farfield', 'pressure-outlet', 'farfield', 'farfield'))
    base = spec.transport_record
    spec.transport_record = lambda g=1.4: _with_stabilization(base(g))
    return spec


@pytest.mark.parametrize('mode', ['persistent', 'phases', 'split'])
def test_srd_rate_viscous_parity(mode):
    """Laminar on an SRD mesh with the viscous dt limited through the SRD map of the rates."""
    from tests.test_gpu_launch_modes import MODES
    spec = srd_rate_spec()
    x, y, pt = airfoils.naca4(0.02, 0.4, 0.12)
    mesh = RefCase.build(spec, x, y, pt).mesh()
    assert mesh.small_cells > 0
    run_pair(mesh, spec, [1, 12], options=default_options(**MODES[mode]))
