"""CPU tests: the C oracle against the reference CPU core and the reference's known answers."""
import json

import numpy as np
import pytest

from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import airfoils, cases
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.mesh import MeshArrays
from oracle.oracle import Oracle, RefCase
from tests.golden.make_golden import SettingsSpec, parse_settings  # noqa: E402


def known(golden):
    return json.loads((golden / 'known_answers.json').read_text())


def example(golden, name):
    z = np.load(golden / 'examples.npz')
    names = list(z['names'])
    i = names.index(name)
    a, b = z['offsets'][i], z['offsets'][i + 1]
    return z['x'][a:b], z['y'][a:b], z['patches'][a:b]


def test_nondimensional_settings_match_reference_pipeline(golden):
    s, _ = parse_settings(known(golden)['settings']['default_LF1'])
    nd = cases.nondimensional()
    assert float(s['mu_star']) == nd['mu_star']
    assert float(s['sutherland_star']) == nd['sutherland_star']
    assert float(s['sa_nu_inf']) == nd['sa_nu_inf']
    assert float(s['outlet_p_star']) == nd['outlet_p_star']


@pytest.mark.parametrize('physics,profile,flux,steps', [('euler', 'LF1', 'hllc', 12), ('sa', 'LF1', 'hllc', 6),
                                                        ('laminar', 'LF1', 'ausm', 6)])
def test_oracle_bitexact_against_reference(physics, profile, flux, steps):
    x, y, pt = airfoils.naca4(0.02, 0.4, 0.12)
    kinds = ('farfield', 'pressure-outlet', 'farfield', 'farfield') if physics == 'laminar' else ('farfield',) * 4
    spec = cases.CaseSpec(naca=(0.02, .4, .12), profile=profile, physics=physics, flux=flux, kinds=kinds,
                          law='constant' if physics == 'laminar' else 'sutherland')
    rc = RefCase.build(spec, x, y, pt)
    m = rc.mesh()
    u0 = cases.initial_state(m, spec.initial_primitive())
    assert np.array_equal(u0, rc.initial(spec.initial_primitive()))
    ref = rc.run_steps(u0, steps)
    o = Oracle(m, spec.params()).run_steps(u0, steps)
    assert o['steps'] == ref['steps'] == steps and o['time'] == ref['time']
    assert np.array_equal(o['u'], ref['u'])
    assert np.array_equal(Oracle(m, spec.params()).rhs(ref['u']), rc.rhs(ref['u']))
    assert np.array_equal(Oracle(m, spec.params()).diagnostics(ref['u']), rc.diagnostics(ref['u']))


def test_oracle_srd_redistribute_matches_reference(golden):
    m = MeshArrays.load(golden / 'mesh_naca0012_lf1_euler_srd.npz')
    spec = cases.CaseSpec(physics='euler', profile='LF1')
    rc = RefCase.from_mesh(m, spec.params())
    rng = np.random.default_rng(7)
    u = cases.initial_state(m, spec.initial_primitive()) * (1 + 0.01 * rng.standard_normal(4 * m.n_cells))
    assert np.array_equal(Oracle(m, spec.params()).redistribute(u), rc.redistribute(u))


@pytest.mark.parametrize('profile', ['LF1', 'LF2'])
def test_short_known_answer_g0001(golden, profile):
    """validation/ten_short_checks.json: cells and steps to t*=0.01 for G0001."""
    ka = known(golden)
    s, boxes = parse_settings(ka['settings']['default_' + profile])
    spec = SettingsSpec(s, boxes, profile)
    x, y, pt = example(golden, 'G0001')
    rc = RefCase.build(spec, x, y, pt)
    m = rc.mesh()
    expect = [c for c in ka['short_checks'] if c['case'] == 'G0001' and c['profile'] == profile][0]
    assert m.n_cells == expect['cells']
    u0 = cases.initial_state(m, spec.initial_primitive())
    out = Oracle(m, spec.params()).run(u0, 0.01, 50000000)
    assert out['status'] == 0 and out['time'] == 0.01 and out['rejected'] == 0
    assert out['steps'] == expect['steps']
    ref = ka['reproduced']['G0001_' + profile]
    assert out['steps'] == ref['steps']
    d = Oracle(m, spec.params()).diagnostics(out['u'])
    assert np.array_equal(d, np.array(ref['diagnostics']))


def test_control_subsonic_outlet_known_steps(golden):
    """validation/controls_checks.json: subsonic pressure outlet, LF2, 65 steps to t*=0.01."""
    ka = known(golden)
    s, boxes = parse_settings(ka['settings']['control_subsonic_outlet'])
    spec = SettingsSpec(s, boxes, 'LF2')
    x, y, pt = example(golden, 'G0001')
    rc = RefCase.build(spec, x, y, pt)
    m = rc.mesh()
    u0 = cases.initial_state(m, spec.initial_primitive())
    out = Oracle(m, spec.params()).run(u0, 0.01, 50000000)
    assert out['status'] == 0 and out['steps'] == ka['controls']['subsonic_outlet']


def test_oracle_rejection_and_fatal_paths(golden):
    """Oversize fixed dt: rejections with dt halving, same counters as the reference."""
    m = MeshArrays.load(golden / 'mesh_naca0012_lf1_euler_srd.npz')
    spec = cases.CaseSpec(physics='euler', profile='LF1', dt_fixed=0.02)
    rc = RefCase.from_mesh(m, spec.params())
    u0 = cases.initial_state(m, spec.initial_primitive())
    ref = rc.run(u0, 0.05, 10)
    o = Oracle(m, spec.params()).run(u0, 0.05, 10)
    assert (o['status'], o['steps'], o['rejected'], o['time']) == (ref['status'], ref['steps'], ref['rejected'], ref['time'])
    assert o['error'] == ref['error']
    assert np.array_equal(o['u'], ref['u'])


def total_inlet_spec():
    """Subsonic channel-like case: total-pressure inlet on xmin (direction +x), static-pressure
    outlet on xmax, farfield top and bottom; NACA 0012, LF1, agglomerated, inviscid."""
    spec = cases.CaseSpec(naca=(0.0, 0.4, 0.12), profile='LF1', physics='euler', mach=0.5, aoa=0.0, agglomerate=True,
                          kinds=('total-inlet', 'pressure-outlet', 'farfield', 'farfield'))
    base = spec.boundary_records
    gamma, mach = 1.4, 0.5

    def records(g=1.4):
        b = base(g)
        w = cases.freestream(mach, 0.0, gamma)
        t_static = w[3] / w[0]  # R = 1
        b[0]['total_temperature'] = t_static * (1 + 0.5 * (gamma - 1) * mach * mach)
        b[0]['total_pressure'] = w[3] * (1 + 0.5 * (gamma - 1) * mach * mach) ** (gamma / (gamma - 1))
        b[0]['gas_constant'] = 1.0
        b[0]['direction'] = (1.0, 0.0)
        return b
    spec.boundary_records = records
    return spec


def test_oracle_total_inlet_bitexact_against_reference():
    spec = total_inlet_spec()
    x, y, pt = airfoils.naca4(0.0, 0.4, 0.12)
    rc = RefCase.build(spec, x, y, pt)
    m = rc.mesh()
    u0 = cases.initial_state(m, spec.initial_primitive())
    ref = rc.run_steps(u0, 15)
    o = Oracle(m, spec.params()).run_steps(u0, 15)
    assert o['steps'] == ref['steps'] == 15 and o['time'] == ref['time']
    assert np.array_equal(o['u'], ref['u'])


def test_oracle_srd_rate_viscous_bitexact_against_reference():
    """Laminar on an SRD (non-agglomerated) mesh with SRD-rate viscous stabilization."""
    spec = cases.CaseSpec(naca=(0.02, 0.4, 0.12), profile='LF1', physics='laminar', agglomerate=False, mach=1.4,
                          kinds=('farfield', 'pressure-outlet', 'farfield', 'farfield'))
    base = spec.transport_record
    spec.transport_record = lambda g=1.4: _with_stabilization(base(g))
    x, y, pt = airfoils.naca4(0.02, 0.4, 0.12)
    rc = RefCase.build(spec, x, y, pt)
    m = rc.mesh()
    assert m.small_cells > 0
    u0 = cases.initial_state(m, spec.initial_primitive())
    ref = rc.run_steps(u0, 10)
    o = Oracle(m, spec.params()).run_steps(u0, 10)
    assert o['steps'] == ref['steps'] == 10 and o['time'] == ref['time']
    assert np.array_equal(o['u'], ref['u'])


def _with_stabilization(t):
    from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import _abi
    t['stabilization'] = _abi.VISCOUS_SRD
    return t
