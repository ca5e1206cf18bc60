"""GPU parity of every launch mode: the persistent cooperative kernel, one kernel per phase, and
the split mode (gradients per cell, each face flux once per face record, in-order gather per
cell).  All three evaluate the same arithmetic in the same order, so in FP64 they agree bit for
bit with each other and stay within 1e-10 (per variable, max-normalised) of the oracle.  In FP32
the modes may round a face flux differently (a fused-slot mode evaluates each face from both of
its cells), so there they agree within 1e-5 of each other, and each is still bit-identical alone
and in a mix of cases."""
import numpy as np
import pytest

from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import _abi, airfoils, cases
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.batch import Batch, case_control
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.mesh import MeshArrays
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.session import StaticAmrGpu, default_options
from oracle.oracle import Oracle, RefCase

pytestmark = pytest.mark.gpu
TOL = 1e-10
MODES = {
    'persistent': dict(launch_mode=_abi.LAUNCH_PERSISTENT, block_threads=256),
    'phases': dict(launch_mode=_abi.LAUNCH_PHASES, block_threads=128),
    'split': dict(launch_mode=_abi.LAUNCH_SPLIT, block_threads=128),
    'tiled': dict(launch_mode=_abi.LAUNCH_TILED, block_threads=128),
}


def rel_err(a, b, nv):
    a = a.reshape(nv, -1)
    b = b.reshape(nv, -1)
    return max(np.abs(a[v] - b[v]).max() / max(np.abs(b[v]).max(), 1e-300) for v in range(nv))


def built(naca, **kw):
    x, y, pt = airfoils.naca4(*naca)
    spec = cases.CaseSpec(naca=naca, **kw)
    return spec, RefCase.build(spec, x, y, pt).mesh()


def session_cases(golden):
    out = [('euler_srd', cases.CaseSpec(physics='euler', profile='LF1', mach=1.65, aoa=1.5),
            MeshArrays.load(golden / 'mesh_naca0012_lf1_euler_srd.npz'), 30),
           ('sa_lf1', cases.CaseSpec(physics='sa', profile='LF1', mach=1.65, aoa=1.5),
            MeshArrays.load(golden / 'mesh_naca2412_lf1_sa.npz'), 20)]
    spec, mesh = built((0.04, 0.3, 0.1), profile='LF1', physics='laminar', law='sutherland', flux='ausm',
                       kinds=('farfield', 'pressure-outlet', 'reflect', 'reflect'), mach=1.4, aoa=2.0)
    out.append(('laminar_ausm', spec, mesh, 15))
    spec, mesh = built((0.0, 0.4, 0.09), profile='LF1', physics='euler', flux='ausm', agglomerate=True, mach=1.8)
    out.append(('euler_agglomerated', spec, mesh, 20))
    return out


def test_session_modes_bit_exact(golden):
    for name, spec, mesh, nsteps in session_cases(golden):
        params = spec.params()
        u0 = cases.initial_state(mesh, spec.initial_primitive())
        ref = Oracle(mesh, params).run(u0, 1e30, nsteps)
        outs = {}
        for mode, opts in MODES.items():
            s = StaticAmrGpu.create(mesh, params, u0, options=default_options(**opts))
            assert s.advance(1e30, nsteps) == 1 and 'status 3' in s.last_error, (name, mode, s.last_error)
            assert (s.steps, s.rejected, s.time) == (ref['steps'], ref['rejected'], ref['time']), (name, mode)
            outs[mode] = s.download()
            err = rel_err(outs[mode], ref['u'], mesh.nv)
            assert err <= TOL, (name, mode, err)
        for mode in MODES:
            assert np.array_equal(outs[mode], outs['split']), (name, mode)


def test_session_residual_all_modes(golden):
    mesh = MeshArrays.load(golden / 'mesh_naca2412_lf1_sa.npz')
    spec = cases.CaseSpec(physics='sa', profile='LF1', mach=1.65, aoa=1.5)
    u0 = cases.initial_state(mesh, spec.initial_primitive())
    res = []
    for mode, opts in MODES.items():
        s = StaticAmrGpu.create(mesh, spec.params(), u0, options=default_options(**opts))
        s.advance(1e30, 3)
        res.append(s.residual())
    for r in res[1:]:
        assert np.array_equal(res[0], r)


def sa_mix():
    out = []
    for naca, profile, mach, aoa in [((0.02, 0.4, 0.12), 'LF1', 1.65, 1.5), ((0.0, 0.4, 0.14), 'LF2', 1.9, 4.0),
                                     ((0.05, 0.3, 0.09), 'LF1', 1.3, -2.0)]:
        out.append(built(naca, profile=profile, physics='sa', mach=mach, aoa=aoa))
    return out


def run_batch(cases_list, precision, nsteps, mode, order=None):
    b = Batch(precision=precision, model=_abi.MODEL_LAMINAR, sa=True, max_cases=8,
              max_cells=sum(m.n_cells for _, m in cases_list) + 1000, **MODES[mode])
    slots = {}
    for i in (order or range(len(cases_list))):
        spec, mesh = cases_list[i]
        u0 = cases.initial_state(mesh, spec.initial_primitive())
        slots[i] = b.admit(mesh, spec.params(), u0, case_control(1e30, nsteps, steady=False, mach=spec.mach, aoa=spec.aoa))
        assert slots[i] is not None
    for _ in range(64):
        b.advance(32)
        if all(b.status(s)['status'] for s in slots.values()):
            break
    out = {}
    for i, s in slots.items():
        st = b.status(s)
        assert st['status'] == _abi.STATUS_MAXSTEPS and st['steps'] == nsteps, (mode, st)
        out[i] = b.download(s)
    assert mode in b.launch_config()
    return out


@pytest.mark.parametrize('mode', ['split', 'tiled'])
def test_batch_fp64_matches_persistent(mode):
    mix = sa_mix()
    a = run_batch(mix, 64, 20, 'persistent')
    b = run_batch(mix, 64, 20, mode, order=[2, 0, 1])
    for i in a:
        assert np.array_equal(a[i], b[i]), i


@pytest.mark.parametrize('mode', ['split', 'tiled'])
def test_batch_fp32_alone_and_in_mix_and_close_to_fused(mode):
    mix = sa_mix()
    got = run_batch(mix, 32, 40, mode, order=[1, 2, 0])
    fused = run_batch(mix, 32, 40, 'phases')
    for i in range(len(mix)):
        alone = run_batch([mix[i]], 32, 40, mode)
        assert np.array_equal(got[i], alone[0]), i
        assert rel_err(got[i], fused[i], 5) <= 1e-5, (i, rel_err(got[i], fused[i], 5))


@pytest.mark.parametrize('mode', ['split', 'tiled'])
def test_release_and_readmit_reuses_ranges(mode):
    """A released case's records and block tiles are dead; a new case admitted into the freed
    ranges computes exactly what it computes in a fresh batch."""
    mix = sa_mix()
    b = Batch(precision=64, model=_abi.MODEL_LAMINAR, sa=True, max_cases=4,
              max_cells=sum(m.n_cells for _, m in mix) + 1000, **MODES[mode])
    specs = []
    for spec, mesh in mix[:2]:
        u0 = cases.initial_state(mesh, spec.initial_primitive())
        specs.append(b.admit(mesh, spec.params(), u0, case_control(1e30, 10, steady=False, mach=spec.mach, aoa=spec.aoa)))
    b.advance(16)
    b.release(specs[0])
    spec, mesh = mix[2]
    u0 = cases.initial_state(mesh, spec.initial_primitive())
    s = b.admit(mesh, spec.params(), u0, case_control(1e30, 10, steady=False, mach=spec.mach, aoa=spec.aoa))
    for _ in range(4):
        b.advance(16)
    assert b.status(s)['status'] == _abi.STATUS_MAXSTEPS
    fresh = run_batch([mix[2]], 64, 10, mode)
    assert np.array_equal(b.download(s), fresh[0])



def test_fp32_laminar_split_close_to_phases_and_oracle():
    """FP32 laminar model (AUSM+-up, Sutherland, outlet and reflecting sides, viscous wall model):
    the split mode's compact records (net flux) stay within 1e-5 of the phase mode and within the
    FP32 tolerance of the FP64 oracle."""
    spec, mesh = built((0.04, 0.3, 0.1), profile='LF1', physics='laminar', law='sutherland', flux='ausm',
                       kinds=('farfield', 'pressure-outlet', 'reflect', 'reflect'), mach=1.4, aoa=2.0)
    params = spec.params()
    u0 = cases.initial_state(mesh, spec.initial_primitive())
    nsteps = 30
    out = {}
    for mode in ('split', 'phases'):
        b = Batch(precision=32, model=_abi.MODEL_LAMINAR, sa=False, flux=_abi.FLUX_AUSMPUP, max_cases=2,
                  max_cells=mesh.n_cells + 100, **MODES[mode])
        s = b.admit(mesh, params, u0, case_control(1e30, nsteps, steady=False, mach=spec.mach, aoa=spec.aoa))
        for _ in range(4):
            b.advance(16)
        st = b.status(s)
        assert st['status'] == _abi.STATUS_MAXSTEPS and st['steps'] == nsteps, (mode, st)
        assert mode in b.launch_config()
        out[mode] = b.download(s)
        b.destroy()
    ref = Oracle(mesh, params).run(u0, 1e30, nsteps)
    assert rel_err(out['split'], out['phases'], 4) <= 1e-5
    assert rel_err(out['split'], ref['u'], 4) <= 2e-4


def test_fp32_euler_srd_split_alone_in_mix_and_close_to_phases_and_oracle(golden):
    """FP32 Euler with non-trivial SRD neighbourhoods: the split mode is bit-identical alone and
    beside another case, within 1e-5 of the phase mode and within the FP32 tolerance of the FP64
    oracle."""
    spec = cases.CaseSpec(physics='euler', profile='LF1', mach=1.65, aoa=1.5)
    mesh = MeshArrays.load(golden / 'mesh_naca0012_lf1_euler_srd.npz')
    other = built((0.02, 0.4, 0.12), profile='LF1', physics='euler', mach=1.8, aoa=3.0)
    params = spec.params()
    nsteps = 40

    def run(mode, with_other):
        items = [(spec, mesh)] + ([other] if with_other else [])
        b = Batch(precision=32, model=_abi.MODEL_EULER, sa=False, max_cases=2,
                  max_cells=sum(m.n_cells for _, m in items) + 100, **MODES[mode])
        slots = [b.admit(m, s.params(), cases.initial_state(m, s.initial_primitive()),
                         case_control(1e30, nsteps, steady=False, mach=s.mach, aoa=s.aoa)) for s, m in items]
        for _ in range(4):
            b.advance(16)
        st = b.status(slots[0])
        assert st['status'] == _abi.STATUS_MAXSTEPS and st['steps'] == nsteps, (mode, st)
        u = b.download(slots[0])
        b.destroy()
        return u

    alone = run('split', False)
    assert np.array_equal(alone, run('split', True))
    ref = Oracle(mesh, params).run(cases.initial_state(mesh, spec.initial_primitive()), 1e30, nsteps)
    assert rel_err(alone, run('phases', False), 4) <= 1e-5
    assert rel_err(alone, ref['u'], 4) <= 2e-4


def test_split_first_update_in_place_rejections_and_fatal_match_oracle(golden):
    """Split mode, SA without SRD (the stage-1 kernels form U1 = U + dt R0 in place): an oversize
    fixed dt is halved and retried exactly as on the CPU; 21 rejections end with status 5 and a
    dt underflow with status 4, the accepted state kept."""
    mesh = MeshArrays.load(golden / 'mesh_naca2412_lf1_sa.npz')
    assert not mesh.small_cells
    opts = default_options(**MODES['split'])
    spec = cases.CaseSpec(physics='sa', profile='LF1', mach=1.65, aoa=1.5, dt_fixed=0.02)
    u0 = cases.initial_state(mesh, spec.initial_primitive())
    ref = Oracle(mesh, spec.params()).run(u0, 1e30, 6)
    s = StaticAmrGpu.create(mesh, spec.params(), u0, options=opts)
    assert s.advance(1e30, 6) == 1 and 'status 3' in s.last_error
    assert 'split' in s.launch_config()
    assert (s.steps, s.rejected, s.time) == (ref['steps'], ref['rejected'], ref['time']) and ref['rejected'] > 0
    assert rel_err(s.download(), ref['u'], mesh.nv) <= TOL
    spec5 = cases.CaseSpec(physics='sa', profile='LF1', mach=1.65, aoa=1.5, dt_fixed=1e10)
    ref5 = Oracle(mesh, spec5.params()).run(u0, 1e12, 5)
    assert 'after 21 trials' in ref5['error']
    s = StaticAmrGpu.create(mesh, spec5.params(), u0, options=opts)
    assert s.advance(1e12, 5) == 1 and 'status 5' in s.last_error
    assert s.rejected == ref5['rejected'] == 21 and np.array_equal(s.download(), u0)
    spec4 = cases.CaseSpec(physics='sa', profile='LF1', mach=1.65, aoa=1.5, dt_fixed=1e-300)
    s = StaticAmrGpu.create(mesh, spec4.params(), u0, time=1.0, options=opts)
    assert s.advance(2.0, 5) == 1 and 'status 4' in s.last_error
    assert np.array_equal(s.download(), u0)
