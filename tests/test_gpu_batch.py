"""GPU tests of the batched form: ragged multi-mesh arrays, per-case control, admission and
release, the FP32 precision form and the steady retirement checks.

Tolerances: FP64 batch == FP64 single session bit for bit (and within 1e-10 of the oracle);
FP32 batch within 2e-4 of the FP64 oracle per variable (max-normalised) after 100 steps and
|dCL|, |dCD|, |dCM| <= 1e-4; every case bit-identical alone and in the mix."""
import numpy as np
import pytest

from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import _abi, airfoils, cases
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.batch import Batch, case_control
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.mesh import MeshArrays
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.session import StaticAmrGpu
from oracle.oracle import Oracle, RefCase, loads

pytestmark = pytest.mark.gpu


def rel_err(a, b, nv):
    a = a.reshape(nv, -1)
    b = b.reshape(nv, -1)
    return max(np.abs(a[v] - b[v]).max() / max(np.abs(b[v]).max(), 1e-300) for v in range(nv))


def make_cases():
    out = []
    for naca, profile, mach, aoa in [((0.02, 0.4, 0.12), 'LF1', 1.65, 1.5), ((0.05, 0.3, 0.09), 'LF1', 1.3, -2.0),
                                     ((0.0, 0.4, 0.14), 'LF2', 1.9, 4.0)]:
        spec = cases.CaseSpec(naca=naca, profile=profile, physics='sa', mach=mach, aoa=aoa)
        x, y, pt = airfoils.naca4(*naca)
        mesh = RefCase.build(spec, x, y, pt).mesh()
        out.append((spec, mesh))
    return out


@pytest.fixture(scope='module')
def sa_cases():
    return make_cases()


def run_batch(cases_list, precision, nsteps, order=None):
    b = Batch(precision=precision, model=_abi.MODEL_LAMINAR, sa=True, max_cases=8,
              max_cells=sum(m.n_cells for _, m in cases_list) + 1000)
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
        assert st['status'] == _abi.STATUS_MAXSTEPS and st['steps'] == nsteps, st
        out[i] = b.download(s)
    return out, b, slots


def test_fp64_batch_equals_single_session_bitwise(sa_cases):
    outs, _, _ = run_batch(sa_cases, 64, 25)
    for i, (spec, mesh) in enumerate(sa_cases):
        u0 = cases.initial_state(mesh, spec.initial_primitive())
        s = StaticAmrGpu.create(mesh, spec.params(), u0)
        s.advance(1e30, 25)
        assert np.array_equal(outs[i], s.download())
        ref = Oracle(mesh, spec.params()).run_steps(u0, 25)
        assert rel_err(outs[i], ref['u'], 5) <= 1e-10


def test_fp32_same_alone_and_in_mix(sa_cases):
    mix, _, _ = run_batch(sa_cases, 32, 40, order=[2, 0, 1])
    for i in range(len(sa_cases)):
        alone, _, _ = run_batch([sa_cases[i]], 32, 40)
        assert np.array_equal(mix[i], alone[0])


def test_fp32_error_against_fp64_oracle(sa_cases):
    nsteps = 100
    outs, b, slots = run_batch(sa_cases, 32, nsteps)
    for i, (spec, mesh) in enumerate(sa_cases):
        u0 = cases.initial_state(mesh, spec.initial_primitive())
        orc = Oracle(mesh, spec.params())
        ref = orc.run_steps(u0, nsteps)
        err = rel_err(outs[i], ref['u'], 5)
        print(f'case {i}: FP32 state max-normalised error after {nsteps} steps: {err:.3e}')
        assert err <= 2e-4
        # loads of the FP32 state evaluated in FP64 vs the FP64 state
        cl32 = loads(orc.diagnostics(outs[i]), spec.mach, spec.aoa)
        cl64 = loads(orc.diagnostics(ref['u']), spec.mach, spec.aoa)
        assert max(abs(a - c) for a, c in zip(cl32, cl64)) <= 1e-4, (cl32, cl64)


def test_admit_release_readmit(sa_cases):
    spec, mesh = sa_cases[0]
    b = Batch(precision=32, model=_abi.MODEL_LAMINAR, sa=True, max_cases=2, max_cells=mesh.n_cells + 10)
    u0 = cases.initial_state(mesh, spec.initial_primitive())
    s0 = b.admit(mesh, spec.params(), u0, case_control(1e30, 10, steady=False))
    assert s0 is not None
    assert b.admit(mesh, spec.params(), u0, case_control(1e30, 10, steady=False)) is None  # no room: returns 3
    for _ in range(2):
        b.advance(8)
    first = b.download(s0)
    b.release(s0)
    assert b.live == 0
    s1 = b.admit(mesh, spec.params(), u0, case_control(1e30, 10, steady=False))
    assert s1 is not None
    for _ in range(2):
        b.advance(8)
    assert np.array_equal(b.download(s1), first)


def test_steady_checks_match_oracle_diagnostics(sa_cases):
    """Check at t*=0.01 and 0.5: norms and loads reduced on the device in FP64 equal the oracle's."""
    spec, mesh = sa_cases[0]
    b = Batch(precision=64, model=_abi.MODEL_LAMINAR, sa=True, max_cases=1, max_cells=mesh.n_cells + 10)
    u0 = cases.initial_state(mesh, spec.initial_primitive())
    s = b.admit(mesh, spec.params(), u0, case_control(0.02, 10 ** 6, steady=True, mach=spec.mach, aoa=spec.aoa,
                                                       check_period=0.015))
    for _ in range(100):
        b.advance(32)
        st = b.status(s)
        if st['time'] >= 0.01:
            break
    b.check()
    st = b.status(s)
    assert st['checks'] == 1 and abs(st['time'] - 0.01) == 0.0
    u = b.download(s)
    orc = Oracle(mesh, spec.params())
    d = orc.diagnostics(u)
    cl, cd, cm = loads(d, spec.mach, spec.aoa)
    np.testing.assert_allclose([st['cl'], st['cd'], st['cm']], [cl, cd, cm], rtol=1e-9, atol=1e-13)
    res = list(d[:4]) + [d[4]]
    np.testing.assert_allclose(st['residual'], res, rtol=1e-9, atol=1e-15)
    ref = orc.run(u0, 0.01, 10 ** 6)
    assert st['steps'] == ref['steps']
