"""GPU tests of the on-device export (amr_gpu_export / amr_batch_export): the wall-stress rows,
SA cell rows and dt limits computed on the device from the FP64 session's state, written by the
snapshot writer, must give files byte-identical to the reference's static_amr_binary_snapshot on
the same state; the FP32 batch's rows must agree with them to FP32 accuracy."""
import numpy as np
import pytest

from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import _abi, airfoils, builder, cases, snapshot
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.batch import Batch, case_control
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.session import StaticAmrGpu
from oracle.oracle import RefCase
from tests.test_snapshot_files import same_tree

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('physics,kinds,steps', [
    ('sa', ('farfield',) * 4, 12),
    ('laminar', ('farfield', 'pressure-outlet', 'no-slip', 'no-slip'), 8),
    ('laminar-srd-rate', ('farfield', 'pressure-outlet', 'farfield', 'farfield'), 6),
])
def test_viscous_snapshot_files_match_reference(tmp_path, physics, kinds, steps):
    naca = (0.02, 0.4, 0.12)
    if physics == 'laminar-srd-rate':
        from tests.test_gpu_parity import srd_rate_spec
        spec = srd_rate_spec()
    else:
        spec = cases.CaseSpec(naca=naca, profile='LF1', physics=physics, kinds=kinds)
    x, y, pt = airfoils.naca4(*naca)
    mesh = builder.build_mesh(spec, x, y, pt)
    rc = RefCase.build(spec, x, y, pt)
    u0 = cases.initial_state(mesh, spec.initial_primitive())
    s = StaticAmrGpu.create(mesh, spec.params(), u0)
    s.advance(1e30, steps)
    u = s.download()
    ref = rc.run_steps(u0, steps)
    assert np.array_equal(u, ref['u']) and s.time == ref['time']
    rows = s.export()
    assert rows['wall_rows'].shape == (mesh.n_walls, 14)
    assert (rows['sa_rows'] is not None) == (physics == 'sa')
    assert np.isfinite(rows['viscous_dt']) and np.isfinite(rows['convective_dt'])
    (tmp_path / 'ours').mkdir()
    (tmp_path / 'ref').mkdir()
    snapshot.write_snapshot_files(tmp_path / 'ours' / 'raw.final', mesh, spec.params(), u, s.time, s.steps, s.rejected,
                                  rows)
    rc.write_snapshot(tmp_path / 'ref' / 'raw.final', ref['u'], ref['time'], ref['steps'], ref['rejected'])
    names = same_tree(tmp_path / 'ours' / 'raw.final', tmp_path / 'ref' / 'raw.final')
    assert '.wall_stress.npy' in names and '.viscous_loads.json' in names and '.timestep_limits.json' in names


def test_batch_export_fp32_close_to_fp64():
    naca = (0.02, 0.4, 0.12)
    spec = cases.CaseSpec(naca=naca, profile='LF1', physics='sa')
    x, y, pt = airfoils.naca4(*naca)
    mesh = builder.build_mesh(spec, x, y, pt)
    u0 = cases.initial_state(mesh, spec.initial_primitive())
    s = StaticAmrGpu.create(mesh, spec.params(), u0)
    s.advance(1e30, 32)
    exact = s.export()
    b = Batch(precision=32, model=_abi.MODEL_LAMINAR, sa=True, max_cases=2, max_cells=2 * mesh.n_cells + 100,
              launch_mode=_abi.LAUNCH_SPLIT, block_threads=128)
    slot = b.admit(mesh, spec.params(), u0, case_control(1e30, 32, steady=False))
    b.advance(32)
    got = b.export(slot, mesh)
    w, we = got['wall_rows'], exact['wall_rows']
    assert np.array_equal(w[:, :3], we[:, :3])                     # indices
    for col in (3, 8, 9, 10):                                       # distance, pressure, pressure forces
        assert np.max(np.abs(w[:, col] - we[:, col])) <= 1e-4 * np.max(np.abs(we[:, col]))
    for col in (4, 11, 12):                                         # viscosity, viscous forces
        assert np.max(np.abs(w[:, col] - we[:, col])) <= 1e-3 * np.max(np.abs(we[:, col]))
    assert abs(got['convective_dt'] / exact['convective_dt'] - 1) < 1e-4
    assert abs(got['viscous_dt'] / exact['viscous_dt'] - 1) < 1e-3
