"""CPU tests of the result-file writers (amr_write_npy, amr_write_mesh_files,
amr_write_snapshot_files): every file must be byte-identical to the one the reference's own
writer (static_amr_write_npy / static_amr_binary_mesh / static_amr_binary_snapshot, compiled from
its sources into oracle/_ref) produces from the same mesh and state."""
import ctypes as C

import numpy as np
import pytest

from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import airfoils, builder, cases, snapshot
from oracle.oracle import RefCase, ref_lib


def same_tree(a_prefix, b_prefix):
    """Names and bytes of every file written under two prefixes."""
    a_dir, b_dir = a_prefix.parent, b_prefix.parent
    a = {p.name[len(a_prefix.name):]: p.read_bytes() for p in a_dir.iterdir() if p.name.startswith(a_prefix.name)}
    b = {p.name[len(b_prefix.name):]: p.read_bytes() for p in b_dir.iterdir() if p.name.startswith(b_prefix.name)}
    assert sorted(a) == sorted(b), (sorted(a), sorted(b))
    for k in a:
        assert a[k] == b[k], k
    return sorted(a)


@pytest.mark.parametrize('shape', [(3, 4), (0, 14), (1, 1), (257, 9)])
def test_npy_bytes_match_reference_writer(tmp_path, shape):
    x = np.random.default_rng(1).standard_normal(shape)
    snapshot.write_npy(tmp_path / 'ours.npy', x)
    ref_lib().ref_write_npy(str(tmp_path / 'ref.npy').encode(), x.ctypes.data if x.size else None, shape[0], shape[1])
    assert (tmp_path / 'ours.npy').read_bytes() == (tmp_path / 'ref.npy').read_bytes()
    assert np.array_equal(np.load(tmp_path / 'ours.npy'), x)


@pytest.mark.parametrize('physics,profile,kinds', [
    ('sa', 'LF1', ('farfield',) * 4),
    ('euler', 'LF1', ('farfield',) * 4),
    ('laminar', 'LF2', ('farfield', 'pressure-outlet', 'no-slip', 'no-slip')),
])
def test_mesh_files_match_reference(tmp_path, physics, profile, kinds):
    naca = (0.02, 0.4, 0.12)
    spec = cases.CaseSpec(naca=naca, profile=profile, physics=physics, kinds=kinds)
    x, y, pt = airfoils.naca4(*naca)
    mesh = builder.build_mesh(spec, x, y, pt)
    (tmp_path / 'ours').mkdir()
    (tmp_path / 'ref').mkdir()
    snapshot.write_mesh_files(tmp_path / 'ours' / 'raw', mesh, spec.params())
    RefCase.build(spec, x, y, pt).write_mesh(tmp_path / 'ref' / 'raw')
    names = same_tree(tmp_path / 'ours' / 'raw', tmp_path / 'ref' / 'raw')
    assert '.cells.npy' in names and '.mesh.json' in names and '.bc.json' in names
    if physics != 'euler':
        assert '.agglomeration.npy' in names and '.gradient_table.csv' in names


def test_euler_snapshot_files_match_reference(tmp_path):
    naca = (0.0, 0.4, 0.12)
    spec = cases.CaseSpec(naca=naca, profile='LF1', physics='euler')
    x, y, pt = airfoils.naca4(*naca)
    rc = RefCase.build(spec, x, y, pt)
    mesh = builder.build_mesh(spec, x, y, pt)
    u0 = cases.initial_state(mesh, spec.initial_primitive())
    out = rc.run_steps(u0, 5)
    (tmp_path / 'ours').mkdir()
    (tmp_path / 'ref').mkdir()
    snapshot.write_snapshot_files(tmp_path / 'ours' / 'raw.final', mesh, spec.params(), out['u'], out['time'],
                                  out['steps'], out['rejected'])
    rc.write_snapshot(tmp_path / 'ref' / 'raw.final', out['u'], out['time'], out['steps'], out['rejected'])
    assert same_tree(tmp_path / 'ours' / 'raw.final', tmp_path / 'ref' / 'raw.final') == ['.json', '.state.npy']


def test_viscous_snapshot_needs_rows(tmp_path):
    naca = (0.0, 0.4, 0.12)
    spec = cases.CaseSpec(naca=naca, profile='LF1', physics='sa')
    x, y, pt = airfoils.naca4(*naca)
    mesh = builder.build_mesh(spec, x, y, pt)
    u0 = cases.initial_state(mesh, spec.initial_primitive())
    with pytest.raises(snapshot.SnapshotError, match='exported wall'):
        snapshot.write_snapshot_files(tmp_path / 'raw.final', mesh, spec.params(), u0, 0.0, 0, 0)
