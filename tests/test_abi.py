"""CPU tests of the C ABI: the library loads and exports every declared entry point; record
layouts agree between the header, the ctypes mirror and the NumPy dtypes."""
import ctypes as C
import re

import numpy as np

from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import _abi, _lib, airfoils, cases
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.mesh import MeshArrays


def declared_functions(root):
    text = (root / 'include' / 'amr_b200.h').read_text()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'^\s*(?:int|void|double|uint64_t)\s+\**(amr_\w+)\s*\(', text, flags=re.M)))


def test_library_exports_every_declared_symbol(golden):
    root = golden.parents[1]
    names = declared_functions(root)
    assert len(names) >= 20
    lib = _lib.lib()
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, name


def test_record_layouts():
    assert _abi.CELL_DTYPE.fields['volume'][1] == 48 and _abi.CELL_DTYPE.fields['wall_count'][1] == 80
    assert _abi.WALL_DTYPE.fields['x0'][1] == 24 and _abi.WALL_DTYPE.fields['length'][1] == 72
    assert C.sizeof(_abi.GpuStats) == 8 * 15
    assert C.sizeof(_abi.MeshView) > 0


def test_mesh_roundtrip(golden, tmp_path):
    m = MeshArrays.load(golden / 'mesh_naca2412_lf1_sa.npz')
    m.save(tmp_path / 'm.npz')
    m2 = MeshArrays.load(tmp_path / 'm.npz')
    v = m2.view()
    back = MeshArrays.from_view(v, m2.options)
    for name in MeshArrays._ARRAYS:
        a, b = getattr(m, name), getattr(back, name)
        if a is None:
            assert b is None
        else:
            if a.dtype.names:
                for f in a.dtype.names:
                    assert np.array_equal(a[f], b[f]), (name, f)
            else:
                assert np.array_equal(a, b), name


def test_naca_generator_convention():
    x, y, pt = airfoils.naca4(0.0, 0.4, 0.12)
    assert len(x) == 200 and x[0] == 1.0 and y[0] == 0.0 and x[100] == 0.0 and y[100] == 0.0
    pts = set(zip(x, y))
    assert len(pts) == 200
    area = 0.5 * np.sum(x * np.roll(y, -1) - np.roll(x, -1) * y)
    assert area > 0
    np.testing.assert_allclose(y[1:100], -y[199:100:-1], rtol=0, atol=1e-15)
    x2, y2, _ = airfoils.naca4(0.02, 0.4, 0.12)
    assert y2[50] > -y2[150]  # cambered upward


def test_initial_state_matches_reference_formula(golden):
    m = MeshArrays.load(golden / 'mesh_naca2412_lf1_sa.npz')
    w = cases.freestream(1.65, 1.5)
    u = cases.initial_state(m, w)
    n = m.n_cells
    assert u[0] == 1.0 and u[n] == w[1] and u[3 * n] == w[3] / (1.4 - 1) + 0.5 * (w[1] * w[1] + w[2] * w[2])
    assert u[4 * n] == cases.nondimensional()['sa_nu_inf']
