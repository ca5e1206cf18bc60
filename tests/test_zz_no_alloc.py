"""GPU test of amr_euler_residual_static, the residual entry point that allocates no device memory.

It serves callers that cannot call cudaMalloc where they need a residual (a foreign memory pool
or allocator, a latency-critical loop, a plug-in handed device buffers); they pass their own
device copies of the mesh and state, and the scratch lives in a static device array.  The test
gives it device buffers (allocated here, by the test), calls it twice in a row through the C ABI
on two different states, and compares each result with the session's amr_gpu_residual within the
parity tolerance of the other GPU tests.  This file is collected last."""
import ctypes as C

import numpy as np
import pytest

from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import cases
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200._lib import errbuf, lib
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.mesh import MeshArrays
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.session import StaticAmrGpu, default_options

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel_err(a, b, nv):
    a = a.reshape(nv, -1)
    b = b.reshape(nv, -1)
    return max(np.abs(a[v] - b[v]).max() / max(np.abs(b[v]).max(), 1e-300) for v in range(nv))


def device_copy(array):
    import torch
    raw = np.ascontiguousarray(array).view(np.uint8).reshape(-1)
    return torch.from_numpy(raw.copy()).cuda()


def static_residual(mesh, params, bufs, u):
    import torch
    d_u = device_copy(u)
    d_r = torch.full((4 * mesh.n_cells,), float('nan'), dtype=torch.float64, device='cuda')
    err = errbuf()
    st = lib().amr_euler_residual_static(
        bufs['cells'].data_ptr(), mesh.n_cells, bufs['faces'].data_ptr(), mesh.n_faces, bufs['walls'].data_ptr(),
        mesh.n_walls, bufs['face_offsets'].data_ptr(), bufs['cell_faces'].data_ptr(), mesh.boundaries.ctypes.data,
        C.addressof(params), d_u.data_ptr(), d_r.data_ptr(), None, err, len(err))
    assert st == 0, err.value.decode()
    torch.cuda.synchronize()
    return d_r.cpu().numpy()


def test_static_residual_matches_session_residual(golden):
    mesh = MeshArrays.load(golden / 'mesh_naca0012_lf1_euler_srd.npz')
    spec = cases.CaseSpec(physics='euler', profile='LF1', mach=1.65, aoa=1.5)
    params = spec.params()
    u0 = cases.initial_state(mesh, spec.initial_primitive())
    bufs = {name: device_copy(getattr(mesh, name)) for name in ('cells', 'faces', 'walls', 'face_offsets', 'cell_faces')}
    s = StaticAmrGpu.create(mesh, params, u0, options=default_options(graph=0))
    # call 1: the uniform initial state
    r0 = static_residual(mesh, params, bufs, u0)
    assert rel_err(r0, s.residual(), 4) <= TOL
    # call 2: a developed state (the scratch still holds call 1's contents)
    s.advance(1e30, 25)
    u = s.download()
    r1 = static_residual(mesh, params, bufs, u)
    assert rel_err(r1, s.residual(), 4) <= TOL
    assert not np.array_equal(r0, r1)


def test_static_residual_rejects_meshes_beyond_capacity(golden):
    mesh = MeshArrays.load(golden / 'mesh_naca0012_lf1_euler_srd.npz')
    params = cases.CaseSpec(physics='euler').params()
    err = errbuf()
    fake = C.c_void_p(16)
    st = lib().amr_euler_residual_static(fake, 16385, fake, 1, None, 0, fake, fake, mesh.boundaries.ctypes.data,
                                         C.addressof(params), fake, fake, None, err, len(err))
    assert st == 1 and 'capacity' in err.value.decode()


def test_static_residual_reports_out_of_range_mesh_indices(golden):
    """A face whose boundary side is not 0..3 and a cell whose wall range runs past n_walls are
    skipped on the device (nothing is read through them) and returned as an error."""
    import torch
    mesh = MeshArrays.load(golden / 'mesh_naca0012_lf1_euler_srd.npz')
    spec = cases.CaseSpec(physics='euler', profile='LF1', mach=1.65, aoa=1.5)
    params = spec.params()
    u0 = cases.initial_state(mesh, spec.initial_primitive())
    for table, field, value in (('faces', 'boundary', 7), ('cells', 'wall_count', mesh.n_walls + 5)):
        broken = getattr(mesh, table).copy()
        broken[field][3] = value
        bufs = {name: device_copy(broken if name == table else getattr(mesh, name))
                for name in ('cells', 'faces', 'walls', 'face_offsets', 'cell_faces')}
        d_u = device_copy(u0)
        d_r = torch.zeros(4 * mesh.n_cells, dtype=torch.float64, device='cuda')
        err = errbuf()
        st = lib().amr_euler_residual_static(
            bufs['cells'].data_ptr(), mesh.n_cells, bufs['faces'].data_ptr(), mesh.n_faces, bufs['walls'].data_ptr(),
            mesh.n_walls, bufs['face_offsets'].data_ptr(), bufs['cell_faces'].data_ptr(), mesh.boundaries.ctypes.data,
            C.addressof(params), d_u.data_ptr(), d_r.data_ptr(), None, err, len(err))
        assert st == 1 and 'out of range' in err.value.decode(), (table, err.value.decode())
    # a well-formed call afterwards still succeeds (the status word is cleared per call)
    bufs = {name: device_copy(getattr(mesh, name)) for name in ('cells', 'faces', 'walls', 'face_offsets', 'cell_faces')}
    r = static_residual(mesh, params, bufs, u0)
    assert np.isfinite(r).all()
