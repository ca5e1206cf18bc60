"""Python mirror of the host mesh builder (amr_mesh_* in include/amr_b200.h).

    mesh = build_mesh(spec, x, y, patches)                 # one mesh, as MeshArrays
    meshes = build_meshes([(spec, x, y, patches), ...])    # many, on all host threads

Each call replaces the reference's static_amr2d_build + static_amr2d_prepare_viscous pair
(src/static_amr2d.cpp:229, src/static_amr2d_viscous.cpp:40) with the same arguments: the
mesh options of the case's profile, the closed body polygon and its patch ids, and the
boundary/transport records the tables depend on.  A failed build raises MeshBuildError with
the reference's message.
"""
import ctypes as C

import numpy as np

from . import _abi
from ._lib import errbuf, lib
from .mesh import MeshArrays


class MeshBuildError(RuntimeError):
    pass


class _Request:
    """Keeps the ctypes request and every buffer it points to alive."""

    def __init__(self, spec, x, y, patches, gamma=1.4):
        o = spec.options()
        self.options_dict = o
        boxes = o.get('boxes', [])
        self.boxes = (_abi.MeshBox * max(1, len(boxes)))()
        for i, b in enumerate(boxes):
            self.boxes[i] = _abi.MeshBox(float(b[0]), float(b[1]), float(b[2]), float(b[3]), int(b[4]))
        self.options = _abi.MeshOptions(int(o['nx']), int(o['ny']), int(o['levels']), int(o['buffer']), float(o['xmin']),
                                        float(o['xmax']), float(o['ymin']), float(o['ymax']), int(o['max_cells']),
                                        int(o.get('agglomerate_small', 0)), len(boxes), C.addressof(self.boxes))
        self.x = np.ascontiguousarray(x, dtype=np.float64)
        self.y = np.ascontiguousarray(y, dtype=np.float64)
        self.patches = None if patches is None else np.ascontiguousarray(patches, dtype=np.int32)
        self.bnd = np.ascontiguousarray(spec.boundary_records(gamma))
        self.tr = np.ascontiguousarray(spec.transport_record(gamma))
        self.params = spec.params(gamma)
        self.req = _abi.MeshRequest(C.addressof(self.options), self.x.ctypes.data, self.y.ctypes.data,
                                    None if self.patches is None else self.patches.ctypes.data, len(self.x),
                                    self.bnd.ctypes.data, self.tr.ctypes.data, C.addressof(self.params))


def _take(handle, options):
    v = _abi.MeshView()
    lib().amr_mesh_view(C.c_void_p(handle), C.byref(v))
    counts = _abi.MeshCounts()
    lib().amr_mesh_get_counts(C.c_void_p(handle), C.byref(counts))
    m = MeshArrays.from_view(v, options)
    m.options.update(background_leaves=counts.background_leaves, split_leaves=counts.split_leaves,
                     coarse_fine_faces=counts.coarse_fine_faces)
    ex = _abi.MeshExtras()
    lib().amr_mesh_get_extras(C.c_void_p(handle), C.byref(ex))
    if ex.n_agglomeration:
        buf = (C.c_double * (9 * ex.n_agglomeration)).from_address(ex.agglomeration)
        m.agglomeration = np.frombuffer(buf, dtype=np.float64).reshape(-1, 9).copy()
    if ex.n_leaf_components:
        buf = (C.c_uint64 * (2 * ex.n_leaf_components)).from_address(ex.leaf_components)
        m.leaf_components = np.frombuffer(buf, dtype=np.uint64).reshape(-1, 2).copy()
    lib().amr_mesh_destroy(C.c_void_p(handle))
    return m


def build_mesh(spec, x, y, patches=None, gamma=1.4):
    r = _Request(spec, x, y, patches, gamma)
    out = C.c_void_p()
    err = errbuf()
    if lib().amr_mesh_build(C.byref(r.req), C.byref(out), err, len(err)):
        raise MeshBuildError(err.value.decode())
    return _take(out.value, r.options_dict)


def build_meshes(items, threads=0, gamma=1.4, raise_on_error=True):
    """Builds [(spec, x, y, patches), ...] on `threads` host threads (0 = all cores).  Returns a
    list of MeshArrays (None where a build failed when raise_on_error is False)."""
    reqs = [_Request(spec, x, y, patches, gamma) for spec, x, y, patches in items]
    n = len(reqs)
    if n == 0:
        return []
    arr = (_abi.MeshRequest * n)(*[r.req for r in reqs])
    handles = (C.c_void_p * n)()
    status = (C.c_int32 * n)()
    stride = 256
    errors = C.create_string_buffer(n * stride)
    lib().amr_mesh_build_many(n, arr, int(threads), handles, status, errors, stride)
    out = []
    for i in range(n):
        if status[i]:
            msg = errors.raw[i * stride:(i + 1) * stride].split(b'\0', 1)[0].decode()
            if raise_on_error:
                for j in range(n):
                    if handles[j]:
                        lib().amr_mesh_destroy(C.c_void_p(handles[j]))
                raise MeshBuildError(f'request {i}: {msg}')
            out.append(None)
        else:
            out.append(_take(handles[i], reqs[i].options_dict))
    return out
