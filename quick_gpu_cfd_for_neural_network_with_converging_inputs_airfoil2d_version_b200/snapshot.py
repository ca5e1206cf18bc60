"""Compact results and result files in the reference's formats.

    rows = session.export()                        # or batch.export(slot, mesh): computed on the device
    write_mesh_files('out/raw', mesh, params)      # <raw>.cells.npy, .walls.npy, .mesh.json, ...
    write_snapshot_files('out/raw.final', mesh, params, u, time, steps, rejected, rows)

The files are those of the reference's static_amr_binary_mesh / static_amr_binary_snapshot
(src/static_amr2d_binary.cpp:25-69), byte for byte, so the reference's pipeline/export.py reads
them unchanged.  Every call goes through the C ABI (amr_write_*, amr_*_export).
"""
import ctypes as C

import numpy as np

from . import _abi
from ._lib import errbuf, lib


class SnapshotError(RuntimeError):
    pass


def export_rows(call, mesh):
    """Runs an amr_*_export call with buffers shaped for `mesh`; returns a dict of wall_rows
    (n_walls x 14, viscous models), sa_rows (n_cells x 3, SA) and the dt limits."""
    viscous = int(mesh.transport['model'][0]) == _abi.MODEL_LAMINAR
    sa = viscous and int(mesh.transport['sa_model'][0]) == 1
    walls = np.zeros((mesh.n_walls if viscous else 0, 14))
    sa_rows = np.zeros((mesh.n_cells if sa else 0, 3))
    limits = np.zeros(2)
    err = errbuf()
    if call(walls.ctypes.data if walls.size else None, walls.size, sa_rows.ctypes.data if sa_rows.size else None,
            sa_rows.size, limits.ctypes.data, err, len(err)):
        raise SnapshotError(err.value.decode())
    return dict(wall_rows=walls if viscous else None, sa_rows=sa_rows if sa else None,
                convective_dt=float(limits[0]), viscous_dt=float(limits[1]))


def _options(mesh):
    o = mesh.options
    boxes = o.get('boxes', [])
    arr = (_abi.MeshBox * max(1, len(boxes)))()
    for i, b in enumerate(boxes):
        arr[i] = _abi.MeshBox(float(b[0]), float(b[1]), float(b[2]), float(b[3]), int(b[4]))
    opts = _abi.MeshOptions(int(o['nx']), int(o['ny']), int(o['levels']), int(o['buffer']), float(o['xmin']),
                            float(o['xmax']), float(o['ymin']), float(o['ymax']), int(o.get('max_cells', 0)),
                            int(mesh.agglomerate_small), len(boxes), C.addressof(arr))
    return opts, arr


def write_npy(path, values):
    a = np.ascontiguousarray(values, dtype=np.float64)
    if a.ndim != 2:
        raise ValueError('write_npy takes a 2-D array')
    err = errbuf()
    if lib().amr_write_npy(str(path).encode(), a.ctypes.data, a.shape[0], a.shape[1], err, len(err)):
        raise SnapshotError(err.value.decode())


def write_mesh_files(prefix, mesh, params):
    view = mesh.view()
    opts, _boxes = _options(mesh)
    ex = _abi.MeshExtras()
    ex.coarse_fine_faces = int(mesh.options.get('coarse_fine_faces', 0))
    ex.split_leaves = int(mesh.options.get('split_leaves', 0))
    agg = None if mesh.agglomeration is None else np.ascontiguousarray(mesh.agglomeration, dtype=np.float64)
    lc = None if mesh.leaf_components is None else np.ascontiguousarray(mesh.leaf_components, dtype=np.uint64)
    if agg is not None:
        ex.agglomeration, ex.n_agglomeration = agg.ctypes.data, len(agg)
    if lc is not None:
        ex.leaf_components, ex.n_leaf_components = lc.ctypes.data, len(lc)
    err = errbuf()
    if lib().amr_write_mesh_files(str(prefix).encode(), C.byref(view), C.byref(opts), C.byref(params), C.byref(ex), err,
                                  len(err)):
        raise SnapshotError(err.value.decode())


def write_snapshot_files(prefix, mesh, params, u, time, steps, rejected, rows=None, backend='cuda'):
    view = mesh.view()
    opts, _boxes = _options(mesh)
    u = np.ascontiguousarray(u, dtype=np.float64)
    if len(u) != mesh.nv * mesh.n_cells:
        raise ValueError('state size does not match the mesh')
    r = _abi.ExportRows()
    keep = []
    if rows is not None:
        if rows.get('wall_rows') is not None:
            w = np.ascontiguousarray(rows['wall_rows'], dtype=np.float64)
            keep.append(w)
            r.wall_rows = w.ctypes.data
        if rows.get('sa_rows') is not None:
            s = np.ascontiguousarray(rows['sa_rows'], dtype=np.float64)
            keep.append(s)
            r.sa_rows = s.ctypes.data
        r.convective_dt, r.viscous_dt = rows['convective_dt'], rows['viscous_dt']
    err = errbuf()
    if lib().amr_write_snapshot_files(str(prefix).encode(), C.byref(view), C.byref(opts), C.byref(params), u.ctypes.data,
                                      float(time), int(steps), int(rejected), backend.encode(),
                                      C.byref(r) if rows is not None else None, err, len(err)):
        raise SnapshotError(err.value.decode())
