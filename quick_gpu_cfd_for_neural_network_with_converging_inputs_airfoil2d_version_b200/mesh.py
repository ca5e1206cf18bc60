"""Host-side container of one static AMR mesh in the flat layout of include/amr_b200.h.

A MeshArrays owns NumPy arrays for every table of the reference's StaticAmrMesh2D
(src/static_amr2d.h:46-66) and AmrViscousTable2D (src/static_amr2d_viscous.h:26-32) and
hands the engine an amr_mesh_view_t of pointers into them.  It also stores the mesh build
options so the mesh can be saved to and loaded from a compressed .npz file.
"""
import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi

_U8 = np.uint64


@dataclass
class MeshArrays:
    cells: np.ndarray
    faces: np.ndarray
    walls: np.ndarray
    face_offsets: np.ndarray
    cell_faces: np.ndarray
    group_offsets: np.ndarray
    group_members: np.ndarray
    member_offsets: np.ndarray
    member_groups: np.ndarray
    group_volume: np.ndarray
    small_cells: int
    agglomerate_small: int
    boundaries: np.ndarray          # BOUNDARY_DTYPE, shape (4,)
    transport: np.ndarray           # TRANSPORT_DTYPE, shape (1,)
    visc_offsets: np.ndarray = None
    visc_terms: np.ndarray = None
    wall_samples: np.ndarray = None
    face_samples: np.ndarray = None
    face_geometry: np.ndarray = None
    wall_distance: np.ndarray = None
    options: dict = field(default_factory=dict)  # build options (bounds, base shape, levels, ...)
    agglomeration: np.ndarray = None      # (n_original, 9) build record of agglomerated meshes
    leaf_components: np.ndarray = None    # (m, 2) uint64 (background leaf, control volume)

    @property
    def n_cells(self):
        return len(self.cells)

    @property
    def n_faces(self):
        return len(self.faces)

    @property
    def n_walls(self):
        return len(self.walls)

    @property
    def nv(self):
        return 5 if int(self.transport['sa_model'][0]) else 4

    @property
    def laminar(self):
        return int(self.transport['model'][0]) == _abi.MODEL_LAMINAR

    def view(self):
        """amr_mesh_view_t pointing into this object's arrays (valid while self lives)."""
        v = _abi.MeshView()
        v.n_cells, v.n_faces, v.n_walls = self.n_cells, self.n_faces, self.n_walls
        p = _abi.ptr
        v.cells, v.faces, v.walls = p(self.cells), p(self.faces), p(self.walls)
        v.face_offsets, v.cell_faces = p(self.face_offsets), p(self.cell_faces)
        v.group_offsets, v.group_members = p(self.group_offsets), p(self.group_members)
        v.member_offsets, v.member_groups = p(self.member_offsets), p(self.member_groups)
        v.group_volume = p(self.group_volume)
        v.small_cells, v.agglomerate_small = int(self.small_cells), int(self.agglomerate_small)
        C.memmove(C.addressof(v.boundaries), self.boundaries.ctypes.data, C.sizeof(v.boundaries))
        C.memmove(C.addressof(v.transport), self.transport.ctypes.data, C.sizeof(v.transport))
        if self.laminar:
            v.visc_offsets, v.visc_terms = p(self.visc_offsets), p(self.visc_terms)
            v.wall_samples, v.face_samples = p(self.wall_samples), p(self.face_samples)
            v.face_geometry = p(self.face_geometry)
            v.wall_distance = p(self.wall_distance)
        return v

    @classmethod
    def from_view(cls, v, options=None):
        """Deep copy of a view's tables into NumPy arrays."""
        def take(address, dtype, count):
            if count == 0:
                return np.zeros(0, dtype=dtype)
            assert address, 'null table pointer'
            buf = (C.c_char * (count * np.dtype(dtype).itemsize)).from_address(address)
            return np.frombuffer(buf, dtype=dtype, count=count).copy()
        n, nf, nw = v.n_cells, v.n_faces, v.n_walls
        face_offsets = take(v.face_offsets, _U8, n + 1)
        group_offsets = take(v.group_offsets, _U8, n + 1)
        member_offsets = take(v.member_offsets, _U8, n + 1)
        boundaries = np.frombuffer(bytes(v.boundaries), dtype=_abi.BOUNDARY_DTYPE).copy()
        transport = np.frombuffer(bytes(v.transport), dtype=_abi.TRANSPORT_DTYPE).copy()
        m = cls(cells=take(v.cells, _abi.CELL_DTYPE, n), faces=take(v.faces, _abi.FACE_DTYPE, nf),
                walls=take(v.walls, _abi.WALL_DTYPE, nw), face_offsets=face_offsets,
                cell_faces=take(v.cell_faces, _U8, int(face_offsets[-1])), group_offsets=group_offsets,
                group_members=take(v.group_members, _U8, int(group_offsets[-1])), member_offsets=member_offsets,
                member_groups=take(v.member_groups, _U8, int(member_offsets[-1])),
                group_volume=take(v.group_volume, np.float64, n), small_cells=int(v.small_cells),
                agglomerate_small=int(v.agglomerate_small), boundaries=boundaries, transport=transport,
                options=dict(options or {}))
        if int(transport['model'][0]) == _abi.MODEL_LAMINAR:
            m.visc_offsets = take(v.visc_offsets, _U8, n + 1)
            m.visc_terms = take(v.visc_terms, _abi.TERM_DTYPE, int(m.visc_offsets[-1]))
            m.wall_samples = take(v.wall_samples, _abi.SAMPLE_DTYPE, nw)
            m.face_samples = take(v.face_samples, _abi.SAMPLE_DTYPE, nf)
            m.face_geometry = take(v.face_geometry, _abi.GEOMETRY_DTYPE, nf)
            if int(transport['sa_model'][0]):
                m.wall_distance = take(v.wall_distance, np.float64, n)
        return m

    _ARRAYS = ('cells', 'faces', 'walls', 'face_offsets', 'cell_faces', 'group_offsets', 'group_members',
               'member_offsets', 'member_groups', 'group_volume', 'boundaries', 'transport', 'visc_offsets',
               'visc_terms', 'wall_samples', 'face_samples', 'face_geometry', 'wall_distance')

    def save(self, path):
        data = {k: getattr(self, k) for k in self._ARRAYS if getattr(self, k) is not None}
        data['scalars'] = np.array([self.small_cells, self.agglomerate_small], dtype=np.int64)
        for k in ('agglomeration', 'leaf_components'):
            if getattr(self, k) is not None:
                data[k] = getattr(self, k)
        opts = dict(self.options)
        data['options_json'] = np.frombuffer(__import__('json').dumps(opts).encode(), dtype=np.uint8)
        np.savez_compressed(path, **data)

    @classmethod
    def load(cls, path):
        import json
        z = np.load(path)
        kw = {k: z[k] for k in cls._ARRAYS if k in z.files}
        small, agg = (int(x) for x in z['scalars'])
        opts = json.loads(bytes(z['options_json']).decode()) if 'options_json' in z.files else {}
        for k in ('agglomeration', 'leaf_components'):
            if k in z.files:
                kw[k] = z[k]
        return cls(small_cells=small, agglomerate_small=agg, options=opts, **kw)

    def with_physics(self, boundaries=None, transport=None):
        """Shallow copy with replaced boundary records and/or transport record."""
        import copy
        m = copy.copy(self)
        if boundaries is not None:
            m.boundaries = np.ascontiguousarray(boundaries, dtype=_abi.BOUNDARY_DTYPE)
        if transport is not None:
            m.transport = np.ascontiguousarray(transport, dtype=_abi.TRANSPORT_DTYPE).reshape(1)
        return m
