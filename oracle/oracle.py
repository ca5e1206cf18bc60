"""TEST INFRASTRUCTURE: ctypes access to the checker libraries in oracle/_ref/.

  RefCase   the reference's own CPU core (mesh builder, static_amr2d_run, static_amr2d_rhs,
            driver diagnostics), compiled from the reference sources by oracle/Makefile.
  Oracle    the C restatement of the time step (oracle/amr_oracle.c).
  RefGpu    the reference CUDA session compiled for sm_100a (timing comparisons only).

Only tests/, the smoke check and bench.py's CPU-baseline leg use this module.
"""
import ctypes as C
import os
import pathlib

import numpy as np

from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import _abi
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.mesh import MeshArrays

HERE = pathlib.Path(__file__).resolve().parent
REF_DIR = HERE / '_ref'


class MeshOptions(C.Structure):
    _fields_ = [('nx', C.c_int32), ('ny', C.c_int32), ('levels', C.c_int32), ('buffer', C.c_int32),
                ('xmin', C.c_double), ('xmax', C.c_double), ('ymin', C.c_double), ('ymax', C.c_double),
                ('max_cells', C.c_uint64), ('agglomerate_small', C.c_int32), ('n_boxes', C.c_int32),
                ('boxes', C.c_void_p)]


def mesh_options_struct(o):
    boxes = np.ascontiguousarray(np.array(o.get('boxes', []), dtype=np.float64).reshape(-1, 5))
    s = MeshOptions(int(o['nx']), int(o['ny']), int(o['levels']), int(o['buffer']), float(o['xmin']),
                    float(o['xmax']), float(o['ymin']), float(o['ymax']), int(o['max_cells']),
                    int(o.get('agglomerate_small', 0)), len(boxes), boxes.ctypes.data if len(boxes) else None)
    return s, boxes


def _load(name):
    path = REF_DIR / name
    if not path.exists():
        raise FileNotFoundError(f'{path} is missing: build it with `make -C oracle {name}`')
    return C.CDLL(str(path))


_ref_libs = {}


def ref_lib(kind='serial'):
    name = {'serial': 'libamr_ref.so', 'omp': 'libamr_ref_omp.so', 'cuda': 'libamr_ref_cuda.so'}[kind]
    if name not in _ref_libs:
        lib = _load(name)
        P = C.c_void_p
        lib.ref_case_build.restype = P
        lib.ref_case_build.argtypes = [P, P, P, P, C.c_int32, P, P, P, C.c_char_p, C.c_uint64]
        lib.ref_case_from_view.restype = P
        lib.ref_case_from_view.argtypes = [P, P, P]
        lib.ref_case_view.argtypes = [P, P]
        lib.ref_case_counts.argtypes = [P, P]
        lib.ref_case_initialize.argtypes = [P, P, P]
        lib.ref_case_run.argtypes = [P, P, C.c_uint64, P, P, P, C.c_double, C.c_int64, C.c_char_p, C.c_uint64]
        lib.ref_case_write_mesh.argtypes = [P, C.c_char_p, C.c_char_p, C.c_uint64]
        lib.ref_case_write_snapshot.argtypes = [P, P, C.c_uint64, C.c_double, C.c_int64, C.c_int64, C.c_char_p,
                                                C.c_char_p, C.c_char_p, C.c_uint64]
        lib.ref_write_npy.argtypes = [C.c_char_p, P, C.c_uint64, C.c_uint64]
        lib.ref_case_run_timed.restype = C.c_double
        lib.ref_case_run_timed.argtypes = [P, P, C.c_uint64, P, P, P, C.c_double, C.c_int64, P]
        lib.ref_case_rhs.argtypes = [P, P, P]
        lib.ref_case_redistribute.argtypes = [P, P]
        lib.ref_case_diagnostics.argtypes = [P, P, P, C.c_double, C.c_double, P]
        lib.ref_case_destroy.argtypes = [P]
        if kind == 'cuda':
            lib.ref_gpu_create.restype = P
            lib.ref_gpu_create.argtypes = [P, P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_uint64]
            lib.ref_gpu_advance.argtypes = [P, C.c_double, C.c_int64, P, P, P, C.c_char_p, C.c_uint64]
            lib.ref_gpu_download.argtypes = [P, P]
            lib.ref_gpu_event_seconds.restype = C.c_double
            lib.ref_gpu_event_seconds.argtypes = [P]
            lib.ref_gpu_graph_nodes.restype = C.c_uint64
            lib.ref_gpu_graph_nodes.argtypes = [P]
            lib.ref_gpu_destroy.argtypes = [P]
        _ref_libs[name] = lib
    return _ref_libs[name]


class RefCase:
    """A mesh + parameters held by the reference CPU core."""

    def __init__(self, handle, lib, params, options):
        self.h, self.lib, self.params, self.options = handle, lib, params, options
        counts = (C.c_uint64 * 11)()
        lib.ref_case_counts(C.c_void_p(handle), counts)
        self.counts = dict(zip(['n', 'nf', 'nw', 'cell_faces', 'group_members', 'member_groups', 'terms',
                                'small_cells', 'coarse_fine_faces', 'background_leaves', 'split_leaves'], list(counts)))
        sa = self.mesh().nv == 5
        self.nv = 5 if sa else 4

    @classmethod
    def build(cls, spec, x, y, patches, kind='serial', gamma=1.4):
        lib = ref_lib(kind)
        o = spec.options()
        opts, boxes = mesh_options_struct(o)
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64)
        patches = np.ascontiguousarray(patches, dtype=np.int32)
        bnd = spec.boundary_records(gamma)
        tr = spec.transport_record(gamma)
        params = spec.params(gamma)
        err = C.create_string_buffer(512)
        h = lib.ref_case_build(C.byref(opts), x.ctypes.data, y.ctypes.data, patches.ctypes.data, len(x),
                               bnd.ctypes.data, tr.ctypes.data, C.byref(params), err, 512)
        if not h:
            raise RuntimeError(err.value.decode())
        return cls(h, lib, params, o)

    @classmethod
    def from_mesh(cls, mesh, params, kind='serial'):
        lib = ref_lib(kind)
        opts, boxes = mesh_options_struct(mesh.options)
        v = mesh.view()
        h = lib.ref_case_from_view(C.byref(v), C.byref(params), C.byref(opts))
        return cls(h, lib, params, dict(mesh.options))

    def mesh(self):
        v = _abi.MeshView()
        self.lib.ref_case_view(C.c_void_p(self.h), C.byref(v))
        return MeshArrays.from_view(v, self.options)

    def initial(self, w):
        w = np.ascontiguousarray(w, dtype=np.float64)
        u = np.zeros(self.nv * self.counts['n'])
        assert self.lib.ref_case_initialize(C.c_void_p(self.h), w.ctypes.data, u.ctypes.data) == 0
        return u

    def run(self, u, tend, maxsteps, time=0.0, steps=0, rejected=0):
        u = np.ascontiguousarray(u, dtype=np.float64).copy()
        t, s, r = C.c_double(time), C.c_int64(steps), C.c_int64(rejected)
        err = C.create_string_buffer(512)
        status = self.lib.ref_case_run(C.c_void_p(self.h), u.ctypes.data, len(u), C.byref(t), C.byref(s), C.byref(r),
                                       float(tend), int(maxsteps), err, 512)
        return dict(u=u, time=t.value, steps=s.value, rejected=r.value, status=status, error=err.value.decode())

    def run_steps(self, u, nsteps, **kw):
        """Exactly nsteps accepted steps (tend = 1e30; the maxsteps error is the expected stop)."""
        out = self.run(u, 1e30, kw.pop('steps', 0) + nsteps, **kw)
        assert out['error'] in ('', 'maxsteps reached before tend'), out['error']
        return out

    def run_timed(self, u, tend, maxsteps):
        u = np.ascontiguousarray(u, dtype=np.float64).copy()
        t, s, r, st = C.c_double(0), C.c_int64(0), C.c_int64(0), C.c_int(0)
        sec = self.lib.ref_case_run_timed(C.c_void_p(self.h), u.ctypes.data, len(u), C.byref(t), C.byref(s),
                                          C.byref(r), float(tend), int(maxsteps), C.byref(st))
        return sec, dict(u=u, time=t.value, steps=s.value, rejected=r.value, status=st.value)

    def rhs(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        r = np.zeros_like(u)
        assert self.lib.ref_case_rhs(C.c_void_p(self.h), u.ctypes.data, r.ctypes.data) == 0
        return r

    def redistribute(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64).copy()
        assert self.lib.ref_case_redistribute(C.c_void_p(self.h), u.ctypes.data) == 0
        return u

    def write_mesh(self, prefix):
        err = C.create_string_buffer(512)
        if self.lib.ref_case_write_mesh(C.c_void_p(self.h), str(prefix).encode(), err, 512):
            raise RuntimeError(err.value.decode())

    def write_snapshot(self, prefix, u, time, steps, rejected, backend='cuda'):
        u = np.ascontiguousarray(u, dtype=np.float64)
        err = C.create_string_buffer(512)
        if self.lib.ref_case_write_snapshot(C.c_void_p(self.h), u.ctypes.data, len(u), float(time), int(steps),
                                            int(rejected), str(prefix).encode(), backend.encode(), err, 512):
            raise RuntimeError(err.value.decode())

    def diagnostics(self, u, region=(-1.0, 3.0, -1.0, 1.0), moment=(0.25, 0.0)):
        u = np.ascontiguousarray(u, dtype=np.float64)
        reg = np.ascontiguousarray(region, dtype=np.float64)
        out = np.zeros(8)
        assert self.lib.ref_case_diagnostics(C.c_void_p(self.h), u.ctypes.data, reg.ctypes.data, moment[0],
                                             moment[1], out.ctypes.data) == 0
        return out

    def __del__(self):
        if getattr(self, 'h', None):
            self.lib.ref_case_destroy(C.c_void_p(self.h))
            self.h = None


class RefGpu:
    """The reference CUDA session (src/static_amr2d_cuda.cu) on the current GPU."""

    def __init__(self, case, u0, batch_trials=32, graph=True, fused=True, sa_fused=True, event_timing=True):
        self.lib = ref_lib('cuda')
        assert case.lib is self.lib, 'build the RefCase with kind="cuda"'
        u0 = np.ascontiguousarray(u0, dtype=np.float64)
        err = C.create_string_buffer(512)
        self.h = self.lib.ref_gpu_create(C.c_void_p(case.h), u0.ctypes.data, batch_trials, int(graph), int(fused),
                                         int(sa_fused), int(event_timing), err, 512)
        if not self.h:
            raise RuntimeError(err.value.decode())
        self.n = len(u0)

    def advance(self, tend, maxsteps):
        t, s, r = C.c_double(), C.c_int64(), C.c_int64()
        err = C.create_string_buffer(512)
        st = self.lib.ref_gpu_advance(C.c_void_p(self.h), float(tend), int(maxsteps), C.byref(t), C.byref(s),
                                      C.byref(r), err, 512)
        return dict(status=st, time=t.value, steps=s.value, rejected=r.value, error=err.value.decode())

    def download(self):
        u = np.zeros(self.n)
        assert self.lib.ref_gpu_download(C.c_void_p(self.h), u.ctypes.data) == 0
        return u

    def event_seconds(self):
        return self.lib.ref_gpu_event_seconds(C.c_void_p(self.h))

    def graph_nodes(self):
        return self.lib.ref_gpu_graph_nodes(C.c_void_p(self.h))

    def __del__(self):
        if getattr(self, 'h', None):
            self.lib.ref_gpu_destroy(C.c_void_p(self.h))
            self.h = None


_oracle = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        lib = _load('libamr_oracle.so')
        P = C.c_void_p
        lib.oracle_rhs.argtypes = [P, P, P, P]
        lib.oracle_redistribute.argtypes = [P, P]
        lib.oracle_run.argtypes = [P, P, C.c_double, C.c_int64, P, P, P, P, C.c_char_p, C.c_size_t]
        lib.oracle_diagnostics.argtypes = [P, P, P, P, C.c_double, C.c_double, P]
        _oracle = lib
    return _oracle


class Oracle:
    """The C restatement (oracle/amr_oracle.c) on a MeshArrays."""

    def __init__(self, mesh, params):
        self.mesh, self.params = mesh, params
        self.view = mesh.view()
        self.lib = oracle_lib()

    def rhs(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        r = np.zeros_like(u)
        st = self.lib.oracle_rhs(C.byref(self.view), C.byref(self.params), u.ctypes.data, r.ctypes.data)
        if st:
            raise RuntimeError('oracle residual failed')
        return r

    def redistribute(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64).copy()
        self.lib.oracle_redistribute(C.byref(self.view), u.ctypes.data)
        return u

    def run(self, u, tend, maxsteps, time=0.0, steps=0, rejected=0):
        u = np.ascontiguousarray(u, dtype=np.float64).copy()
        t, s, r = C.c_double(time), C.c_int64(steps), C.c_int64(rejected)
        msg = C.create_string_buffer(256)
        st = self.lib.oracle_run(C.byref(self.view), C.byref(self.params), float(tend), int(maxsteps), u.ctypes.data,
                                 C.byref(t), C.byref(s), C.byref(r), msg, 256)
        return dict(u=u, time=t.value, steps=s.value, rejected=r.value, status=st, error=msg.value.decode())

    def run_steps(self, u, nsteps, **kw):
        out = self.run(u, 1e30, kw.pop('steps', 0) + nsteps, **kw)
        assert out['error'] in ('', 'maxsteps reached before tend'), out['error']
        return out

    def diagnostics(self, u, region=(-1.0, 3.0, -1.0, 1.0), moment=(0.25, 0.0)):
        u = np.ascontiguousarray(u, dtype=np.float64)
        reg = np.ascontiguousarray(region, dtype=np.float64)
        out = np.zeros(8)
        st = self.lib.oracle_diagnostics(C.byref(self.view), C.byref(self.params), u.ctypes.data, reg.ctypes.data,
                                         moment[0], moment[1], out.ctypes.data)
        if st:
            raise RuntimeError('oracle diagnostics failed')
        return out


def loads(out, mach, aoa_degrees):
    """CL, CD, CM from diagnostics' Fx, Fy, Mz (src/quick_airfoil.cpp:152,199)."""
    import math
    a = aoa_degrees * math.acos(-1.0) / 180
    cs, sn, q = math.cos(a), math.sin(a), .5 * mach * mach
    fx, fy, mz = out[5], out[6], out[7]
    return (-fx * sn + fy * cs) / q, (fx * cs + fy * sn) / q, mz / q
