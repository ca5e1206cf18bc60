"""Python mirror of the reference session API (src/static_amr2d_gpu.h:17-24 in the reference).

    s = StaticAmrGpu.create(mesh, params, u0, time=0, steps=0, rejected=0, options=None)
    status = s.advance(tend, maxsteps, wall_budget_seconds=0)   # 0 done, 1 fatal, 2 budget
    u = s.download()
    stats = s.stats()
    s.destroy()

Same argument meaning, return codes and error behaviour as static_amr_gpu_create / advance /
download / stats / destroy; the state is SoA u[var*n + cell].  Every call goes through the C ABI
of include/amr_b200.h (libamr_b200.so).
"""
import ctypes as C

import numpy as np

from . import _abi
from ._lib import errbuf, lib


class AmrGpuError(RuntimeError):
    pass


def default_options(**overrides):
    o = _abi.GpuOptions()
    lib().amr_gpu_default_options(C.byref(o))
    for k, v in overrides.items():
        setattr(o, k, v)
    return o


class StaticAmrGpu:
    def __init__(self, handle, mesh, nv):
        self._h = handle
        self.mesh = mesh
        self.nv = nv
        self.meta = _abi.StateMeta()
        self.last_error = ''

    @classmethod
    def create(cls, mesh, params, u0, time=0.0, steps=0, rejected=0, options=None):
        u0 = np.ascontiguousarray(u0, dtype=np.float64)
        view = mesh.view()
        opts = options if options is not None else default_options()
        out = C.c_void_p()
        err = errbuf()
        st = lib().amr_gpu_create(C.byref(view), C.byref(params), u0.ctypes.data, len(u0), float(time), int(steps),
                                  int(rejected), C.byref(opts), C.byref(out), err, len(err))
        if st:
            raise AmrGpuError(err.value.decode())
        s = cls(out.value, mesh, mesh.nv)
        s.meta.time, s.meta.steps, s.meta.rejected = time, steps, rejected
        return s

    def advance(self, tend, maxsteps, wall_budget_seconds=0.0):
        err = errbuf()
        st = lib().amr_gpu_advance(self._h, float(tend), int(maxsteps), float(wall_budget_seconds), C.byref(self.meta),
                                   err, len(err))
        self.last_error = err.value.decode()
        return st

    def download(self):
        u = np.empty(self.nv * self.mesh.n_cells)
        err = errbuf()
        if lib().amr_gpu_download(self._h, u.ctypes.data, len(u), C.byref(self.meta), err, len(err)):
            raise AmrGpuError(err.value.decode())
        return u

    def export(self):
        """Device-computed compact results of the accepted state: wall-stress rows (n_walls x 14,
        viscous models), SA cell rows (n_cells x 3) and the (convective, viscous) dt limits."""
        from .snapshot import export_rows
        return export_rows(lambda *a: lib().amr_gpu_export(self._h, *a), self.mesh)

    def residual(self):
        r = np.empty(self.nv * self.mesh.n_cells)
        err = errbuf()
        if lib().amr_gpu_residual(self._h, r.ctypes.data, len(r), err, len(err)):
            raise AmrGpuError(err.value.decode())
        return r

    def diagnostics(self, region=(-1.0, 3.0, -1.0, 1.0), moment=(0.25, 0.0)):
        reg = np.ascontiguousarray(region, dtype=np.float64)
        out = np.zeros(8)
        err = errbuf()
        if lib().amr_gpu_diagnostics(self._h, reg.ctypes.data, moment[0], moment[1], out.ctypes.data, err, len(err)):
            raise AmrGpuError(err.value.decode())
        return out

    def stats(self):
        s = _abi.GpuStats()
        lib().amr_gpu_stats(self._h, C.byref(s))
        return {name: getattr(s, name) for name, _ in s._fields_}

    def launch_config(self):
        b = errbuf(128)
        lib().amr_gpu_launch_config(self._h, b, len(b))
        return b.value.decode()

    def kernel_launches(self):
        return lib().amr_gpu_kernel_launches(self._h)

    @property
    def time(self):
        return self.meta.time

    @property
    def steps(self):
        return self.meta.steps

    @property
    def rejected(self):
        return self.meta.rejected

    def destroy(self):
        if self._h:
            lib().amr_gpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
