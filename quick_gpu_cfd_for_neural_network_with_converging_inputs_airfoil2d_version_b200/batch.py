"""Python mirror of the batched C API (amr_batch_* in include/amr_b200.h).

Many meshes live in one device arena; each case keeps its own time, dt, retry counter and
status, and is retired by the reference driver's steady rule (src/quick_airfoil.cpp:180-208)
evaluated on the device in FP64.
"""
import ctypes as C

import numpy as np

from . import _abi, cases
from ._lib import errbuf, lib


class BatchError(RuntimeError):
    pass


def device_memory(device=0):
    """(free, total) bytes of device memory (cudaMemGetInfo)."""
    free, total = C.c_uint64(), C.c_uint64()
    if lib().amr_device_memory(int(device), C.byref(free), C.byref(total)):
        raise BatchError(f'cannot query device {device}')
    return free.value, total.value


def group_advance(batches, trials=32):
    """Runs `trials` trials of every batch (all on one device) with their work in flight together,
    each on its own stream after one start event; returns the device seconds from that start to
    the last batch's end.  Each batch ends exactly as after its own advance(trials)."""
    n = len(batches)
    handles = (C.c_void_p * n)(*[b._h for b in batches])
    seconds = C.c_double()
    err = errbuf()
    if lib().amr_batch_group_advance(handles, n, int(trials), C.byref(seconds), err, len(err)):
        raise BatchError(err.value.decode())
    return seconds.value


def case_control(tend, maxsteps, steady=True, mach=1.65, aoa=1.5, **kw):
    c = _abi.CaseControl()
    s = dict(cases.STEADY)
    s.update(kw)
    c.tend, c.maxsteps = float(tend), int(maxsteps)
    c.first_check = s['first_check']
    c.check_period = s['check_period'] if steady else 0.0
    c.min_time, c.raw_tol, c.load_tol, c.hold = s['min_time'], s['raw_tol'], s['load_tol'], int(s['hold'])
    for i in range(4):
        c.region[i] = s['region'][i]
    c.moment_x, c.moment_y = s['moment_x'], s['moment_y']
    c.mach, c.aoa_degrees = mach, aoa
    return c


class Batch:
    def __init__(self, precision=32, model=_abi.MODEL_LAMINAR, sa=True, flux=_abi.FLUX_HLLC, max_cases=256,
                 max_cells=0, max_faces=0, max_walls=0, max_terms=0, max_srd=0, hbm_bytes=0, block_threads=0,
                 grid_blocks=0, device=0, launch_mode=0):
        cfg = _abi.BatchConfig()
        cfg.precision, cfg.device, cfg.model, cfg.sa_model, cfg.flux = precision, device, model, int(sa), flux
        cfg.max_cases = max_cases
        cfg.max_cells, cfg.max_faces, cfg.max_walls, cfg.max_terms, cfg.max_srd = max_cells, max_faces, max_walls, max_terms, max_srd
        cfg.hbm_bytes, cfg.block_threads, cfg.grid_blocks = hbm_bytes, block_threads, grid_blocks
        cfg.launch_mode = launch_mode
        out = C.c_void_p()
        err = errbuf()
        if lib().amr_batch_create(C.byref(cfg), C.byref(out), err, len(err)):
            raise BatchError(err.value.decode())
        self._h = out.value
        self.nv = 5 if (model == _abi.MODEL_LAMINAR and sa) else 4
        self.ncells = {}

    def admit(self, mesh, params, u0, control):
        """Admits one case; u0 is the SoA start state (nv * n_cells values) or, for a uniform start,
        the nv conserved values (cases.uniform_state), which the device fills in.  Returns the slot,
        or None when the arena has no room."""
        u0 = np.ascontiguousarray(u0, dtype=np.float64)
        view = mesh.view()
        slot = C.c_int32(-1)
        err = errbuf()
        st = lib().amr_batch_admit(self._h, C.byref(view), C.byref(params), u0.ctypes.data, len(u0), C.byref(control),
                                   C.byref(slot), err, len(err))
        if st == 3:
            return None
        if st:
            raise BatchError(err.value.decode())
        self.ncells[slot.value] = mesh.n_cells
        return slot.value

    def admit_many(self, items, threads=0):
        """Admits (mesh, params, u0, control) tuples in one call, converting them on `threads`
        host threads (0: up to 16).  Returns one slot per item (None where the arena had no
        room); slots and placement equal those of admitting the items one by one, in order.
        Raises BatchError naming the first invalid item (the valid ones stay admitted; their
        slots are on the exception's `slots`)."""
        n = len(items)
        if n == 0:
            return []
        u0s = [np.ascontiguousarray(u0, dtype=np.float64) for _, _, u0, _ in items]
        views = [mesh.view() for mesh, _, _, _ in items]
        params = [p for _, p, _, _ in items]
        controls = [c for _, _, _, c in items]
        P = C.c_void_p * n
        meshes_p = P(*[C.addressof(v) for v in views])
        params_p = P(*[C.addressof(p) for p in params])
        u0_p = P(*[u.ctypes.data for u in u0s])
        ctl_p = P(*[C.addressof(c) for c in controls])
        counts = (C.c_uint64 * n)(*[len(u) for u in u0s])
        slots = (C.c_int32 * n)()
        status = (C.c_int32 * n)()
        err = errbuf()
        lib().amr_batch_admit_many(self._h, n, meshes_p, params_p, u0_p, counts, ctl_p, int(threads), slots, status,
                                   err, len(err))
        out = []
        for (mesh, _, _, _), s, st in zip(items, slots, status):
            if st == 0:
                self.ncells[s] = mesh.n_cells
            out.append(s if st == 0 else None)
        if any(st == 1 for st in status):
            e = BatchError(err.value.decode())
            e.slots = out
            raise e
        return out

    def advance(self, trials=32):
        err = errbuf()
        if lib().amr_batch_advance(self._h, int(trials), err, len(err)):
            raise BatchError(err.value.decode())

    def advance_async(self, trials=32):
        """Enqueues `trials` trials and returns at once; wait() completes them.  Make no other call
        on the batch in between."""
        err = errbuf()
        if lib().amr_batch_advance_async(self._h, int(trials), err, len(err)):
            raise BatchError(err.value.decode())

    def wait(self):
        err = errbuf()
        if lib().amr_batch_wait(self._h, err, len(err)):
            raise BatchError(err.value.decode())

    def check(self):
        err = errbuf()
        if lib().amr_batch_check(self._h, err, len(err)):
            raise BatchError(err.value.decode())

    def status(self, slot):
        s = _abi.CaseStatus()
        lib().amr_batch_status(self._h, int(slot), C.byref(s))
        return dict(time=s.time, steps=s.steps, rejected=s.rejected, status=s.status, finished=s.finished,
                    converged=s.converged, checks=s.checks, hold=s.hold, residual=list(s.residual), cl=s.cl, cd=s.cd,
                    cm=s.cm)

    def download(self, slot):
        u = np.empty(self.nv * self.ncells[slot])
        err = errbuf()
        if lib().amr_batch_download(self._h, int(slot), u.ctypes.data, len(u), err, len(err)):
            raise BatchError(err.value.decode())
        return u

    def download_many(self, slots):
        """The accepted states of several cases (one staged copy, one synchronisation)."""
        slots = list(slots)
        outs = [np.empty(self.nv * self.ncells[s]) for s in slots]
        n = len(slots)
        if n == 0:
            return []
        err = errbuf()
        if lib().amr_batch_download_many(self._h, n, (C.c_int32 * n)(*slots), (C.c_void_p * n)(*[u.ctypes.data for u in outs]),
                                         (C.c_uint64 * n)(*[len(u) for u in outs]), err, len(err)):
            raise BatchError(err.value.decode())
        return outs

    def export(self, slot, mesh):
        """Device-computed compact results of a case (see StaticAmrGpu.export)."""
        from .snapshot import export_rows
        return export_rows(lambda *a: lib().amr_batch_export(self._h, int(slot), *a), mesh)

    def residual(self, slot):
        r = np.empty(self.nv * self.ncells[slot])
        err = errbuf()
        if lib().amr_batch_residual(self._h, int(slot), r.ctypes.data, len(r), err, len(err)):
            raise BatchError(err.value.decode())
        return r

    def set_target(self, slot, target, maxsteps):
        err = errbuf()
        if lib().amr_batch_set_target(self._h, int(slot), float(target), int(maxsteps), err, len(err)):
            raise BatchError(err.value.decode())

    def release(self, slot):
        lib().amr_batch_release(self._h, int(slot))
        self.ncells.pop(slot, None)

    def autotune(self, trials=4):
        err = errbuf()
        if lib().amr_batch_autotune(self._h, int(trials), err, len(err)):
            raise BatchError(err.value.decode())

    def set_graph(self, on):
        lib().amr_batch_set_graph(self._h, int(bool(on)))

    def set_lanes(self, lanes):
        """Split mode, viscous models without SRD: run the live cases as `lanes` (1..4) chains of
        kernels in flight together (amr_batch_set_lanes)."""
        if lib().amr_batch_set_lanes(self._h, int(lanes)):
            raise BatchError('lanes must be 1..4')

    def launch_config(self):
        b = errbuf(128)
        lib().amr_batch_launch_config(self._h, b, len(b))
        return b.value.decode()

    @property
    def device_bytes(self):
        """Device memory the batch allocated."""
        return lib().amr_batch_device_bytes(self._h)

    @property
    def live(self):
        return lib().amr_batch_live_cases(self._h)

    @property
    def free_cells(self):
        return lib().amr_batch_free_cells(self._h)

    @property
    def last_advance_seconds(self):
        return lib().amr_batch_last_advance_seconds(self._h)

    @property
    def kernel_launches(self):
        return lib().amr_batch_kernel_launches(self._h)

    def destroy(self):
        if self._h:
            lib().amr_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
