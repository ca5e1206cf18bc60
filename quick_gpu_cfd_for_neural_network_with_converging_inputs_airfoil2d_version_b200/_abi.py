"""ctypes and NumPy mirrors of the C ABI in include/amr_b200.h.

The structured dtypes use C alignment, so their itemsize and field offsets equal those of
the C records, which in turn equal the reference's mesh records (AmrCell2D, AmrFace2D,
WallFragment2D, ... in the reference's src/static_amr2d.h:37-45 and src/euler2d.h:186-190).
"""
import ctypes as C

import numpy as np

ABI_VERSION = 1

BC_INHERIT, BC_TRANSMISSIVE, BC_REFLECT, BC_FARFIELD, BC_TOTAL_INLET, BC_PRESSURE_OUTLET, BC_NOSLIP = -1, 1, 2, 3, 4, 5, 6
MODEL_EULER, MODEL_LAMINAR = 0, 1
MU_CONSTANT, MU_SUTHERLAND = 0, 1
VISCOUS_VOLUME, VISCOUS_SRD = 0, 1
FLUX_HLLC, FLUX_AUSMPUP = 0, 1
LIMITER_FIRST_ORDER = 3
TIME_SSP_RK3 = 0
STATUS_OK, STATUS_NONPHYSICAL_BASE, STATUS_MAXSTEPS, STATUS_DT_UNDERFLOW, STATUS_REJECTIONS, STATUS_BARRIER_TIMEOUT = 0, 2, 3, 4, 5, 9
PRECISION_FP64, PRECISION_FP32 = 64, 32
LAUNCH_AUTO, LAUNCH_PERSISTENT, LAUNCH_PHASES, LAUNCH_SPLIT, LAUNCH_TILED = 0, 1, 2, 3, 4

CELL_DTYPE = np.dtype([('ix', '<i4'), ('iy', '<i4'), ('span', '<i4'), ('level', '<i4'),
                       ('x0', '<f8'), ('x1', '<f8'), ('y0', '<f8'), ('y1', '<f8'),
                       ('volume', '<f8'), ('cx', '<f8'), ('cy', '<f8'),
                       ('wall_begin', '<u8'), ('wall_count', '<u8')], align=True)
FACE_DTYPE = np.dtype([('left', '<i4'), ('right', '<i4'), ('axis', '<i4'), ('boundary', '<i4'),
                       ('coordinate', '<f8'), ('lo', '<f8'), ('hi', '<f8'), ('length', '<f8'),
                       ('centroid', '<f8')], align=True)
WALL_DTYPE = np.dtype([('owner_cell', '<u8'), ('source_edge_id', '<i4'), ('body_id', '<i4'),
                       ('patch_id', '<i4'), ('x0', '<f8'), ('y0', '<f8'), ('x1', '<f8'), ('y1', '<f8'),
                       ('nx', '<f8'), ('ny', '<f8'), ('length', '<f8')], align=True)
TERM_DTYPE = np.dtype([('source', '<i4'), ('side', '<i4'), ('x', '<f8'), ('y', '<f8')], align=True)
SAMPLE_DTYPE = np.dtype([('donor', '<i4'), ('distance', '<f8')], align=True)
GEOMETRY_DTYPE = np.dtype([('dx', '<f8'), ('dy', '<f8'), ('ex', '<f8'), ('ey', '<f8'), ('distance', '<f8')], align=True)
BOUNDARY_DTYPE = np.dtype([('kind', '<i4'), ('reference', '<f8', (4,)), ('total_pressure', '<f8'),
                           ('total_temperature', '<f8'), ('gas_constant', '<f8'), ('direction', '<f8', (2,)),
                           ('outlet_pressure', '<f8'), ('wall_velocity', '<f8', (2,))], align=True)
TRANSPORT_DTYPE = np.dtype([('model', '<i4'), ('law', '<i4'), ('stabilization', '<i4'), ('mu_ref', '<f8'),
                            ('gas_constant', '<f8'), ('temperature_ref', '<f8'), ('sutherland', '<f8'),
                            ('viscous_cfl', '<f8'), ('sa_model', '<i4'), ('sa_nu_inf', '<f8'), ('sa_cfl', '<f8'),
                            ('wall_probe_min_h', '<f8')], align=True)
assert CELL_DTYPE.itemsize == 88 and FACE_DTYPE.itemsize == 56 and WALL_DTYPE.itemsize == 80
assert TERM_DTYPE.itemsize == 24 and SAMPLE_DTYPE.itemsize == 16 and GEOMETRY_DTYPE.itemsize == 40


class Boundary(C.Structure):
    _fields_ = [('kind', C.c_int32), ('reference', C.c_double * 4), ('total_pressure', C.c_double),
                ('total_temperature', C.c_double), ('gas_constant', C.c_double), ('direction', C.c_double * 2),
                ('outlet_pressure', C.c_double), ('wall_velocity', C.c_double * 2)]


class Transport(C.Structure):
    _fields_ = [('model', C.c_int32), ('law', C.c_int32), ('stabilization', C.c_int32), ('mu_ref', C.c_double),
                ('gas_constant', C.c_double), ('temperature_ref', C.c_double), ('sutherland', C.c_double),
                ('viscous_cfl', C.c_double), ('sa_model', C.c_int32), ('sa_nu_inf', C.c_double),
                ('sa_cfl', C.c_double), ('wall_probe_min_h', C.c_double)]


assert C.sizeof(Boundary) == BOUNDARY_DTYPE.itemsize and C.sizeof(Transport) == TRANSPORT_DTYPE.itemsize


class Params(C.Structure):
    _fields_ = [('gamma', C.c_double), ('cfl', C.c_double), ('dt_fixed', C.c_double), ('ausm_mco', C.c_double),
                ('flux', C.c_int32), ('limiter', C.c_int32), ('time_integrator', C.c_int32), ('bc', C.c_int32 * 4)]


_P = C.c_void_p


class MeshView(C.Structure):
    _fields_ = [('n_cells', C.c_uint64), ('n_faces', C.c_uint64), ('n_walls', C.c_uint64),
                ('cells', _P), ('faces', _P), ('walls', _P),
                ('face_offsets', _P), ('cell_faces', _P),
                ('group_offsets', _P), ('group_members', _P), ('member_offsets', _P), ('member_groups', _P),
                ('group_volume', _P), ('small_cells', C.c_uint64), ('agglomerate_small', C.c_int32),
                ('boundaries', Boundary * 4), ('transport', Transport),
                ('visc_offsets', _P), ('visc_terms', _P), ('wall_samples', _P), ('face_samples', _P),
                ('face_geometry', _P), ('wall_distance', _P)]


class MeshBox(C.Structure):
    _fields_ = [('x0', C.c_double), ('x1', C.c_double), ('y0', C.c_double), ('y1', C.c_double), ('level', C.c_int32)]


class MeshOptions(C.Structure):
    _fields_ = [('nx', C.c_int32), ('ny', C.c_int32), ('levels', C.c_int32), ('buffer', C.c_int32),
                ('xmin', C.c_double), ('xmax', C.c_double), ('ymin', C.c_double), ('ymax', C.c_double),
                ('max_cells', C.c_uint64), ('agglomerate_small', C.c_int32), ('n_boxes', C.c_int32), ('boxes', _P)]


class MeshRequest(C.Structure):
    _fields_ = [('options', _P), ('px', _P), ('py', _P), ('patches', _P), ('n_points', C.c_uint64),
                ('boundaries', _P), ('transport', _P), ('params', _P)]


class MeshExtras(C.Structure):
    _fields_ = [('coarse_fine_faces', C.c_uint64), ('split_leaves', C.c_uint64), ('agglomeration', _P),
                ('n_agglomeration', C.c_uint64), ('leaf_components', _P), ('n_leaf_components', C.c_uint64)]


class ExportRows(C.Structure):
    _fields_ = [('wall_rows', _P), ('sa_rows', _P), ('convective_dt', C.c_double), ('viscous_dt', C.c_double)]


class MeshCounts(C.Structure):
    _fields_ = [('background_leaves', C.c_uint64), ('split_leaves', C.c_uint64), ('coarse_fine_faces', C.c_uint64),
                ('small_cells', C.c_uint64), ('n_terms', C.c_uint64)]


class GpuOptions(C.Structure):
    _fields_ = [('batch_trials', C.c_int32), ('graph', C.c_int32), ('fused', C.c_int32), ('event_timing', C.c_int32),
                ('sa_fused', C.c_int32), ('device', C.c_int32), ('block_threads', C.c_int32), ('grid_blocks', C.c_int32),
                ('launch_mode', C.c_int32)]


class GpuStats(C.Structure):
    _fields_ = [('allocated_bytes', C.c_uint64), ('pinned_bytes', C.c_uint64), ('geometry_h2d_bytes', C.c_uint64),
                ('state_h2d_bytes', C.c_uint64), ('control_h2d_bytes', C.c_uint64), ('control_d2h_bytes', C.c_uint64),
                ('state_d2h_bytes', C.c_uint64), ('status_polls', C.c_uint64), ('full_downloads', C.c_uint64),
                ('setup_seconds', C.c_double), ('advance_seconds', C.c_double), ('download_seconds', C.c_double),
                ('advance_event_seconds', C.c_double), ('event_batches', C.c_uint64),
                ('graph_nodes_per_trial', C.c_uint64)]


class StateMeta(C.Structure):
    _fields_ = [('time', C.c_double), ('steps', C.c_int64), ('rejected', C.c_int64), ('status', C.c_int32),
                ('finished', C.c_int32)]


class BatchConfig(C.Structure):
    _fields_ = [('precision', C.c_int32), ('device', C.c_int32), ('model', C.c_int32), ('sa_model', C.c_int32),
                ('flux', C.c_int32), ('max_cases', C.c_int32), ('max_cells', C.c_uint64), ('max_faces', C.c_uint64),
                ('max_walls', C.c_uint64), ('max_terms', C.c_uint64), ('max_srd', C.c_uint64), ('hbm_bytes', C.c_uint64),
                ('block_threads', C.c_int32), ('grid_blocks', C.c_int32), ('launch_mode', C.c_int32)]


class CaseControl(C.Structure):
    _fields_ = [('tend', C.c_double), ('maxsteps', C.c_int64), ('first_check', C.c_double), ('check_period', C.c_double),
                ('min_time', C.c_double), ('raw_tol', C.c_double), ('load_tol', C.c_double), ('hold', C.c_int32),
                ('region', C.c_double * 4), ('moment_x', C.c_double), ('moment_y', C.c_double), ('mach', C.c_double),
                ('aoa_degrees', C.c_double)]


class CaseStatus(C.Structure):
    _fields_ = [('time', C.c_double), ('steps', C.c_int64), ('rejected', C.c_int64), ('status', C.c_int32),
                ('finished', C.c_int32), ('converged', C.c_int32), ('checks', C.c_int32), ('hold', C.c_int32),
                ('residual', C.c_double * 5), ('cl', C.c_double), ('cd', C.c_double), ('cm', C.c_double)]


def ptr(array):
    """Address of a contiguous NumPy array (None for None)."""
    if array is None:
        return None
    assert array.flags['C_CONTIGUOUS']
    return array.ctypes.data
