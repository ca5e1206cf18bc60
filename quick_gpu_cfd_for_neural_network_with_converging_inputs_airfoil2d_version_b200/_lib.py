"""Loads libamr_b200.so (the CUDA engine behind include/amr_b200.h) and declares its symbols.

There is no fallback: if the library is missing or does not load, every entry point raises.
"""
import ctypes as C
import pathlib

from . import _abi

LIB_PATH = pathlib.Path(__file__).resolve().parent / 'libamr_b200.so'

# name -> (restype, argtypes); every symbol declared in include/amr_b200.h plus the extras
_P = C.c_void_p
_S = C.c_char_p
SIGNATURES = {
    'amr_gpu_default_options': (None, [_P]),
    'amr_gpu_create': (C.c_int, [_P, _P, _P, C.c_uint64, C.c_double, C.c_int64, C.c_int64, _P, _P, _S, C.c_uint64]),
    'amr_gpu_advance': (C.c_int, [_P, C.c_double, C.c_int64, C.c_double, _P, _S, C.c_uint64]),
    'amr_gpu_download': (C.c_int, [_P, _P, C.c_uint64, _P, _S, C.c_uint64]),
    'amr_gpu_stats': (C.c_int, [_P, _P]),
    'amr_gpu_destroy': (None, [_P]),
    'amr_gpu_residual': (C.c_int, [_P, _P, C.c_uint64, _S, C.c_uint64]),
    'amr_gpu_diagnostics': (C.c_int, [_P, _P, C.c_double, C.c_double, _P, _S, C.c_uint64]),
    'amr_euler_residual_static': (C.c_int, [_P, C.c_uint64, _P, C.c_uint64, _P, C.c_uint64, _P, _P, _P, _P, _P, _P, _P,
                                            _S, C.c_uint64]),
    'amr_batch_create': (C.c_int, [_P, _P, _S, C.c_uint64]),
    'amr_batch_admit': (C.c_int, [_P, _P, _P, _P, C.c_uint64, _P, _P, _S, C.c_uint64]),
    'amr_batch_admit_many': (C.c_int, [_P, C.c_uint64, _P, _P, _P, _P, _P, C.c_int32, _P, _P, _S, C.c_uint64]),
    'amr_batch_advance': (C.c_int, [_P, C.c_int32, _S, C.c_uint64]),
    'amr_batch_advance_async': (C.c_int, [_P, C.c_int32, _S, C.c_uint64]),
    'amr_batch_wait': (C.c_int, [_P, _S, C.c_uint64]),
    'amr_batch_group_advance': (C.c_int, [_P, C.c_int32, C.c_int32, _P, _S, C.c_uint64]),
    'amr_batch_device_bytes': (C.c_uint64, [_P]),
    'amr_device_memory': (C.c_int, [C.c_int32, _P, _P]),
    'amr_batch_check': (C.c_int, [_P, _S, C.c_uint64]),
    'amr_batch_status': (C.c_int, [_P, C.c_int32, _P]),
    'amr_batch_download': (C.c_int, [_P, C.c_int32, _P, C.c_uint64, _S, C.c_uint64]),
    'amr_batch_download_many': (C.c_int, [_P, C.c_uint64, _P, _P, _P, _S, C.c_uint64]),
    'amr_batch_release': (C.c_int, [_P, C.c_int32]),
    'amr_batch_live_cases': (C.c_int, [_P]),
    'amr_batch_free_cells': (C.c_uint64, [_P]),
    'amr_batch_last_advance_seconds': (C.c_double, [_P]),
    'amr_batch_kernel_launches': (C.c_uint64, [_P]),
    'amr_batch_destroy': (None, [_P]),
    'amr_mesh_build': (C.c_int, [_P, _P, _S, C.c_uint64]),
    'amr_mesh_build_many': (C.c_int, [C.c_uint64, _P, C.c_int32, _P, _P, _P, C.c_uint64]),
    'amr_mesh_view': (C.c_int, [_P, _P]),
    'amr_mesh_get_counts': (C.c_int, [_P, _P]),
    'amr_mesh_destroy': (None, [_P]),
    'amr_mesh_get_extras': (C.c_int, [_P, _P]),
    'amr_gpu_export': (C.c_int, [_P, _P, C.c_uint64, _P, C.c_uint64, _P, _S, C.c_uint64]),
    'amr_batch_export': (C.c_int, [_P, C.c_int32, _P, C.c_uint64, _P, C.c_uint64, _P, _S, C.c_uint64]),
    'amr_write_npy': (C.c_int, [_S, _P, C.c_uint64, C.c_uint64, _S, C.c_uint64]),
    'amr_write_mesh_files': (C.c_int, [_S, _P, _P, _P, _P, _S, C.c_uint64]),
    'amr_write_snapshot_files': (C.c_int, [_S, _P, _P, _P, _P, C.c_double, C.c_int64, C.c_int64, _S, _P, _S,
                                           C.c_uint64]),
    # extras used by the host mirror
    'amr_batch_autotune': (C.c_int, [_P, C.c_int32, _S, C.c_uint64]),
    'amr_batch_launch_config': (C.c_int, [_P, _S, C.c_uint64]),
    'amr_batch_set_graph': (C.c_int, [_P, C.c_int32]),
    'amr_batch_set_lanes': (C.c_int, [_P, C.c_int32]),
    'amr_batch_set_target': (C.c_int, [_P, C.c_int32, C.c_double, C.c_int64, _S, C.c_uint64]),
    'amr_batch_residual': (C.c_int, [_P, C.c_int32, _P, C.c_uint64, _S, C.c_uint64]),
    'amr_gpu_launch_config': (C.c_int, [_P, _S, C.c_uint64]),
    'amr_gpu_kernel_launches': (C.c_uint64, [_P]),
}

_lib = None


def lib():
    """The loaded engine library; raises if it is absent or incomplete."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f'{LIB_PATH} is missing; build it with '
                               'python -m quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.build')
        h = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _lib = h
    return _lib


def errbuf(n=512):
    return C.create_string_buffer(n)
