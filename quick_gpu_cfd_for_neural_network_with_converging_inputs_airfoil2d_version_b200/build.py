"""Builds libamr_b200.so (sm_100a) in the package directory.

    python -m quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.build

The FP64 unit is compiled with -fmad=false so its arithmetic rounds exactly like the
reference CPU code; the FP32 unit uses contraction and the fast division, square root and
transcendental paths (its accuracy is set by the FP32 state, not by the last bit of these).
"""
import concurrent.futures
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
CSRC = PKG / 'csrc'
BUILD = PKG / '_build'
LIB = PKG / 'libamr_b200.so'
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
COMMON = ['-O3', '-std=c++17', '-lineinfo', '-Xcompiler', '-fPIC', '-I', str(PKG.parent / 'include')]
UNITS = {
    'amr_engine_f64.cu': ['-fmad=false'],
    'amr_engine_f32.cu': ['--use_fast_math'],
    'amr_capi.cu': [],
    'amr_static.cu': ['-fmad=false'],
}
# Host-only units, compiled by the system g++ (the compiler, libstdc++ and libm the reference
# CPU core is built with) without floating-point contraction.
HOST_UNITS = {
    'amr_mesh.cpp': ['-O2', '-ffp-contract=off', '-fno-fast-math'],
    'amr_export.cpp': ['-O2', '-ffp-contract=off', '-fno-fast-math'],
}
HOST_CXX = '/usr/bin/g++' if os.path.exists('/usr/bin/g++') else (shutil.which('g++') or 'g++')


def nvcc():
    path = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    if not os.path.exists(path):
        raise RuntimeError('nvcc not found')
    return path


def _sources():
    return (sorted(CSRC.glob('*.cu')) + sorted(CSRC.glob('*.cuh')) + sorted(CSRC.glob('*.h')) + sorted(CSRC.glob('*.cpp')) +
            [PKG.parent / 'include' / 'amr_b200.h'])


def up_to_date():
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(s.stat().st_mtime <= t for s in _sources())


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    BUILD.mkdir(exist_ok=True)
    cc = nvcc()

    def compile_unit(item):
        name, extra = item
        obj = BUILD / (name + '.o')
        if name in HOST_UNITS:
            cmd = [HOST_CXX, '-std=c++17', '-fPIC', '-g', '-I', str(PKG.parent / 'include'), *extra, '-c', str(CSRC / name),
                   '-o', str(obj)]
        else:
            cmd = [cc, *ARCH, *COMMON, *extra, '-c', str(CSRC / name), '-o', str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(f'nvcc failed for {name}:\n{r.stderr[-4000:]}')
        if verbose:
            print(r.stderr)
        return obj

    units = {**UNITS, **HOST_UNITS}
    with concurrent.futures.ThreadPoolExecutor(max_workers=len(units)) as ex:
        objs = list(ex.map(compile_unit, units.items()))
    tmp = LIB.with_suffix('.so.tmp')
    r = subprocess.run([cc, *ARCH, '-shared', '-o', str(tmp), *map(str, objs), '-lcudart', '-lpthread'], capture_output=True,
                       text=True)
    if r.returncode:
        raise RuntimeError('link failed:\n' + r.stderr[-4000:])
    os.replace(tmp, LIB)
    return LIB


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose='-v' in sys.argv)
    print(LIB)
