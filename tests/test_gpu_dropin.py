"""The reference's own driver (src/quick_airfoil.cpp), built against this engine through
include/static_amr2d_gpu.h in place of the reference CUDA backend (oracle/Makefile `dropin`),
run with backend cuda and backend cpu on the reference's example G0001."""
import json
import pathlib
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = pathlib.Path(__file__).resolve().parents[1]
BIN = ROOT / 'oracle' / '_ref' / 'quick_airfoil_b200'


def write_inputs(golden, folder, mode, backend, profile='LF1'):
    ka = json.loads((golden / 'known_answers.json').read_text())
    lines = []
    for line in ka['settings']['default_' + profile].splitlines():
        key = line.split(' ', 1)[0]
        if key == 'mode':
            line = 'mode ' + mode
        elif key == 'backend':
            line = 'backend ' + backend
        lines.append(line)
    (folder / 'settings.txt').write_text('\n'.join(lines) + '\n')
    z = np.load(golden / 'examples.npz')
    i = list(z['names']).index('G0001')
    a, b = z['offsets'][i], z['offsets'][i + 1]
    (folder / 'airfoil.csv').write_text('x,y\n' + ''.join(f'{float(x)!r},{float(y)!r}\n' for x, y in zip(z['x'][a:b], z['y'][a:b])))
    (folder / 'patches.csv').write_text('edge,patch\n' + ''.join(f'{j},{int(p)}\n' for j, p in enumerate(z['patches'][a:b])))


def run(golden, tmp_path, mode, backend, profile='LF1'):
    folder = tmp_path / f'{mode}_{backend}_{profile}'
    (folder / 'internal').mkdir(parents=True)
    write_inputs(golden, folder, mode, backend, profile)
    cmd = [str(BIN), '--settings', str(folder / 'settings.txt'), '--geometry', str(folder / 'airfoil.csv'),
           '--patches', str(folder / 'patches.csv'), '--out', str(folder / 'internal' / 'flow')]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    return json.loads((folder / 'internal' / 'flow.result.json').read_text())


def test_reference_driver_on_b200_matches_cpu_backend(golden, tmp_path):
    if not BIN.exists():
        pytest.fail(f'{BIN} missing: make -C oracle dropin')
    gpu = run(golden, tmp_path, 'smoke', 'cuda')
    cpu = run(golden, tmp_path, 'smoke', 'cpu')
    assert gpu['fluid_control_volumes'] == cpu['fluid_control_volumes'] == 4725
    assert gpu['steps'] == cpu['steps'] == 41 and gpu['rejected'] == cpu['rejected'] == 0
    assert gpu['physical_time'] == cpu['physical_time'] == 0.01
    for key in ('Cl', 'Cd', 'Cm'):
        assert abs(gpu[key] - cpu[key]) <= 1e-8, (key, gpu[key], cpu[key])
    for a, b in zip(gpu['raw_residual'], cpu['raw_residual']):
        assert abs(a - b) <= 1e-8 * max(abs(b), 1e-12)


def test_reference_driver_rest_state_on_b200(golden, tmp_path):
    """The driver's own known answer: a rest state stays within L_inf 2e-11 (exit code 0)."""
    if not BIN.exists():
        pytest.fail(f'{BIN} missing: make -C oracle dropin')
    r = run(golden, tmp_path, 'rest', 'cuda')
    assert r['rest_linf'] <= 2e-11 and not r['failed']
