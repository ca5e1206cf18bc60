"""Generates the golden fixtures in tests/golden/ (run in a container that has the reference).

    python tests/golden/make_golden.py [--reference <reference checkout>]  (default: beside this repository)

Writes
  examples.npz      the reference's ten example contours (examples/G*.csv) prepared by the
                    reference's own pipeline/geometry.py: closed polygon + edge patches
  known_answers.json
                    - cells and steps to t*=0.01 per example and profile, from the reference's
                      validation/ten_short_checks.json, re-run here through the reference CPU core
                    - steps of the three control runs (validation/controls_checks.json)
                    - the nondimensional settings the reference pipeline writes
                      (pipeline/configuration.py:143-167) for the default and control configs
                    - published full-steady G0001 loads (validation/summary.json)
  mesh_*.npz        static meshes built by the reference mesh builder, used as synthetic
                    inputs of the single-case workloads (the reference builder is host code
                    that stays on the host; these files stand in for its output on machines
                    without the reference)
"""
import argparse
import json
import math
import pathlib
import sys
import tempfile

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import airfoils, cases  # noqa: E402
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.settings import (  # noqa: E402,F401
    SettingsSpec, parse_settings, spec_from_settings, transport_from_settings)
from oracle.oracle import RefCase  # noqa: E402

GOLDEN = ROOT / 'tests' / 'golden'


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--reference', default=str(pathlib.Path(__file__).resolve().parents[3] / 'reference'))
    args = ap.parse_args()
    ref = pathlib.Path(args.reference)
    sys.path.insert(0, str(ref))
    from pipeline import configuration as rcfg  # the reference's own Python
    from pipeline import geometry as rgeo

    ten = json.loads((ref / 'validation/ten_short_checks.json').read_text())
    controls = json.loads((ref / 'validation/controls_checks.json').read_text())
    summary = json.loads((ref / 'validation/summary.json').read_text())

    # 1. example contours through the reference's contour preparation
    names, xs, ys, ps, offsets = [], [], [], [], [0]
    with tempfile.TemporaryDirectory() as tmp:
        for src in sorted((ref / 'examples').glob('G*_airfoil_points.csv')):
            dst = pathlib.Path(tmp) / src.stem
            rgeo.prepare(src, dst)
            poly = np.loadtxt(dst / 'airfoil.csv', delimiter=',', skiprows=1)
            patch = np.loadtxt(dst / 'patches.csv', delimiter=',', skiprows=1, dtype=np.int64)[:, 1]
            names.append(src.stem.split('_')[0])
            xs.append(poly[:, 0]); ys.append(poly[:, 1]); ps.append(patch.astype(np.int32))
            offsets.append(offsets[-1] + len(poly))
    np.savez_compressed(GOLDEN / 'examples.npz', names=np.array(names), x=np.concatenate(xs), y=np.concatenate(ys),
                        patches=np.concatenate(ps), offsets=np.array(offsets))

    # 2. reference settings for the default config and the three controls
    default_cfg = rcfg.validate(rcfg.load())
    settings = {}
    for label in ('LF1', 'LF2'):
        settings['default_' + label] = rcfg.settings(default_cfg, label, 'G0001')
    control_cfgs = {}
    for name in ('subsonic_outlet', 'fixed_dt', 'cpu_ausm'):
        c = rcfg.validate(rcfg.load(ref / 'validation' / ('control_' + name + '.json')))
        control_cfgs[name] = c
        settings['control_' + name] = rcfg.settings(c, 'LF2', 'G0001')

    # 3. re-run the short known answers through the reference CPU core (G0001 both profiles)
    gamma = 1.4
    known = dict(short_checks=[dict(case=c['case'], profile=c['profile'], cells=c['cells'], steps=c['steps'])
                               for c in ten['cases']],
                 controls={c['name']: c['steps'] for c in controls['cases']},
                 settings=settings,
                 full_steady={row['profile']: dict(cells=row['cells'], steps=row['steps'], t=row['physical_time_star'],
                                                   Cl=row['Cl'], Cd=row['Cd'], Cm=row['Cm'])
                              for row in summary['full_steady']},
                 reproduced={})
    for label in ('LF1', 'LF2'):
        s, boxes = parse_settings(settings['default_' + label])
        spec = SettingsSpec(s, boxes, label)
        i = names.index('G0001')
        rc = RefCase.build(spec, xs[i], ys[i], ps[i], gamma=gamma)
        u0 = rc.initial(spec.initial_primitive(gamma))
        out = rc.run(u0, 0.01, 50000000)
        assert out['status'] == 0, out['error']
        d = rc.diagnostics(out['u'])
        known['reproduced']['G0001_' + label] = dict(cells=rc.counts['n'], steps=out['steps'], time=out['time'],
                                                     rejected=out['rejected'], diagnostics=d.tolist())
        print(label, rc.counts['n'], out['steps'], out['time'])
    (GOLDEN / 'known_answers.json').write_text(json.dumps(known, indent=1) + '\n')

    # 4. single-case mesh inputs
    x, y, pt = airfoils.naca4(0.0, 0.4, 0.12)
    euler = cases.CaseSpec(naca=(0.0, 0.4, 0.12), profile='LF1', physics='euler', mach=1.65, aoa=1.5)
    RefCase.build(euler, x, y, pt).mesh().save(GOLDEN / 'mesh_naca0012_lf1_euler_srd.npz')
    x, y, pt = airfoils.naca4(0.02, 0.4, 0.12)
    sa = cases.CaseSpec(naca=(0.02, 0.4, 0.12), profile='LF2', physics='sa', mach=1.65, aoa=1.5)
    RefCase.build(sa, x, y, pt).mesh().save(GOLDEN / 'mesh_naca2412_lf2_sa.npz')
    sa1 = cases.CaseSpec(naca=(0.02, 0.4, 0.12), profile='LF1', physics='sa', mach=1.65, aoa=1.5)
    RefCase.build(sa1, x, y, pt).mesh().save(GOLDEN / 'mesh_naca2412_lf1_sa.npz')
    print('done')


if __name__ == '__main__':
    main()
