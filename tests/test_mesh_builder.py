"""CPU tests of the native host mesh builder (amr_mesh_build / amr_mesh_build_many).

Pins: the reference's own validation cell counts for its ten example airfoils on both mesh
profiles (validation/ten_short_checks.json, carried in known_answers.json), and table-for-table
equality with the reference builder compiled from its sources (oracle/_ref): every field of
every cell, face, wall, CSR, SRD, gradient-term, donor, face-geometry and wall-distance record,
compared field by field (struct padding excluded), must be bit-identical.  Failing builds must
fail with the reference's message."""
import json

import numpy as np
import pytest

from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import airfoils, builder, cases
from tests.golden.make_golden import SettingsSpec, parse_settings


def example(golden, name):
    z = np.load(golden / 'examples.npz')
    names = list(z['names'])
    i = names.index(name)
    a, b = z['offsets'][i], z['offsets'][i + 1]
    return z['x'][a:b], z['y'][a:b], z['patches'][a:b]


def identical(ours, ref):
    """Field-by-field bit equality of two MeshArrays; returns the first differing table or None."""
    for k in ours._ARRAYS:
        a, b = getattr(ours, k), getattr(ref, k)
        if a is None and b is None:
            continue
        if a is None or b is None or a.shape != b.shape:
            return k
        fields = a.dtype.names or [None]
        for f in fields:
            x, y = (a, b) if f is None else (a[f], b[f])
            if x.tobytes() != y.tobytes():
                return k if f is None else f'{k}.{f}'
    if (ours.small_cells, ours.agglomerate_small) != (ref.small_cells, ref.agglomerate_small):
        return 'scalars'
    return None


def reference_mesh(spec, x, y, pt):
    from oracle.oracle import RefCase
    return RefCase.build(spec, x, y, pt).mesh()


def test_ten_examples_cell_counts_match_reference_validation(golden):
    """Cells of every example airfoil on LF1 and LF2 with the reference pipeline's settings."""
    ka = json.loads((golden / 'known_answers.json').read_text())
    items, expect = [], []
    for check in ka['short_checks']:
        s, boxes = parse_settings(ka['settings']['default_' + check['profile']])
        spec = SettingsSpec(s, boxes, check['profile'])
        x, y, pt = example(golden, check['case'])
        items.append((spec, x, y, pt))
        expect.append(check['cells'])
    meshes = builder.build_meshes(items, threads=0)
    assert [m.n_cells for m in meshes] == expect


@pytest.mark.parametrize('physics', ['euler', 'laminar', 'sa'])
@pytest.mark.parametrize('profile', ['LF1', 'LF2'])
def test_bit_identical_to_reference_builder_naca(physics, profile):
    rng = np.random.default_rng(20261203 + len(physics) + 7 * len(profile))
    for naca in [(0.02, 0.4, 0.12), airfoils.seeded_naca(rng)]:
        kinds = ('farfield', 'pressure-outlet', 'farfield', 'farfield') if physics == 'laminar' else ('farfield',) * 4
        spec = cases.CaseSpec(naca=naca, profile=profile, physics=physics, kinds=kinds)
        x, y, pt = airfoils.naca4(*naca)
        try:
            ref = reference_mesh(spec, x, y, pt)
        except RuntimeError as e:  # the draw fails in the reference: ours must fail the same way
            with pytest.raises(builder.MeshBuildError) as err:
                builder.build_mesh(spec, x, y, pt)
            assert str(err.value) in str(e)
            continue
        ours = builder.build_mesh(spec, x, y, pt)
        assert identical(ours, ref) is None, (naca, identical(ours, ref))


def test_bit_identical_examples_and_variants(golden):
    ka = json.loads((golden / 'known_answers.json').read_text())
    s, boxes = parse_settings(ka['settings']['default_LF1'])
    for name in ('G0001', 'G0100', 'G0300', 'G0490'):
        x, y, pt = example(golden, name)
        spec = SettingsSpec(s, boxes, 'LF1')
        assert identical(builder.build_mesh(spec, x, y, pt), reference_mesh(spec, x, y, pt)) is None, name
    # agglomerated Euler with AUSM+-up, and a laminar case with no-slip exterior walls
    x, y, pt = airfoils.naca4(0.0, 0.4, 0.09)
    spec = cases.CaseSpec(naca=(0.0, .4, .09), profile='LF1', physics='euler', flux='ausm', agglomerate=True)
    assert identical(builder.build_mesh(spec, x, y, pt), reference_mesh(spec, x, y, pt)) is None
    spec = cases.CaseSpec(naca=(0.0, .4, .09), profile='LF1', physics='laminar', agglomerate=True,
                          kinds=('farfield', 'transmissive', 'no-slip', 'no-slip'))
    assert identical(builder.build_mesh(spec, x, y, pt), reference_mesh(spec, x, y, pt)) is None


def test_threaded_builds_equal_serial_builds():
    rng = np.random.default_rng(5)
    items = []
    for i in range(8):
        naca = airfoils.seeded_naca(rng)
        spec = cases.CaseSpec(naca=naca, profile='LF1' if i % 2 else 'LF2', physics='sa')
        x, y, pt = airfoils.naca4(*naca)
        items.append((spec, x, y, pt))
    many = builder.build_meshes(items, threads=4, raise_on_error=False)
    for (spec, x, y, pt), m in zip(items, many):
        if m is None:
            with pytest.raises(builder.MeshBuildError):
                builder.build_mesh(spec, x, y, pt)
            continue
        assert identical(m, builder.build_mesh(spec, x, y, pt)) is None


def test_invalid_requests_fail_with_reference_messages():
    x, y, pt = airfoils.naca4(0.02, 0.4, 0.12)
    spec = cases.CaseSpec(naca=(0.02, .4, .12), profile='LF1', physics='euler')
    bad = cases.CaseSpec(naca=(0.02, .4, .12), profile='LF1', physics='euler')
    bad.options = lambda: dict(spec.options(), buffer=1)
    with pytest.raises(builder.MeshBuildError, match='invalid mesh options or polygon arrays'):
        builder.build_mesh(bad, x, y, pt)
    with pytest.raises(builder.MeshBuildError, match='invalid polygon vertex or patch'):
        builder.build_mesh(spec, np.r_[x, x[:1]], np.r_[y, y[:1]], np.r_[pt, pt[:1]])
    with pytest.raises(builder.MeshBuildError, match='three finest cells of domain clearance'):
        builder.build_mesh(spec, x * 40, y, pt)
    small = cases.CaseSpec(naca=(0.02, .4, .12), profile='LF1', physics='euler')
    small.options = lambda: dict(spec.options(), max_cells=1000)
    with pytest.raises(builder.MeshBuildError, match='max-cells exceeded'):
        builder.build_mesh(small, x, y, pt)
    box = cases.CaseSpec(naca=(0.02, .4, .12), profile='LF1', physics='euler')
    box.options = lambda: dict(spec.options(), boxes=[[0.0, -1.0, 0.0, 1.0, 2]])
    with pytest.raises(builder.MeshBuildError, match='invalid refinement box'):
        builder.build_mesh(box, x, y, pt)
    sa_srd = cases.CaseSpec(naca=(0.02, .4, .12), profile='LF1', physics='sa', agglomerate=False)
    with pytest.raises(builder.MeshBuildError, match='SA-neg requires agglomerated true-volume mesh without SRD'):
        builder.build_mesh(sa_srd, x, y, pt)
