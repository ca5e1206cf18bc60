"""GPU tests of bulk admission (amr_batch_admit_many): cases converted on several host threads
land in the same slots and arena ranges as one-by-one admissions in request order, so the
batch computes bit for bit the same; an invalid or unplaceable entry is reported per entry
while the others are admitted."""
import numpy as np
import pytest

from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import _abi, cases
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.batch import Batch, BatchError, case_control
from tests.test_gpu_launch_modes import MODES, sa_mix

pytestmark = pytest.mark.gpu


def items_of(mix, nsteps):
    out = []
    for spec, mesh in mix:
        u0 = cases.initial_state(mesh, spec.initial_primitive())
        out.append((mesh, spec.params(), u0, case_control(1e30, nsteps, steady=False, mach=spec.mach, aoa=spec.aoa)))
    return out


def run(items, precision, mode, threads, max_cases, bulk):
    b = Batch(precision=precision, model=_abi.MODEL_LAMINAR, sa=True, max_cases=max_cases,
              max_cells=sum(m.n_cells for m, _, _, _ in items) + 1000, **MODES[mode])
    if bulk:
        slots = b.admit_many(items, threads=threads)
    else:
        slots = [b.admit(*it) for it in items]
    for _ in range(8):
        b.advance(16)
    states = [b.download(s) for s in slots]
    steps = [b.status(s)['steps'] for s in slots]
    b.destroy()
    return slots, states, steps


@pytest.mark.parametrize('precision,mode', [(32, 'split'), (64, 'tiled')])
def test_bulk_equals_sequential(precision, mode):
    mix = sa_mix()
    items = items_of(mix + mix[:2], 12)
    ref_slots, ref_states, ref_steps = run(items, precision, mode, 1, 8, bulk=False)
    for threads in (1, 4, 0):
        slots, states, steps = run(items, precision, mode, threads, 8, bulk=True)
        assert slots == ref_slots and steps == ref_steps, threads
        for a, b in zip(states, ref_states):
            assert np.array_equal(a, b), threads


def test_bulk_more_cases_than_a_chunk():
    """40 entries span two preparation chunks; slots follow the request order."""
    mix = sa_mix()
    items = items_of([mix[i % 3] for i in range(40)], 4)
    ref_slots, ref_states, _ = run(items, 32, 'split', 1, 40, bulk=False)
    slots, states, _ = run(items, 32, 'split', 6, 40, bulk=True)
    assert slots == ref_slots == list(range(40))
    for a, b in zip(states, ref_states):
        assert np.array_equal(a, b)


def test_bulk_reports_invalid_and_full_entries():
    mix = sa_mix()
    items = items_of(mix, 8)
    mesh, params, u0, ctl = items[1]
    bad = (mesh, params, u0[:-1], ctl)  # wrong state size
    b = Batch(precision=32, model=_abi.MODEL_LAMINAR, sa=True, max_cases=2,
              max_cells=sum(m.n_cells for _, m in mix) + 1000, **MODES['split'])
    with pytest.raises(BatchError) as e:
        b.admit_many([items[0], bad, items[2], items[1]], threads=3)
    assert 'case 1' in str(e.value) and 'initial state size mismatch' in str(e.value)
    assert e.value.slots == [0, None, 1, None]  # entry 3 found no free case slot
    b.advance(16)
    alone = run([items[2]], 32, 'split', 1, 2, bulk=False)[1][0]
    assert np.array_equal(b.download(1), alone)
    b.destroy()


def test_bulk_euler_srd_fp64_equals_sequential(golden):
    """Non-trivial SRD neighbourhoods (Euler, no agglomeration) prepared on several threads: the
    bulk admission computes bit for bit what one-by-one admissions compute."""
    from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.mesh import MeshArrays
    from tests.test_gpu_launch_modes import built
    mix = [(cases.CaseSpec(physics='euler', profile='LF1', mach=1.65, aoa=1.5),
            MeshArrays.load(golden / 'mesh_naca0012_lf1_euler_srd.npz'))]
    mix.append(built((0.02, 0.4, 0.12), profile='LF1', physics='euler', mach=1.8, aoa=3.0))
    assert all(m.small_cells for _, m in mix)
    items = items_of(mix + mix[:1], 20)
    out = []
    for bulk in (False, True):
        b = Batch(precision=64, model=_abi.MODEL_EULER, sa=False, max_cases=4,
                  max_cells=sum(m.n_cells for m, _, _, _ in items) + 100, **MODES['split'])
        slots = b.admit_many(items, threads=3) if bulk else [b.admit(*it) for it in items]
        for _ in range(2):
            b.advance(16)
        out.append((slots, [b.status(s)['steps'] for s in slots], [b.download(s) for s in slots]))
        b.destroy()
    assert out[0][0] == out[1][0] and out[0][1] == out[1][1] == [20] * 3
    for a, c in zip(out[0][2], out[1][2]):
        assert np.array_equal(a, c)


def test_bulk_no_room_by_cells_and_readmit_into_freed_ranges():
    """A batch with cells for two of three cases: the third entry finds no room (3) while the
    others are admitted; after a release, a bulk re-admission reuses the freed ranges and computes
    exactly what the case computes alone.  An empty request list admits nothing."""
    mix = sa_mix()
    items = items_of(mix, 8)
    cells = sorted(m.n_cells for m, _, _, _ in items)
    b = Batch(precision=32, model=_abi.MODEL_LAMINAR, sa=True, max_cases=4,
              max_cells=cells[1] + cells[2] + 8, **MODES['split'])
    assert b.admit_many([]) == []
    big_two = sorted(range(3), key=lambda i: items[i][0].n_cells)[1:]
    small = min(range(3), key=lambda i: items[i][0].n_cells)
    first = b.admit_many([items[i] for i in big_two] + [items[small]], threads=2)
    assert first[:2] == [0, 1] and first[2] is None
    b.release(first[0])
    again = b.admit_many([items[small]], threads=2)
    assert again == [0]
    for _ in range(2):
        b.advance(16)
    alone = run([items[small]], 32, 'split', 1, 1, bulk=False)[1][0]
    assert np.array_equal(b.download(0), alone)
    b.destroy()


@pytest.mark.parametrize('precision,mode', [(32, 'split'), (64, 'phases')])
def test_uniform_start_filled_on_device_equals_staged_start(precision, mode):
    """A start given as the nv conserved values (filled on the device, leading and trailing words)
    runs bit for bit like the same state staged cell by cell, alone and in bulk admission."""
    mix = sa_mix()
    staged = items_of(mix, 12)
    uniform = [(mesh, spec.params(), cases.uniform_state(mesh, spec.initial_primitive()),
                case_control(1e30, 12, steady=False, mach=spec.mach, aoa=spec.aoa)) for spec, mesh in mix]
    ref_slots, ref_states, ref_steps = run(staged, precision, mode, 1, 4, bulk=False)
    for bulk in (False, True):
        slots, states, steps = run(uniform, precision, mode, 4, 4, bulk=bulk)
        assert slots == ref_slots and steps == ref_steps
        for a, b in zip(states, ref_states):
            assert np.array_equal(a, b), bulk


def test_download_many_equals_per_case_downloads():
    """The bulk download returns every case's state exactly as one download per case does (both
    FP32 words summed)."""
    mix = sa_mix()
    items = items_of(mix + mix[:1], 10)
    b = Batch(precision=32, model=_abi.MODEL_LAMINAR, sa=True, max_cases=4,
              max_cells=sum(m.n_cells for m, _, _, _ in items) + 1000, **MODES['split'])
    slots = b.admit_many(items)
    for _ in range(2):
        b.advance(8)
    bulk = b.download_many(slots[::-1])
    for s, u in zip(slots[::-1], bulk):
        assert np.array_equal(u, b.download(s))
    b.destroy()


def test_face_listing_error_found_in_fill_releases_the_case():
    """A mesh whose cell lists a face of another cell (indices in range) is refused while its
    tables are filled, after its slot was reserved: the entry reports the error, its slot and
    ranges are released, and a valid case admitted next computes bit for bit as alone."""
    import dataclasses
    mix = sa_mix()
    items = items_of(mix, 8)
    mesh, params, u0, ctl = items[0]
    cf = mesh.cell_faces.copy()
    cf[int(mesh.face_offsets[0])] = cf[int(mesh.face_offsets[-2])]  # cell 0 lists the last cell's face
    bad = (dataclasses.replace(mesh, cell_faces=cf), params, u0, ctl)
    b = Batch(precision=32, model=_abi.MODEL_LAMINAR, sa=True, max_cases=1,
              max_cells=max(m.n_cells for _, m in mix) + 1000, **MODES['split'])
    with pytest.raises(BatchError, match='lists a face of another cell'):
        b.admit_many([bad])
    with pytest.raises(BatchError, match='lists a face of another cell'):
        b.admit(*bad)
    slot = b.admit(*items[2])
    assert slot == 0
    b.advance(16)
    alone = run([items[2]], 32, 'split', 1, 2, bulk=False)[1][0]
    assert np.array_equal(b.download(slot), alone)
    b.destroy()
