"""GPU tests of amr_batch_group_advance: several batches of one device advanced with their work in
flight together end bit for bit where each ends when advanced alone, the group reports its device
time, and a group naming one batch twice (or no batch) is refused with a message."""
import numpy as np
import pytest

from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import _abi
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.batch import (Batch, BatchError,
                                                                                                  group_advance)
from tests.test_gpu_admit_many import items_of
from tests.test_gpu_launch_modes import MODES, sa_mix

pytestmark = pytest.mark.gpu


def make(items, precision):
    b = Batch(precision=precision, model=_abi.MODEL_LAMINAR, sa=True, max_cases=len(items),
              max_cells=sum(m.n_cells for m, _, _, _ in items) + 1000, **MODES['split'])
    return b, b.admit_many(items)


def finish(b, slots):
    out = [(b.download(s), b.status(s)['steps'], b.status(s)['time']) for s in slots]
    b.destroy()
    return out


@pytest.mark.parametrize('precision', [32, 64])
def test_group_equals_alone(precision):
    mix = sa_mix()
    groups = [items_of(mix[:1], 40), items_of(mix[1:], 40)]
    alone = []
    for g in groups:
        b, slots = make(g, precision)
        for _ in range(3):
            b.advance(16)
        alone.append(finish(b, slots))
    made = [make(g, precision) for g in groups]
    seconds = [group_advance([b for b, _ in made], 16) for _ in range(3)]
    assert all(s > 0 for s in seconds), seconds
    together = [finish(b, slots) for b, slots in made]
    for a_batch, t_batch in zip(alone, together):
        for (ua, sa, ta), (ut, st, tt) in zip(a_batch, t_batch):
            assert sa == st == 40 and ta == tt
            assert np.array_equal(ua, ut)


def test_group_refuses_repeated_or_no_batch():
    mix = sa_mix()
    b, _ = make(items_of(mix[:1], 10), 32)
    try:
        with pytest.raises(BatchError, match='twice'):
            group_advance([b, b], 4)
        with pytest.raises(BatchError, match='no batches'):
            group_advance([], 4)
        assert group_advance([b], 4) > 0  # a group of one is a plain advance
    finally:
        b.destroy()
