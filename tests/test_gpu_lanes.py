"""GPU tests of the split mode in lanes (amr_batch_set_lanes): the live cases run as independent
chains of kernels, one stream each.  Every case must end bit for bit where it ends in one lane, in
FP32 and FP64, with two and four lanes, also after a release and a new admission have reordered the
arena ranges."""
import numpy as np
import pytest

from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import _abi
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.batch import Batch
from tests.test_gpu_admit_many import items_of
from tests.test_gpu_launch_modes import MODES, sa_mix

pytestmark = pytest.mark.gpu


def run(items, precision, lanes, churn=False):
    b = Batch(precision=precision, model=_abi.MODEL_LAMINAR, sa=True, max_cases=len(items) + 1,
              max_cells=sum(m.n_cells for m, _, _, _ in items) * 2 + 1000, **MODES['split'])
    try:
        b.set_lanes(lanes)
        slots = b.admit_many(items)
        b.advance(8)
        if churn:  # an LF1 case leaves; an LF2 case, too large for its gap, goes above the others
            b.release(slots[0])
            slots[0] = b.admit(*items[1])
        for _ in range(3):
            b.advance(16)
        cfg = b.launch_config()
        return [b.download(s) for s in slots], [b.status(s)['steps'] for s in slots], cfg
    finally:
        b.destroy()


@pytest.mark.parametrize('precision,lanes', [(32, 2), (64, 2), (32, 4)])
def test_lanes_equal_one(precision, lanes):
    items = items_of(sa_mix() * 2, 48)  # six cases
    one, steps1, cfg1 = run(items, precision, 1)
    two, steps2, cfg2 = run(items, precision, lanes)
    assert 'lanes' not in cfg1 and f'lanes={lanes}' in cfg2, (cfg1, cfg2)
    assert steps1 == steps2
    for a, b in zip(one, two):
        assert np.array_equal(a, b)


def test_lanes_after_release_and_readmission():
    items = items_of(sa_mix() * 2, 60)
    one, steps1, _ = run(items, 32, 1, churn=True)
    two, steps2, _ = run(items, 32, 2, churn=True)
    assert steps1 == steps2
    for a, b in zip(one, two):
        assert np.array_equal(a, b)
