"""GPU test of the page-locked staging pool: admissions and downloads of every batch in a process
borrow their page-locked staging from one shared pool for the length of the call.  Two batches
driven from two host threads at once (bulk admission, advances, bulk and single downloads) must
end bit for bit where each ends when run alone."""
import threading

import numpy as np
import pytest

from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import _abi
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.batch import Batch
from tests.test_gpu_admit_many import items_of
from tests.test_gpu_launch_modes import MODES, sa_mix

pytestmark = pytest.mark.gpu


def run(items, rounds=3):
    b = Batch(precision=32, model=_abi.MODEL_LAMINAR, sa=True, max_cases=len(items),
              max_cells=sum(m.n_cells for m, _, _, _ in items) + 1000, **MODES['split'])
    try:
        slots = b.admit_many(items, threads=2)
        for _ in range(rounds):
            b.advance(16)
            bulk = b.download_many(slots)
        single = [b.download(s) for s in slots]
        return bulk, single
    finally:
        b.destroy()


def test_two_batches_on_two_threads_equal_alone():
    mix = sa_mix()
    half = len(mix) // 2
    groups = [items_of(mix[:half], 48), items_of(mix[half:], 48)]
    alone = [run(g) for g in groups]
    together = [None, None]
    errors = []

    def worker(i):
        try:
            together[i] = run(groups[i])
        except Exception as e:  # reported below, on the test's thread
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(i,)) for i in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for (bulk_a, single_a), (bulk_t, single_t) in zip(alone, together):
        for x, y in zip(bulk_a + single_a, bulk_t + single_t):
            assert np.array_equal(x, y)
        for x, y in zip(bulk_t, single_t):  # bulk and single downloads agree
            assert np.array_equal(x, y)
