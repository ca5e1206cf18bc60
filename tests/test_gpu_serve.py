"""GPU test of the serving loop on the real engine: natively built meshes, admission while the
arena has room or into new arenas while the device has free memory, device steady-rule retirement
and the step cap; a served case must end bit for bit where the same case run alone in a batch
ends, also when it shared the device with other requests."""
import numpy as np
import pytest

from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import _abi, cases, serve
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.batch import Batch, case_control

pytestmark = pytest.mark.gpu


def test_capped_and_converged_requests():
    reqs = serve.poisson_requests(6, rate=200.0, seed=11)
    # a steady rule loose enough to hold within a few checks (check every 0.004 time units)
    loose = dict(first_check=0.002, check_period=0.004, min_time=0.0, raw_tol=1e9, load_tol=1e9, hold=2)
    batch = Batch(precision=32, model=_abi.MODEL_LAMINAR, sa=True, max_cases=3, max_cells=3 * 9800,
                  launch_mode=_abi.LAUNCH_SPLIT, block_threads=128)
    server = serve.Server(batch, max_steps=400, trials=16, builder_threads=4, steady=loose)
    results = server.run(reqs)
    assert all(r.outcome == 'converged' for r in results), [(r.outcome, r.error) for r in results]
    for r in results:
        assert 0 < r.steps < 400 and r.latency > 0 and np.isfinite(r.cl) and np.isfinite(r.cd)
    # at most three cases fit: some admissions had to wait for a retirement
    assert max(r.admitted for r in results) > min(r.finished for r in results)

    capped_batch = Batch(precision=32, model=_abi.MODEL_LAMINAR, sa=True, max_cases=8, max_cells=8 * 9800,
                         launch_mode=_abi.LAUNCH_SPLIT, block_threads=128)
    capped = serve.Server(capped_batch, max_steps=96, trials=32, builder_threads=4).run(reqs[:4])
    assert [r.outcome for r in capped] == ['capped'] * 4 and all(r.steps == 96 for r in capped)
    s = serve.summarize(capped, 1.0)
    assert s['outcomes'] == {'capped': 4}


def test_served_case_matches_a_lone_batch_run():
    req = serve.poisson_requests(1, rate=100.0, seed=5)[0]
    mesh = serve.build_request_mesh(req)
    batch = Batch(precision=32, model=_abi.MODEL_LAMINAR, sa=True, max_cases=2, max_cells=2 * 9800,
                  launch_mode=_abi.LAUNCH_SPLIT, block_threads=128)
    server = serve.Server(batch, max_steps=64, trials=32)
    res = server.run([req])[0]
    assert res.outcome == 'capped' and res.steps == 64

    lone = Batch(precision=32, model=_abi.MODEL_LAMINAR, sa=True, max_cases=1, max_cells=9800,
                 launch_mode=_abi.LAUNCH_SPLIT, block_threads=128)
    u0 = cases.initial_state(mesh, req.spec.initial_primitive())
    slot = lone.admit(mesh, req.spec.params(), u0, case_control(1e30, 64, steady=True, mach=req.spec.mach,
                                                                 aoa=req.spec.aoa))
    for _ in range(4):
        lone.advance(32)
        lone.check()
    st = lone.status(slot)
    assert st['status'] == _abi.STATUS_MAXSTEPS and st['steps'] == 64
    assert (st['cl'], st['cd'], st['cm']) == (res.cl, res.cd, res.cm)


def lone_run(req, mesh, max_steps, trials=32):
    """The request alone in its own batch, polled and checked as the server does."""
    lone = Batch(precision=32, model=_abi.MODEL_LAMINAR, sa=True, max_cases=1, max_cells=mesh.n_cells + 64,
                 launch_mode=_abi.LAUNCH_SPLIT, block_threads=128)
    u0 = cases.initial_state(mesh, req.spec.initial_primitive())
    slot = lone.admit(mesh, req.spec.params(), u0, case_control(1e30, max_steps, steady=True, mach=req.spec.mach,
                                                                 aoa=req.spec.aoa))
    while True:
        lone.advance(trials)
        lone.check()
        st = lone.status(slot)
        if st['finished'] or st['status']:
            break
    u = lone.download(slot)
    lone.destroy()
    return st, u


def test_overlapping_requests_each_equal_alone():
    """Four requests 20 ms apart, two per arena (so a second arena opens by free device memory and
    both arenas' trials are in flight together); later requests are admitted while earlier ones run.
    Each served case's final state and loads equal its lone run bit for bit."""
    reqs = serve.poisson_requests(4, rate=50.0, seed=7)
    make = lambda: Batch(precision=32, model=_abi.MODEL_LAMINAR, sa=True, max_cases=2, max_cells=2 * 9800,
                         launch_mode=_abi.LAUNCH_SPLIT, block_threads=128)
    server = serve.Server(make, max_steps=3000, trials=32, builder_threads=4, keep_states=True)
    results = server.run(reqs)
    assert all(r.outcome == 'capped' and r.steps == 3000 for r in results), [(r.outcome, r.steps) for r in results]
    assert server.peak_arenas == 2 and len(server.arenas) == 1
    first_done = min(r.finished for r in results)
    assert sum(1 for r in results if r.admitted < first_done) >= 3  # at least three on the device together
    for req, res in zip(reqs, results):
        st, u = lone_run(req, serve.build_request_mesh(req), 3000)
        assert st['steps'] == res.steps and (st['cl'], st['cd'], st['cm']) == (res.cl, res.cd, res.cm)
        assert np.array_equal(u, res.u), req.id
