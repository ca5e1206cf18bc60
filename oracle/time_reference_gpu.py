"""TEST INFRASTRUCTURE: times the reference's CUDA session (src/static_amr2d_cuda.cu, compiled for
sm_100a by `make -C oracle ref_cuda`) beside this engine's FP64 session on the same meshes.

    python oracle/time_reference_gpu.py [--steps 256]

Prints one JSON line per mesh with microseconds per step of both (CUDA-event time, after warm-up).
The reference session runs with its driver's settings (fused kernels, fused SA, graphs, 32 trials
per poll)."""
import argparse
import json
import pathlib
import sys

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200 import cases  # noqa: E402
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.mesh import MeshArrays  # noqa: E402
from quick_gpu_cfd_for_neural_network_with_converging_inputs_airfoil2d_version_b200.session import StaticAmrGpu  # noqa: E402
from oracle.oracle import RefCase, RefGpu  # noqa: E402

GOLDEN = ROOT / 'tests' / 'golden'


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--steps', type=int, default=256)
    args = ap.parse_args()
    runs = [('naca0012 LF1 euler+srd', 'mesh_naca0012_lf1_euler_srd.npz', cases.CaseSpec(physics='euler', profile='LF1')),
            ('naca2412 LF1 sa', 'mesh_naca2412_lf1_sa.npz', cases.CaseSpec(physics='sa', profile='LF1')),
            ('naca2412 LF2 sa', 'mesh_naca2412_lf2_sa.npz', cases.CaseSpec(physics='sa', profile='LF2'))]
    for name, fname, spec in runs:
        mesh = MeshArrays.load(GOLDEN / fname)
        params = spec.params()
        u0 = cases.initial_state(mesh, spec.initial_primitive())
        rc = RefCase.from_mesh(mesh, params, kind='cuda')
        ref = RefGpu(rc, u0, batch_trials=32, graph=True, fused=True, sa_fused=True, event_timing=True)
        ref.advance(1e30, 64)                     # warm-up (maxsteps is fatal and sticky)
        ref = RefGpu(rc, u0, batch_trials=32, graph=True, fused=True, sa_fused=True, event_timing=True)
        out = ref.advance(1e30, args.steps)
        ref_us = 1e6 * ref.event_seconds() / out['steps']
        u_ref = ref.download()
        ours = StaticAmrGpu.create(mesh, params, u0)
        ours.advance(1e30, args.steps)
        st = ours.stats()
        ours_us = 1e6 * st['advance_event_seconds'] / ours.steps
        u = ours.download()
        import numpy as np
        diff = max(np.abs(u.reshape(mesh.nv, -1)[v] - u_ref.reshape(mesh.nv, -1)[v]).max() /
                   np.abs(u_ref.reshape(mesh.nv, -1)[v]).max() for v in range(mesh.nv))
        print(json.dumps(dict(mesh=name, cells=mesh.n_cells, steps=args.steps, reference_us_per_step=ref_us,
                              reference_graph_nodes=ref.graph_nodes(), ours_us_per_step=ours_us,
                              ours_launch=ours.launch_config(), speedup=ref_us / ours_us,
                              state_rel_diff_vs_reference_gpu=diff)), flush=True)


if __name__ == '__main__':
    main()
