"""Seeded synthetic workloads of the batched, time-accurate and served forms.

Every airfoil is a NACA 4-digit section (airfoils.naca4: 201 cosine-spaced points with the
closing trailing-edge vertex dropped) on the reference's LF1/LF2 mesh profiles, built by the
native host builder (builder.build_meshes, bit-identical tables to the reference builder's
static_amr2d_build + static_amr2d_prepare_viscous).  Shapes and flow conditions come from one
NumPy PCG64 stream per workload seed; a draw the mesh builder rejects is replaced by the next
draw of the same stream and counted in `redraws`, so a workload depends on its seed alone.

    batched_sa(256)          256 SA-neg/Sutherland HLLC cases, LF1:LF2 1:1, M~U[1.2,2.0], AoA~U[-3,5]
    time_accurate_laminar(128)  128 LF2 laminar constant-viscosity AUSM+-up cases with a pressure
                             outlet (1.0x freestream p) on xmax, M~U[1.2,1.8], AoA~U[-3,5]
    naca2412_lf2_sa()        the single LF2 NACA 2412 SA case (M 1.65, AoA 1.5)
"""
import dataclasses

import numpy as np

from . import airfoils, builder, cases

SEED = 20261203


@dataclasses.dataclass
class Workload:
    name: str
    items: list            # [(CaseSpec, MeshArrays)]
    seed: int
    redraws: int = 0

    @property
    def cells(self):
        return sum(m.n_cells for _, m in self.items)

    def describe(self):
        prof = {}
        for spec, mesh in self.items:
            p = prof.setdefault(spec.profile, [0, 0])
            p[0] += 1
            p[1] += mesh.n_cells
        return dict(workload=self.name, cases=len(self.items), cells=self.cells, seed=self.seed, redraws=self.redraws,
                    profiles={k: dict(cases=v[0], mean_cells=v[1] / v[0]) for k, v in sorted(prof.items())})


def _draws(n, seed, make_spec, threads=0):
    """n specs with built meshes from one seeded stream; rejected draws are replaced in order."""
    rng = np.random.default_rng(seed)
    specs = [make_spec(i, rng) for i in range(n)]
    redraws = 0
    meshes = [None] * n
    todo = list(range(n))
    while todo:
        items = []
        for i in todo:
            x, y, pt = airfoils.naca4(*specs[i].naca)
            items.append((specs[i], x, y, pt))
        built = builder.build_meshes(items, threads=threads, raise_on_error=False)
        failed = []
        for i, m in zip(todo, built):
            if m is None:
                failed.append(i)
            else:
                meshes[i] = m
        for i in failed:  # the next draws of the stream replace rejected ones, in case order
            specs[i] = make_spec(i, rng)
            redraws += 1
        todo = failed
        if redraws > 10 * n + 10:
            raise RuntimeError('too many rejected draws')
    return list(zip(specs, meshes)), redraws


def _batched_sa_spec(i, rng):
    naca = airfoils.seeded_naca(rng)
    return cases.CaseSpec(naca=naca, profile='LF1' if i % 2 == 0 else 'LF2', physics='sa',
                          mach=float(rng.uniform(1.2, 2.0)), aoa=float(rng.uniform(-3.0, 5.0)))


def batched_sa(ncases=256, seed=SEED, threads=0):
    """SA-neg with Sutherland viscosity, HLLC, no-slip airfoil, characteristic farfield on every
    side; LF1 and LF2 alternate (1:1); NACA m~U[0,0.06], p~U[0.2,0.6], t~U[0.08,0.15]."""
    items, redraws = _draws(ncases, seed, _batched_sa_spec, threads)
    return Workload('batched-sa-fp32-%d' % ncases, items, seed, redraws)


def batched_sa_specs(ncases, seed=SEED):
    """The first ncases draws of batched_sa's stream, without building meshes (equal to the first
    cases of batched_sa(n, seed) for any n >= ncases whose builds of those draws succeed)."""
    rng = np.random.default_rng(seed)
    return [_batched_sa_spec(i, rng) for i in range(ncases)]


def time_accurate_laminar(ncases=128, seed=SEED + 4, threads=0, profile='LF2'):
    """Laminar with constant viscosity (the Sutherland value at the freestream temperature),
    AUSM+-up, pressure outlet at 1.0x the freestream pressure on xmax and characteristic
    farfield on the other sides, M~U[1.2,1.8], AoA~U[-3,5]; all cases on LF2."""

    def make(i, rng):
        naca = airfoils.seeded_naca(rng)
        return cases.CaseSpec(naca=naca, profile=profile, physics='laminar', law='constant', flux='ausm',
                              kinds=('farfield', 'pressure-outlet', 'farfield', 'farfield'),
                              mach=float(rng.uniform(1.2, 1.8)), aoa=float(rng.uniform(-3.0, 5.0)))

    items, redraws = _draws(ncases, seed, make, threads)
    return Workload('time-accurate-laminar-ausm-%d' % ncases, items, seed, redraws)


def naca2412_lf2_sa():
    """The single-case accuracy workload: NACA 2412 on LF2, SA-neg with Sutherland, HLLC, M 1.65,
    AoA 1.5 deg, farfield on every side."""
    spec = cases.CaseSpec(naca=(0.02, 0.4, 0.12), profile='LF2', physics='sa', mach=1.65, aoa=1.5)
    x, y, pt = airfoils.naca4(*spec.naca)
    return Workload('naca2412-lf2-sa', [(spec, builder.build_mesh(spec, x, y, pt))], 0, 0)


def batch_kwargs(items):
    """Batch() keyword arguments for a list of (spec, mesh) of one physics."""
    from . import _abi
    spec0 = items[0][0]
    model = _abi.MODEL_EULER if spec0.physics == 'euler' else _abi.MODEL_LAMINAR
    flux = _abi.FLUX_HLLC if spec0.flux == 'hllc' else _abi.FLUX_AUSMPUP
    return dict(model=model, sa=spec0.physics == 'sa', flux=flux, max_cases=len(items),
                max_cells=sum(m.n_cells for _, m in items) + 64)
