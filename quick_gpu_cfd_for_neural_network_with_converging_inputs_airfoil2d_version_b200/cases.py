"""Case presets: mesh profiles, freestream scaling and boundary/transport records.

Mesh profiles LF1/LF2 and the default freestream are the reference's defaults
(config/default.json:2-60, 76-134).  Nondimensional scales follow the reference pipeline
(pipeline/configuration.py:129-167): density, speed of sound and chord are the units, so the
freestream is rho=1, (u,v)=M(cos a, sin a), p=1/gamma; the Sutherland reference temperature
is 1/gamma; viscosity is scaled by rho a c.  Boundary records are set as the reference driver
sets them (src/quick_airfoil.cpp:159-162).
"""
import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi

DOMAIN = dict(xmin=-7.0, xmax=14.0, ymin=-10.0, ymax=10.0, nx=42, ny=40, buffer=4, max_cells=2000000)
PROFILES = {
    'LF1': dict(levels=5, boxes=[[-0.5, 2.0, -0.75, 0.75, 3], [1.0, 4.0, -0.35, 0.65, 3], [-2.0, 6.0, -3.0, 3.0, 1]]),
    'LF2': dict(levels=6, boxes=[[-0.5, 2.0, -0.75, 0.75, 4], [1.0, 4.0, -0.35, 0.65, 3], [-2.0, 6.0, -3.0, 3.0, 1],
                                 [2.0, 3.25, -0.35, 0.65, 4]]),
}
STEADY = dict(first_check=0.01, check_period=0.5, min_time=3.0, raw_tol=1e-3, load_tol=0.005, hold=5,
              region=(-1.0, 3.0, -1.0, 1.0), moment_x=0.25, moment_y=0.0)


def scales(p_pa=18754.0, T=216.65, gamma=1.4, R=287.05, chord=1.0, mu0=1.716e-05, T0=273.15, S=110.4,
           viscosity='sutherland', constant_mu=None):
    rho = p_pa / (R * T)
    a = math.sqrt(gamma * R * T)
    mu = mu0 * (T / T0) ** 1.5 * (T0 + S) / (T + S)
    if viscosity == 'constant' and constant_mu is not None:
        mu = constant_mu
    return dict(rho=rho, velocity=a, length=chord, pressure=rho * a * a, temperature=gamma * T,
                time=chord / a, viscosity=rho * a * chord, mu_inf=mu, S=S)


def nondimensional(gamma=1.4, nu_ratio=3.0, outlet_p_pa=18754.0, **kw):
    s = scales(gamma=gamma, **kw)
    mu_star = s['mu_inf'] / s['viscosity']
    return dict(mu_star=mu_star, sutherland_star=s['S'] / s['temperature'], temperature_ref=1.0 / gamma,
                sa_nu_inf=nu_ratio * mu_star, outlet_p_star=outlet_p_pa / s['pressure'])


def freestream(mach, aoa_degrees, gamma=1.4):
    a = aoa_degrees * math.acos(-1.0) / 180
    return np.array([1.0, mach * math.cos(a), mach * math.sin(a), 1.0 / gamma])


def boundaries(mach, aoa_degrees, gamma=1.4, kinds=('farfield',) * 4, outlet_pressure=None):
    names = {'farfield': _abi.BC_FARFIELD, 'pressure-outlet': _abi.BC_PRESSURE_OUTLET,
             'transmissive': _abi.BC_TRANSMISSIVE, 'reflect': _abi.BC_REFLECT, 'no-slip': _abi.BC_NOSLIP,
             'total-inlet': _abi.BC_TOTAL_INLET}
    b = np.zeros(4, dtype=_abi.BOUNDARY_DTYPE)
    ref = freestream(mach, aoa_degrees, gamma)
    for side in range(4):
        b[side]['kind'] = names[kinds[side]]
        b[side]['reference'] = ref
        b[side]['gas_constant'] = 1.0
        b[side]['direction'] = (1.0, 0.0)
        b[side]['outlet_pressure'] = outlet_pressure if outlet_pressure is not None else 1.0 / gamma
    return b


def transport(model='euler', sa=False, law='sutherland', mu=None, sutherland=None, gamma=1.4,
              viscous_cfl=0.1, sa_cfl=0.1, sa_nu_inf=None, wall_probe_min_h=0.25):
    t = np.zeros(1, dtype=_abi.TRANSPORT_DTYPE)
    t['gas_constant'] = 1.0
    t['temperature_ref'] = 1.0
    t['viscous_cfl'] = 0.1
    t['sa_cfl'] = 0.1
    if model == 'euler':
        t['model'] = _abi.MODEL_EULER
        return t
    nd = nondimensional(gamma=gamma)
    t['model'] = _abi.MODEL_LAMINAR
    t['mu_ref'] = nd['mu_star'] if mu is None else mu
    if law == 'sutherland':
        t['law'] = _abi.MU_SUTHERLAND
        t['temperature_ref'] = 1.0 / gamma
        t['sutherland'] = nd['sutherland_star'] if sutherland is None else sutherland
    else:
        t['law'] = _abi.MU_CONSTANT
    t['viscous_cfl'] = viscous_cfl
    t['sa_cfl'] = sa_cfl
    t['sa_model'] = 1 if sa else 0
    t['sa_nu_inf'] = (nd['sa_nu_inf'] if sa_nu_inf is None else sa_nu_inf) if sa else 0.0
    t['wall_probe_min_h'] = wall_probe_min_h
    t['stabilization'] = _abi.VISCOUS_VOLUME
    return t


def params(gamma=1.4, cfl=0.15, flux='hllc', dt_fixed=0.0, mco=1.0):
    p = _abi.Params()
    p.gamma, p.cfl, p.dt_fixed, p.ausm_mco = gamma, cfl, dt_fixed, mco
    p.flux = _abi.FLUX_HLLC if flux == 'hllc' else _abi.FLUX_AUSMPUP
    p.limiter = _abi.LIMITER_FIRST_ORDER
    p.time_integrator = _abi.TIME_SSP_RK3
    for i in range(4):
        p.bc[i] = _abi.BC_TRANSMISSIVE
    return p


def mesh_options(profile, agglomerate):
    o = dict(DOMAIN)
    o.update(levels=PROFILES[profile]['levels'], boxes=[list(b) for b in PROFILES[profile]['boxes']],
             agglomerate_small=1 if agglomerate else 0, profile=profile)
    return o


@dataclass
class CaseSpec:
    """One solve: airfoil, mesh profile and physics."""
    naca: tuple = (0.0, 0.4, 0.12)
    profile: str = 'LF1'
    mach: float = 1.65
    aoa: float = 1.5
    physics: str = 'sa'            # 'euler' | 'laminar' | 'sa'
    law: str = 'sutherland'        # laminar/sa viscosity law
    flux: str = 'hllc'
    cfl: float = 0.15
    viscous_cfl: float = 0.1
    sa_cfl: float = 0.1
    agglomerate: bool = None       # default: True unless Euler
    kinds: tuple = ('farfield',) * 4
    dt_fixed: float = 0.0
    extra: dict = field(default_factory=dict)

    def agglomerated(self):
        return self.physics != 'euler' if self.agglomerate is None else bool(self.agglomerate)

    def options(self):
        return mesh_options(self.profile, self.agglomerated())

    def boundary_records(self, gamma=1.4):
        nd = nondimensional(gamma=gamma)
        return boundaries(self.mach, self.aoa, gamma, self.kinds, nd['outlet_p_star'])

    def transport_record(self, gamma=1.4):
        if self.physics == 'euler':
            return transport('euler')
        return transport('laminar', sa=self.physics == 'sa', law=self.law, gamma=gamma,
                         viscous_cfl=self.viscous_cfl, sa_cfl=self.sa_cfl)

    def params(self, gamma=1.4):
        return params(gamma, self.cfl, self.flux, self.dt_fixed)

    def initial_primitive(self, gamma=1.4):
        return freestream(self.mach, self.aoa, gamma)


def uniform_state(mesh, w, gamma=1.4):
    """The nv conserved values of a uniform start from primitives w = (rho, u, v, p): the values
    initial_state repeats over the cells.  A batch given these nv values fills the state on the
    device (no per-cell upload)."""
    values = [w[0], w[0] * w[1], w[0] * w[2], w[3] / (gamma - 1) + 0.5 * w[0] * (w[1] * w[1] + w[2] * w[2])]
    if mesh.nv == 5:
        values.append(w[0] * float(mesh.transport['sa_nu_inf'][0]))
    return np.array(values, dtype=np.float64)


def initial_state(mesh, w, gamma=1.4):
    """Uniform conserved state from primitives w = (rho, u, v, p), SoA u[var*n + cell]
    (the reference's static_amr2d_initialize, src/static_amr2d.cpp:360-367)."""
    n = mesh.n_cells
    values = [w[0], w[0] * w[1], w[0] * w[2], w[3] / (gamma - 1) + 0.5 * w[0] * (w[1] * w[1] + w[2] * w[2])]
    if mesh.nv == 5:
        values.append(w[0] * float(mesh.transport['sa_nu_inf'][0]))
    return np.concatenate([np.full(n, v, dtype=np.float64) for v in values])
