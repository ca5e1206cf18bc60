"""Cases described by the reference driver's settings file (the key/value settings.txt that its
pipeline writes, pipeline/configuration.py:143-167, and that src/quick_airfoil.cpp:15-27 reads).

    s, boxes = parse_settings(text)
    spec = SettingsSpec(s, boxes, 'LF1')   # a CaseSpec whose mesh, boundary and transport records
                                           # come verbatim from the settings values
"""
from . import cases


def parse_settings(text):
    out, boxes = {}, []
    for line in text.splitlines():
        parts = line.split()
        if not parts:
            continue
        if parts[0] == 'box':
            boxes.append([float(v) for v in parts[1:]])
        else:
            out[parts[0]] = parts[1]
    return out, boxes


def spec_from_settings(s, boxes, profile):
    """CaseSpec equivalent of a reference settings.txt (src/quick_airfoil.cpp:149-162)."""
    spec = cases.CaseSpec(profile=profile, mach=float(s['mach']), aoa=float(s['aoa']),
                          physics='sa' if s['turbulence'] == 'sa-neg' else 'laminar',
                          law=s['viscosity'], flux='hllc' if s['flux'] == 'hllc' else 'ausm', cfl=float(s['cfl']),
                          viscous_cfl=float(s['viscous_cfl']), sa_cfl=float(s['sa_cfl']), agglomerate=True,
                          kinds=tuple(s['bc%d' % i] for i in range(4)), dt_fixed=float(s['fixed_dt']))
    return spec


def transport_from_settings(s, gamma):
    t = cases.transport('laminar', sa=s['turbulence'] == 'sa-neg', law=s['viscosity'], mu=float(s['mu_star']),
                        sutherland=float(s['sutherland_star']), gamma=gamma, viscous_cfl=float(s['viscous_cfl']),
                        sa_cfl=float(s['sa_cfl']), sa_nu_inf=float(s['sa_nu_inf']),
                        wall_probe_min_h=float(s['wall_probe_min_h']))
    if s['viscosity'] != 'sutherland':
        t['temperature_ref'] = 1.0
        t['sutherland'] = 0.0
    return t


class SettingsSpec(cases.CaseSpec):
    """A CaseSpec whose records come verbatim from reference settings values."""

    def __init__(self, s, boxes, profile):
        base = spec_from_settings(s, boxes, profile)
        super().__init__(**{k: getattr(base, k) for k in base.__dataclass_fields__})
        self._s = s
        self._boxes = boxes

    def options(self):
        s = self._s
        return dict(xmin=float(s['xmin']), xmax=float(s['xmax']), ymin=float(s['ymin']), ymax=float(s['ymax']),
                    nx=int(float(s['nx'])), ny=int(float(s['ny'])), buffer=int(float(s['buffer'])),
                    max_cells=int(float(s['max_cells'])), levels=int(float(s['levels'])), boxes=self._boxes,
                    agglomerate_small=1, profile=self.profile)

    def boundary_records(self, gamma=1.4):
        return cases.boundaries(self.mach, self.aoa, gamma, self.kinds, float(self._s['outlet_p_star']))

    def transport_record(self, gamma=1.4):
        return transport_from_settings(self._s, gamma)
