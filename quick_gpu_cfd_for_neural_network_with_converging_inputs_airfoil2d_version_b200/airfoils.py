"""Synthetic airfoil contours: NACA 4-digit polygons in the reference's point convention.

The published NACA 4-digit section: half-thickness
    yt = 5 t (0.2969 sqrt(x) - 0.1260 x - 0.3516 x^2 + 0.2843 x^3 - 0.1036 x^4)
(closed trailing edge), applied normal to the camber line
    yc = m/p^2 (2 p x - x^2)              for x < p
    yc = m/(1-p)^2 ((1 - 2p) + 2 p x - x^2) for x >= p.
Points follow the reference's polygon convention (src/sdf.h:97-114): `panels` cosine-spaced
panels per surface, upper surface from the trailing edge toward the leading edge, then the
lower surface from the leading edge to the trailing edge.  The duplicated closing trailing
edge vertex is dropped (the mesh builder rejects repeated vertices), leaving 2*panels unique
vertices; the leading and trailing edges are placed exactly at (0,0) and (1,0).
Edge patches: 1 upper surface, 2 lower surface.
"""
import math

import numpy as np


def naca4(m, p, t, panels=100):
    """Return (x, y, patches) for a NACA 4-digit airfoil with unit chord."""
    m, p, t = float(m), float(p), float(t)
    if not (0 <= m < 0.2 and 0 < p < 1 and 0 < t < 0.5):
        raise ValueError('NACA parameters out of range')

    def camber(x):
        if m == 0:
            return 0.0, 0.0
        if x < p:
            return m / (p * p) * (2 * p * x - x * x), 2 * m / (p * p) * (p - x)
        return m / ((1 - p) ** 2) * ((1 - 2 * p) + 2 * p * x - x * x), 2 * m / ((1 - p) ** 2) * (p - x)

    def thickness(x):
        s = math.sqrt(x) if x > 0 else 0.0
        return 5 * t * (0.2969 * s - 0.1260 * x - 0.3516 * x * x + 0.2843 * x ** 3 - 0.1036 * x ** 4)

    def point(x, upper):
        if x == 0.0:
            return 0.0, 0.0
        if x == 1.0:
            return 1.0, 0.0
        yc, dy = camber(x)
        yt = thickness(x)
        th = math.atan(dy)
        if upper:
            return x - yt * math.sin(th), yc + yt * math.cos(th)
        return x + yt * math.sin(th), yc - yt * math.cos(th)

    xs, ys = [], []
    for i in range(panels):                      # upper: trailing edge -> leading edge (exclusive)
        x = 0.5 * (1 - math.cos(math.pi * (1 - i / panels)))
        px, py = point(x, True)
        xs.append(px), ys.append(py)
    for i in range(panels):                      # lower: leading edge -> trailing edge (exclusive)
        x = 0.5 * (1 - math.cos(math.pi * i / panels))
        px, py = point(x, False)
        xs.append(px), ys.append(py)
    patches = [1] * panels + [2] * panels
    return np.array(xs), np.array(ys), np.array(patches, dtype=np.int32)


def seeded_naca(rng):
    """One draw of the synthetic batch distribution: m~U[0,0.06], p~U[0.2,0.6], t~U[0.08,0.15]."""
    return float(rng.uniform(0.0, 0.06)), float(rng.uniform(0.2, 0.6)), float(rng.uniform(0.08, 0.15))
