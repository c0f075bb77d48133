"""Analytic wing surfaces (closed, outward-oriented triangle meshes) for the preprocessing entry
point ``pcfd_topology_build``.

The reference imports a closed OpenCascade solid from STEP (src/core/geometry/step_import.*) and
writes analytic NACA STEP files (src/core/geometry/naca_step.cpp:85-108).  Here the same
analytic shapes are produced directly as triangle meshes:

* ``naca4_section`` -- NACA 4-digit thickness and camber (published formulas), closed trailing
  edge (x^4 coefficient -0.1036, as the reference's closed_sharp option, naca_step.h:14-16);
* ``extruded_wing`` -- a section extruded over a span, with flat closed tips;
* ``paraglider_wing`` -- elliptic planform on an anhedral arc, jittered surface points.
"""
from __future__ import annotations

import numpy as np


def naca4_section(digits: int, points_per_side: int = 64, chord: float = 1.0) -> np.ndarray:
    """Closed counter-clockwise (x, z) polygon, trailing edge first, cosine spacing."""
    m = (digits // 1000) / 100.0
    p = ((digits // 100) % 10) / 10.0
    t = (digits % 100) / 100.0
    beta = np.linspace(0.0, np.pi, points_per_side + 1)
    x = 0.5 * (1.0 - np.cos(beta))
    yt = 5 * t * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3 - 0.1036 * x ** 4)
    yc = np.zeros_like(x)
    slope = np.zeros_like(x)
    if m > 0 and p > 0:
        fore = x < p
        yc[fore] = m / p ** 2 * (2 * p * x[fore] - x[fore] ** 2)
        slope[fore] = 2 * m / p ** 2 * (p - x[fore])
        aft = ~fore
        yc[aft] = m / (1 - p) ** 2 * ((1 - 2 * p) + 2 * p * x[aft] - x[aft] ** 2)
        slope[aft] = 2 * m / (1 - p) ** 2 * (p - x[aft])
    theta = np.arctan(slope)
    xu, zu = x - yt * np.sin(theta), yc + yt * np.cos(theta)
    xl, zl = x + yt * np.sin(theta), yc - yt * np.cos(theta)
    upper = np.stack([xu, zu], 1)[::-1]          # TE -> LE
    lower = np.stack([xl, zl], 1)[1:-1]          # LE (exclusive) -> TE (exclusive)
    poly = np.concatenate([upper, lower]) * chord
    poly[0] = (chord, 0.0)
    area = 0.5 * np.sum(poly[:, 0] * np.roll(poly[:, 1], -1) - np.roll(poly[:, 0], -1) * poly[:, 1])
    return poly if area > 0 else poly[::-1].copy()


def rotate_section(poly: np.ndarray, aoa_deg: float, pivot=(0.25, 0.0)) -> np.ndarray:
    """Nose-up rotation by the angle of attack about the pivot (flow along +X)."""
    a = np.radians(aoa_deg)
    c, s = np.cos(a), np.sin(a)
    d = poly - np.asarray(pivot)
    return np.stack([pivot[0] + c * d[:, 0] + s * d[:, 1], pivot[1] - s * d[:, 0] + c * d[:, 1]], 1)


def _orient_outward(vertices: np.ndarray, triangles: np.ndarray) -> np.ndarray:
    p0, p1, p2 = (vertices[triangles[:, q]] for q in range(3))
    volume = np.einsum("ij,ij->i", p0, np.cross(p1, p2)).sum()
    return triangles if volume > 0 else triangles[:, [0, 2, 1]].copy()


def extruded_wing(section: np.ndarray, y0: float, y1: float, offset=(0.0, 0.0, 0.0), caps: bool = True):
    """Section (x, z) swept along +Y from y0 to y1; returns (vertices[N,3], triangles[M,3])."""
    n = len(section)
    bottom = np.stack([section[:, 0], np.full(n, y0), section[:, 1]], 1)
    top = np.stack([section[:, 0], np.full(n, y1), section[:, 1]], 1)
    vertices = [bottom, top]
    tris = []
    for q in range(n):
        a0, b0, a1, b1 = q, (q + 1) % n, n + q, n + (q + 1) % n
        tris += [(a0, a1, b1), (a0, b1, b0)]
    if caps:
        centre = section.mean(0)
        c0 = 2 * n
        vertices.append(np.array([[centre[0], y0, centre[1]], [centre[0], y1, centre[1]]]))
        for q in range(n):
            a, b = q, (q + 1) % n
            # the section runs counter-clockwise in (x, z): (centre, a, b) faces -Y, (centre, b, a) +Y
            tris += [(c0, a, b), (c0 + 1, n + b, n + a)]
    v = np.concatenate(vertices) + np.asarray(offset)
    t = _orient_outward(v, np.array(tris, np.int64))
    return v.astype(np.float64), t.astype(np.uint32)


def paraglider_wing(span: float = 10.0, root_chord: float = 2.5, arc_radius: float = 6.0, digits: int = 4415,
                    aoa_deg: float = 8.0, stations: int = 96, points_per_side: int = 48, jitter: float = 1e-4,
                    seed: int = 20261203, tip_chord: float = 0.02, tip_clustering: bool = False,
                    flat_tips: bool = True):
    """Elliptic planform c(eta) = c0 sqrt(1 - eta^2) on a circular anhedral arc of the given
    radius (projected span ``span``), NACA section, tips closed at a small residual chord.
    Surface points are displaced by a seeded uniform jitter of at most ``jitter * root_chord``.
    With ``flat_tips`` the two tip sections and their cap centres keep their exact positions, so
    each closed tip is one plane: a jittered cap folds at the 1e-4 chord scale, and the cut-cell
    builder then finds isolated fluid slivers (~1e-12 m^3) whose pressure-gradient stencils have
    rank 1, which the composite system rejects."""
    section = rotate_section(naca4_section(digits, points_per_side, 1.0), aoa_deg, pivot=(0.25, 0.0))
    half = 0.5 * span
    theta_max = np.arcsin(min(1.0, half / arc_radius))
    eta = np.sin(np.linspace(-np.pi / 2, np.pi / 2, stations)) if tip_clustering else np.linspace(-1.0, 1.0, stations)
    theta = eta * theta_max
    chord = root_chord * np.sqrt(np.maximum(1.0 - eta ** 2, 0.0))
    chord = np.maximum(chord, tip_chord * root_chord)
    n = len(section)
    rings = []
    for k in range(stations):
        c = chord[k]
        x = (section[:, 0] - 0.25) * c + 0.25 * root_chord
        local_z = section[:, 1] * c
        # arc: the section plane is rotated by theta about X, centred on the arc
        y = (arc_radius + local_z) * np.sin(theta[k])
        z = (arc_radius + local_z) * np.cos(theta[k]) - arc_radius
        rings.append(np.stack([x, y, z], 1))
    v = np.concatenate(rings)
    tris = []
    for k in range(stations - 1):
        for q in range(n):
            a0, b0 = k * n + q, k * n + (q + 1) % n
            a1, b1 = a0 + n, b0 + n
            tris += [(a0, a1, b1), (a0, b1, b0)]
    c0 = len(v)
    v = np.concatenate([v, rings[0].mean(0, keepdims=True), rings[-1].mean(0, keepdims=True)])
    last = (stations - 1) * n
    for q in range(n):
        a, b = q, (q + 1) % n
        tris += [(c0, a, b), (c0 + 1, last + b, last + a)]
    rng = np.random.default_rng(seed)
    offset = rng.uniform(-jitter * root_chord, jitter * root_chord, size=v.shape)
    if flat_tips:
        offset[:n] = 0.0
        offset[last:] = 0.0
    v = v + offset
    t = _orient_outward(v, np.array(tris, np.int64))
    return v.astype(np.float64), t.astype(np.uint32)
