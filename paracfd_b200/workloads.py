"""Named analytic workloads for the time-step path (geometry + brick-hierarchy settings).

``naca0012_slab`` is the single-level case: a uniform 128 x 64 x 64 grid over a 4c x 2c x 2c box
(c = 1 m, h = c/32) around a NACA 0012 section at AoA 4 deg extruded through both Y walls.
``naca4412_wing`` is the 3-level ~4 M-cell case: a NACA 4412 wing of span 3c with flat closed
tips at AoA 6 deg in an 8c x 6c x 6c domain, the finest level in a 0.1c band around the surface
(base h 0.05 m: 4.20 M leaf cells).  Both are the cases the learned preconditioner harvests its
training pairs from and is measured on.

``paraglider16m`` is the 4-level ~16 M leaf-cell paraglider case: elliptic planform, span 10 m,
root chord 2.5 m, anhedral arc radius 6 m, NACA 4415, AoA 8 deg, surface points jittered by at
most 1e-4 chord (seeded), freestream 11 m/s.  The outer surface is closed, so the 2 mm internal
ribs of an inflated wing lie inside the solid and do not enter the flow grid.  ``paraglider5m``
(3 levels, 5.1 M cells) and ``paraglider1m`` (coarser base grid, 1.1 M cells) are the same wing
on smaller grids for profiling captures and quick checks.
"""
from __future__ import annotations

from dataclasses import dataclass, field

from . import BuiltTopology
from .geometry import extruded_wing, naca4_section, paraglider_wing, rotate_section


@dataclass(frozen=True)
class Workload:
    name: str
    domain_lo: tuple
    domain_hi: tuple
    base_cell_size: float
    max_levels: int
    brick_size: int = 8
    wing_refinement_distance: float = 0.5
    surface_refinement_distance: float = 0.25
    wake_length: float = 5.0
    wake_radius: float = 1.5
    speed: float = 11.0
    min_volume_fraction: float = 0.25
    geometry: str = "paraglider"
    aoa: float = 8.0
    case: dict = field(default_factory=lambda: dict(rho=1.225, nu=1.5e-5, cfl=0.5, smagorinsky_cs=0.10,
                                                     projection_tolerance=1e-8, projection_max_iterations=600))

    def describe(self) -> dict:
        names = {"paraglider": "paraglider NACA4415 span10 chord2.5 arcR6 aoa8",
                 "naca0012_slab": f"NACA0012 slab through the Y walls aoa{self.aoa:g}",
                 "naca4412_wing": f"NACA4412 wing span3 flat tips aoa{self.aoa:g}"}
        return {"workload": self.name, "geometry": names[self.geometry],
                "levels": self.max_levels, "brick": self.brick_size, "base_h": self.base_cell_size,
                "domain": [list(self.domain_lo), list(self.domain_hi)], "speed": self.speed,
                "tolerance": self.case["projection_tolerance"], "cfl": self.case["cfl"]}

    def surface(self):
        if self.geometry == "naca0012_slab":
            section = rotate_section(naca4_section(12, 96, 1.0), self.aoa)
            return extruded_wing(section, self.domain_lo[1] - 0.25, self.domain_hi[1] + 0.25)
        if self.geometry == "naca4412_wing":
            section = rotate_section(naca4_section(4412, 96, 1.0), self.aoa)
            return extruded_wing(section, -1.5, 1.5)
        return paraglider_wing()

    def build(self) -> BuiltTopology:
        vertices, triangles = self.surface()
        return BuiltTopology(vertices, triangles, self.domain_lo, self.domain_hi, self.base_cell_size, self.max_levels,
                             self.brick_size, wing_refinement_distance=self.wing_refinement_distance,
                             surface_refinement_distance=self.surface_refinement_distance,
                             wake_length=self.wake_length, wake_radius=self.wake_radius)


WORKLOADS = {
    "paraglider16m": Workload("paraglider16m", (-5.0, -7.5, -8.5), (15.0, 7.5, 6.5), 0.125, 4),
    "paraglider5m": Workload("paraglider5m", (-5.0, -7.5, -8.5), (15.0, 7.5, 6.5), 0.125, 3),
    "paraglider1m": Workload("paraglider1m", (-5.0, -7.5, -8.5), (15.0, 7.5, 6.5), 0.25, 3,
                             wing_refinement_distance=0.5, surface_refinement_distance=0.5),
    "naca0012_slab": Workload("naca0012_slab", (-1.5, -1.0, -1.0), (2.5, 1.0, 1.0), 1.0 / 32.0, 1, speed=10.0,
                              geometry="naca0012_slab", aoa=4.0),
    "naca4412_wing": Workload("naca4412_wing", (-2.5, -3.0, -3.0), (5.5, 3.0, 3.0), 0.05, 3,
                              wing_refinement_distance=0.5, surface_refinement_distance=0.1, wake_length=3.0,
                              wake_radius=0.75, speed=10.0, geometry="naca4412_wing", aoa=6.0),
}


def sweep_instances(seed: int = 20261203) -> list:
    """The batched angle sweep: 16 naca4412_wing instances at AoA -4..11 deg (1 deg steps), each
    with its surface and wing refinement bands drawn from a seeded uniform distribution
    (U[0.03, 0.12] m and U[0.2, 0.6] m), so brick counts vary unevenly between instances."""
    import dataclasses

    import numpy as np

    rng = np.random.default_rng(seed)
    base = WORKLOADS["naca4412_wing"]
    return [dataclasses.replace(base, name=f"naca4412_aoa{a}", aoa=float(a),
                                surface_refinement_distance=round(float(rng.uniform(0.03, 0.12)), 4),
                                wing_refinement_distance=round(float(rng.uniform(0.2, 0.6)), 4))
            for a in range(-4, 12)]


def with_aoa(name: str, aoa: float) -> Workload:
    """The named workload at another angle of attack (the learned preconditioner's harvest runs)."""
    from dataclasses import replace
    return replace(WORKLOADS[name], aoa=aoa)
