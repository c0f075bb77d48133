"""Named analytic workloads for the time-step path (geometry + brick-hierarchy settings).

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
from .geometry import paraglider_wing


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
    case: dict = field(default_factory=lambda: dict(rho=1.225, nu=1.5e-5, cfl=0.5, smagorinsky_cs=0.10,
                                                     projection_tolerance=1e-8, projection_max_iterations=600))

    def describe(self) -> dict:
        return {"workload": self.name, "geometry": "paraglider NACA4415 span10 chord2.5 arcR6 aoa8",
                "levels": self.max_levels, "brick": self.brick_size, "base_h": self.base_cell_size,
                "domain": [list(self.domain_lo), list(self.domain_hi)], "speed": self.speed,
                "tolerance": self.case["projection_tolerance"], "cfl": self.case["cfl"]}

    def build(self) -> BuiltTopology:
        vertices, triangles = paraglider_wing()
        return BuiltTopology(vertices, triangles, self.domain_lo, self.domain_hi, self.base_cell_size, self.max_levels,
                             self.brick_size, wing_refinement_distance=self.wing_refinement_distance,
                             surface_refinement_distance=self.surface_refinement_distance,
                             wake_length=self.wake_length, wake_radius=self.wake_radius)


WORKLOADS = {
    "paraglider16m": Workload("paraglider16m", (-5.0, -7.5, -8.5), (15.0, 7.5, 6.5), 0.125, 4),
    "paraglider5m": Workload("paraglider5m", (-5.0, -7.5, -8.5), (15.0, 7.5, 6.5), 0.125, 3),
    "paraglider1m": Workload("paraglider1m", (-5.0, -7.5, -8.5), (15.0, 7.5, 6.5), 0.25, 3,
                             wing_refinement_distance=0.5, surface_refinement_distance=0.5),
}
