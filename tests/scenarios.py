"""Scenario helpers shared by the CPU and GPU parity tests.

Turns the collider descriptions stored in the golden fixtures (and the
synthetic benchmark configurations) into oracle collider specs, mirroring the
argument handling of the reference's collider factories
(phys_sim/diff_simulator/warp_mpm/mpm_solver_diff.py:437-938).
"""
from __future__ import annotations

import json
import math

import numpy as np

from oracle import oracle as O

SURFACE_TYPES = {"sticky": 0, "slip": 1, "cut": 11}


def _unit(v):
    s = 1.0 / math.sqrt(float(sum(t * t for t in v)))
    return tuple(s * t for t in v)


def oracle_colliders(specs, mask=None):
    out = []
    for s in specs:
        k = s["kind"]
        if k == "surface":
            out.append(O.OrColliderSpec(O.SURFACE, surface_type=SURFACE_TYPES.get(s.get("surface", "sticky"), 2),
                                        point=tuple(s["point"]), normal=_unit(s["normal"]),
                                        start_time=s.get("start_time", 0.0), end_time=s.get("end_time", 999.0)))
        elif k in ("geometry", "grid_velocity"):
            c = O.OrColliderSpec(O.GEOMETRY if k == "geometry" else O.GRID_VELOCITY)
            c.surface_type = SURFACE_TYPES.get(s.get("surface", "sticky"), 2)
            shape = s["shape"]
            if shape == "cube":
                c.shape, c.point, c.size = O.CUBE, tuple(s["center"]), tuple(s["size"])
            elif shape == "sphere":
                c.shape, c.point, c.radius = O.SPHERE, tuple(s["center"]), s["radius"]
            elif shape == "cylinder":
                c.shape, c.point, c.normal = O.CYLINDER, tuple(s["center"]), _unit(s["axis"])
                c.radius, c.half_height = s["radius"], s["half_height"]
            else:
                c.shape, c.point, c.normal = O.HALFSPACE, tuple(s["point"]), _unit(s["normal"])
            c.velocity = tuple(s.get("velocity", (0.0, 0.0, 0.0)))
            c.angular_velocity = s.get("angular_velocity", 0.0)
            c.rot_axis = tuple(s.get("rot_axis", (1.0, 0.0, 0.0)))
            c.start_time = s.get("start_time", 0.0)
            c.end_time = s.get("end_time", 999.0)
            c.reset = s.get("reset", 0)
            c.active = s.get("active", True)
            out.append(c)
        elif k == "cuboid":
            out.append(O.OrColliderSpec(O.CUBOID_VELOCITY, point=tuple(s["point"]), size=tuple(s["size"]),
                                        velocity=tuple(s["velocity"]), start_time=s.get("start_time", 0.0),
                                        end_time=s.get("end_time", 999.0), reset=s.get("reset", 0)))
        elif k == "bbox":
            out.append(O.OrColliderSpec(O.BOUNDING_BOX))
        elif k == "grid_mask":
            out.append(O.OrColliderSpec(O.GRID_MASK, mask=np.ascontiguousarray(mask.reshape(-1), dtype=np.int32)))
        else:
            raise ValueError(k)
    return out


MATERIAL_IDS = {"jelly": 0, "metal": 1, "sand": 2, "foam": 3, "snow": 4, "plasticine": 5, "neo-hookean": 6}


def oracle_from_rollout(d, key, precision="fp64"):
    """OracleSim for a rollout fixture written by tests/golden/make_golden.py."""
    s = json.loads(str(d[f"{key}/scenario"]))
    n = s["n"]
    x0 = d[f"{key}/x0"]
    vol = np.full(n, s["vol"])
    rho = np.full(n, np.float32(s["rho"]), dtype=np.float64)
    params = s["params"]
    sim = O.OracleSim(x0, d[f"{key}/v0"], vol, rho * vol, d[f"{key}/E"], d[f"{key}/nu"], n_grid=s["G"],
                      material=MATERIAL_IDS[params["material"]], gravity=tuple(s["gravity"]),
                      yield_stress=d[f"{key}/ys_in"], softening=params.get("softening", 0.1),
                      plastic_viscosity=params.get("plastic_viscosity", 0.0),
                      friction_angle=params.get("friction_angle", 25.0),
                      rpic_damping=params.get("rpic_damping", 0.0),
                      grid_v_damping_scale=params.get("grid_v_damping_scale", 1.1), precision=precision)
    sim.colliders = oracle_colliders(s["colliders"])
    return sim, s
