"""Oracle-side helpers: collider descriptions -> OrColliderSpec, and an
OracleSim for a synthetic workload. TEST INFRASTRUCTURE ONLY (tests and the
bench's CPU-baseline leg); mirrors the argument handling of the reference's
collider factories (phys_sim/diff_simulator/warp_mpm/mpm_solver_diff.py:437-938).
"""
from __future__ import annotations

import math

import numpy as np

from . import oracle as O

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


def sim_from_workload(w, precision="fp64", collider_f32=False):
    """OracleSim for an empm_b200.workloads.Workload."""
    sim = O.OracleSim(w.x, w.v, w.vol, w.rho.astype(np.float64) * w.vol, w.E, w.nu, n_grid=w.G,
                      material=MATERIAL_IDS[w.material], gravity=w.gravity, yield_stress=w.ys, precision=precision,
                      collider_f32=collider_f32)
    sim.colliders = oracle_colliders(w.colliders)
    return sim


def workload_callback(w):
    """Per-substep callback applying the workload's cuboid velocity schedule."""
    if w.velocity_schedule is None:
        return None
    k = [i for i, c in enumerate(w.colliders) if c["kind"] == "cuboid"][0]

    def cb(sim, step):
        sim.colliders[k].velocity = tuple(w.velocity_schedule(step))

    return cb
