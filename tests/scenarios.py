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

from oracle.specs import SURFACE_TYPES, _unit, oracle_colliders  # noqa: F401


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
