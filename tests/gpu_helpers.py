"""Helpers for the GPU parity tests: build the product simulator from a
golden rollout scenario through the reference-facing API."""
from __future__ import annotations

import json

import numpy as np
import torch

from empm_b200 import WarpMPMWrapper


def product_from_rollout(d, key, device="cuda:0"):
    s = json.loads(str(d[f"{key}/scenario"]))
    mpm = WarpMPMWrapper(grid_size=s["G"], grid_lim=1.0, frame_dt=s["frame_dt"], sim_dt=s["sim_dt"], device=device)
    mpm.gravity = list(s["gravity"])
    mpm.material_params = dict(s["params"])
    x0 = torch.from_numpy(d[f"{key}/x0"]).float()
    v0 = torch.from_numpy(d[f"{key}/v0"]).float()
    mpm.add_particles(x0, v0, float(s["vol"]), torch.from_numpy(d[f"{key}/E"]).float(),
                      torch.from_numpy(d[f"{key}/nu"]).float(), float(s["rho"]))
    bbox = False
    for c in s["colliders"]:
        if c["kind"] == "surface":
            mpm.surface_colliders.append([tuple(c["point"]), tuple(c["normal"]), c.get("surface", "sticky"), 0.0])
        elif c["kind"] == "cuboid":
            mpm.moving_boundaries.append([c["point"], c["size"], c["velocity"], 0.0])
        elif c["kind"] == "grid_velocity":
            g = {k: v for k, v in c.items() if k != "kind"}
            mpm.grid_geometry_movers.append(g)
        elif c["kind"] == "geometry":
            g = {k: v for k, v in c.items() if k != "kind"}
            mpm.geometry_colliders.append(g)
        elif c["kind"] == "bbox":
            bbox = True
    mpm.initialize()
    if bbox:
        mpm.mpm_solver.add_bounding_box()
    mpm.mpm_model.yield_stress.copy_(torch.from_numpy(d[f"{key}/ys_in"]).float().to(device))
    return mpm, s


def max_abs(a, b):
    a = a.detach().double().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a, np.float64)
    b = b.detach().double().cpu().numpy() if isinstance(b, torch.Tensor) else np.asarray(b, np.float64)
    return float(np.abs(a - b).max())
