"""Simulator facade with the reference's public API.

Keeps the names, arguments, defaults and results of ``WarpMPMWrapper``,
``material_gallery``, ``sample_cube`` / ``sample_sphere`` and the PLY helpers
(phys_sim/diff_simulator/warp_mpm/warp_mpm_wrapper.py:26-499), on this
library's solver:

* particles added by ``add_particles`` are kept as per-call pieces and joined
  once, when the attributes are read or the simulator is initialised;
* ``advance_to`` runs each frame as one library rollout (ping-pong between two
  device states, replayed as a CUDA graph) instead of a Python loop of
  ``partial_clone`` + kernel launches per substep; with a ``step_callback``
  it steps one substep at a time so that the callback sees every substep;
* both optimisation loops drive ``MPMDifferentiableSimulationTrail`` through
  one helper, with the reference's optimiser settings (AdamW, lr 1e-4 online
  and 1e-3 offline, no weight decay; ReduceLROnPlateau(factor 0.1,
  patience 5) and a stop once the learning rate falls below 1e-5 offline).
"""
from __future__ import annotations

import os
from typing import Dict, List, Optional, Sequence

import numpy as np
import torch
from torch import Tensor

from .interface import MPMDifferentiableSimulationTrail
from .mpm_data_structure import MPMModelStruct, MPMStateStruct
from .mpm_solver_diff import MPMWARPDiff

DTYPE = torch.float32

# Material presets by name (the reference's table; "fluid" has no material id
# there either, so selecting it raises TypeError at initialize()).
material_gallery = {
    "jelly": {"material": "jelly"},
    "metal": {"material": "metal"},
    "sand": {"material": "sand", "friction_angle": 35},
    "foam": {"material": "foam"},
    "snow": {"material": "snow"},
    "plasticine": {"material": "plasticine", "yield_stress": 5000., "softening": 0.1},
    "neo-hookean": {"material": "neo-hookean"},
    "fluid": {"material": "fluid"},
}


def sample_cube(lower_corner, cube_size, N):
    """N points uniform in the axis-aligned box [lower_corner, lower_corner +
    cube_size), drawn from numpy's global generator."""
    u = np.random.random_sample((N, 3))
    return np.asarray(lower_corner, dtype=np.float64) + u * np.asarray(cube_size, dtype=np.float64)


def sample_sphere(center, radius, N):
    """N points uniform in a ball: isotropic directions from normalised
    Gaussian triples, radii radius * U^(1/3) (numpy's global generator)."""
    d = np.random.standard_normal((N, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = radius * np.cbrt(np.random.random_sample(N))
    return np.asarray(center, dtype=np.float64) + d * r[:, None]


def _points_np(vertices) -> np.ndarray:
    if isinstance(vertices, Tensor):
        return vertices.detach().cpu().numpy()
    return np.asarray(vertices)


def save_ply_file(vertices, filename=""):
    """Write an ASCII PLY point cloud (the reference writes it with pyvista)."""
    pts = _points_np(vertices).reshape(-1, 3)
    header = "\n".join(["ply", "format ascii 1.0", f"element vertex {len(pts)}", "property float x",
                        "property float y", "property float z", "end_header"])
    with open(filename, "w") as f:
        f.write(header + "\n")
        np.savetxt(f, pts, fmt="%.7g")


def save_ply_seq(vertices, save_path="./outputs/sim", prefix="sim_"):
    """One PLY file per frame of a [F, N, 3] sequence."""
    os.makedirs(save_path, exist_ok=True)
    for i, frame in enumerate(vertices):
        save_ply_file(frame, os.path.join(save_path, f"{prefix}{i:04d}.ply"))


def _per_particle(value, n: int, device) -> Tensor:
    """One scalar attribute for n particles as float32 on `device`: a number
    or a 0-d tensor is broadcast; an array or a 1-d tensor is taken as given
    (a tensor keeps its autograd history, as in the reference)."""
    if isinstance(value, Tensor):
        t = torch.full((n,), float(value.item())) if value.ndim == 0 else value
    elif isinstance(value, np.ndarray):
        t = torch.tensor(value)
    else:
        t = torch.full((n,), float(value))
    return t.to(device=device, dtype=DTYPE)


def _vectors(value, n: int, device) -> Tensor:
    """[n, 3] positions or velocities (None: zeros) as float32 on `device`."""
    if value is None:
        return torch.zeros((n, 3), dtype=DTYPE, device=device)
    t = torch.tensor(value) if isinstance(value, np.ndarray) else value
    return t.to(device=device, dtype=DTYPE)


class _ParticleTable:
    """Per-particle attributes of the bodies added so far, as one list of
    pieces per column; a column is joined once when it is read."""
    COLUMNS = ("x", "v", "vol", "E", "nu", "rho")

    def __init__(self, device):
        self.device = device
        self.pieces: Dict[str, List[Tensor]] = {c: [] for c in self.COLUMNS}
        self.n = 0

    def append(self, n: int, **cols) -> None:
        for c in self.COLUMNS:
            self.pieces[c].append(cols[c])
        self.n += n

    def column(self, c: str) -> Tensor:
        parts = self.pieces[c]
        if not parts:
            shape = (0, 3) if c in ("x", "v") else (0,)
            return torch.empty(shape, dtype=DTYPE, device=self.device)
        if len(parts) > 1:
            self.pieces[c] = parts = [torch.cat(parts)]
        return parts[0]

    def replace(self, c: str, value: Tensor) -> None:
        self.pieces[c] = [value]


def _column_property(c: str):
    return property(lambda self: self._table.column(c), lambda self, value: self._table.replace(c, value))


class WarpMPMWrapper:
    x_t = _column_property("x")
    v_t = _column_property("v")
    vol_t = _column_property("vol")
    E_t = _column_property("E")
    nu_t = _column_property("nu")
    rho_t = _column_property("rho")

    def __init__(self, grid_size=100, grid_lim=1.0, frame_dt=0.01, sim_dt=1e-3, device="cuda:0",
                 requires_grad=False, frame_callback=None, step_callback=None, optim_callback=None):
        self.grid_size = grid_size
        self.grid_lim = grid_lim
        self.frame_dt = frame_dt
        self.sim_dt = sim_dt
        self.device = device
        self.requires_grad = requires_grad
        self.gravity = [0.0, 0.0, -9.8]
        # boundary conditions registered on the solver by initialize(), in this order
        self.surface_colliders = []        # (point, normal, surface, friction)
        self.moving_boundaries = []        # (point, size, velocity, start_time)
        self.geometry_colliders = []       # geo_args dicts
        self.grid_geometry_movers = []     # geo_args dicts
        self.particle_geometry_movers = []
        self.frame_callback = frame_callback
        self.step_callback = step_callback
        self.optim_callback = optim_callback
        self.material_params = material_gallery["jelly"]
        self.initialized = False
        self._table = _ParticleTable(device)
        self._spare_state: Optional[MPMStateStruct] = None

    @property
    def n_particles(self) -> int:
        return self._table.n

    # -- scene set-up -----------------------------------------------------------
    def add_particles(self, x, v=None, vol=1e-5, E=5e4, nu=0.3, rho=2000.0):
        """Append a body of x.shape[0] particles; scalar attributes are
        broadcast. Every position must lie strictly inside (0, grid_lim)."""
        n = x.shape[0]
        xs = _vectors(x, n, self.device)
        assert xs.min().item() > 0.0 and xs.max().item() < self.grid_lim
        self._table.append(n, x=xs, v=_vectors(v, n, self.device), vol=_per_particle(vol, n, self.device),
                           E=_per_particle(E, n, self.device), nu=_per_particle(nu, n, self.device),
                           rho=_per_particle(rho, n, self.device))

    def set_paramters(self, params):
        """Change E (broadcast to every particle) and/or refresh nu on the
        initialised simulator (the reference's spelling of the name)."""
        assert self.initialized
        if "E" in params:
            self.E_t = torch.full((self.n_particles,), 1.0, dtype=DTYPE, device=self.device) * params["E"]
        if "E" in params or "nu" in params:
            self._apply_elasticity()

    def add_grid_geometry_mover(self, geo_args):
        self.grid_geometry_movers.append(geo_args)
        return len(self.grid_geometry_movers) - 1

    def add_particle_mover(self, geo_args):
        """A cylinder of particles held at zero velocity (a rotation modifier
        with both scales 0, active from t = 0 to 999)."""
        self.mpm_solver.enforce_particle_velocity_rotation(
            self.mpm_state, point=geo_args["center"], normal=geo_args["axis"],
            half_height_and_radius=[geo_args["half_height"], geo_args["radius"]], rotation_scale=0.0,
            translation_scale=0.0, start_time=0.0, end_time=999.0)

    def _apply_elasticity(self):
        self.mpm_solver.set_E_nu_from_torch(self.mpm_model, self.E_t, self.nu_t, device=self.device)
        self.mpm_solver.prepare_mu_lam(self.mpm_model, self.mpm_state, self.device)

    def _register_boundaries(self):
        s = self.mpm_solver
        for args in self.surface_colliders:
            s.add_surface_collider(*args[:4])
        for args in self.moving_boundaries:
            s.set_velocity_on_cuboid(*args[:4])
        for geo in self.geometry_colliders:
            s.add_geometry_collider(geo_args=geo)
        for geo in self.grid_geometry_movers:
            s.set_grid_velocity_on_geometry(geo_args=geo)

    def initialize(self):
        """Build the state, the model and the solver from the bodies, the
        material preset and the registered boundary conditions."""
        n, dev, rg = self.n_particles, self.device, self.requires_grad
        st = MPMStateStruct()
        st.init(n, device=dev, requires_grad=rg)
        st.from_torch(self.x_t, self.vol_t, None, self.v_t, n_grid=self.grid_size, grid_lim=self.grid_lim,
                      device=dev, requires_grad=rg)
        st.reset_density(tensor_density=self.rho_t, selection_mask=None, device=dev, update_mass=True)
        md = MPMModelStruct()
        md.init(n, device=dev, requires_grad=rg)
        md.init_other_params(n_grid=self.grid_size, grid_lim=self.grid_lim, device=dev)
        md.gravitational_accelaration = tuple(float(g) for g in self.gravity[:3])
        solver = MPMWARPDiff()
        solver.initialize(n, n_grid=self.grid_size, grid_lim=self.grid_lim, device=dev)
        solver.set_parameters_dict(md, st, self.material_params)
        self.mpm_state, self.mpm_model, self.mpm_solver = st, md, solver
        self._apply_elasticity()
        self._register_boundaries()
        self._spare_state = None
        self.initialized = True

    # -- forward simulation -----------------------------------------------------
    def advance_to_static(self, n_frames=10):
        """advance_to without the per-frame callback."""
        saved, self.frame_callback = self.frame_callback, None
        try:
            self.advance_to(n_frames=n_frames)
        finally:
            self.frame_callback = saved

    def _spare_for(self, state: MPMStateStruct) -> MPMStateStruct:
        """A second device state to ping-pong with `state` (kept between
        frames; its per-particle constants are refreshed from `state`)."""
        spare = self._spare_state
        if spare is None or spare is state or spare.n_particles != state.n_particles:
            return state.partial_clone(requires_grad=False)
        spare.particle_vol.copy_(state.particle_vol)
        spare.particle_density.copy_(state.particle_density)
        spare._x4[:, 3].copy_(state._x4[:, 3])
        return spare

    def _one_frame(self, state: MPMStateStruct, n_substeps: int, first_step: int) -> MPMStateStruct:
        if self.step_callback is None:
            spare = self._spare_for(state)
            out = self.mpm_solver.rollout(self.mpm_model, state, spare, self.sim_dt, n_substeps)
            self._spare_state = spare if out is state else state
            return out
        for k in range(n_substeps):
            self.step_callback(self, first_step + k)
            spare = self._spare_for(state)
            self.mpm_solver.p2g2p_differentiable(self.mpm_model, state, spare, self.sim_dt, device=self.device)
            self._spare_state, state = state, spare
        return state

    def advance_to(self, n_frames):
        """Simulate n_frames frames of frame_dt / sim_dt substeps from the
        current state. Returns the positions before the first frame and after
        every frame, [n_frames + 1, N, 3]."""
        n_substeps = int(self.frame_dt / self.sim_dt)
        state = self.mpm_state
        frames = [state.particle_x.clone()]
        for f in range(n_frames):
            if self.frame_callback:
                self.frame_callback(self, f)
            state = self._one_frame(state, n_substeps, f * n_substeps)
            frames.append(state.particle_x.clone())
        self.mpm_state = state
        return torch.stack(frames)

    # -- differentiable optimisation --------------------------------------------
    def _trail_positions(self, state, x, v, E, nu, rho, n_train_frames):
        """Positions once per frame over n_train_frames frames, differentiable
        in v, E, nu and rho (the trainer's Trail call; all densities may change)."""
        n_substeps = int(self.frame_dt / self.sim_dt)
        every_particle = torch.ones(self.n_particles, dtype=torch.bool, device=self.device)
        return MPMDifferentiableSimulationTrail.apply(
            self.mpm_solver, state, self.mpm_model, n_substeps, self.sim_dt, n_train_frames * n_substeps,
            x, v, E, nu, rho, every_particle, None, self.device, True, 0)

    def _leaf(self, value, per_particle: bool) -> Tensor:
        """A trainable copy of an initial guess: 0-d, or one value per particle."""
        shape = (self.n_particles,) if per_particle else ()
        return torch.full(shape, 1.0, dtype=DTYPE, device=self.device).mul(value).requires_grad_()

    def prepare_online_optimization(self, x, parameters):
        if not self.initialized:
            self.initialize()
        self.optim = {"trainable_params": [self._leaf(parameters["E"], False)]}

    def run_online_optimization_step(self, x, parameters, n_train_frames=1, n_iters=1, loss_func=None):
        """n_iters AdamW steps (lr 1e-4) on a scalar E from parameters["E"],
        from a differentiable copy of the current state. Returns the fitted E,
        the mean loss and the last rollout's positions."""
        E = self._leaf(parameters["E"], False)
        opt = torch.optim.AdamW([E], lr=1e-4, weight_decay=0.)
        state = self.mpm_state.partial_clone(requires_grad=True)
        x0 = x.clone()
        losses, pos = [], None
        for _ in range(n_iters):
            opt.zero_grad()
            if self.optim_callback:
                self.optim_callback(self)
            pos = self._trail_positions(state, x0, self.v_t, E, self.nu_t, self.rho_t, n_train_frames)
            loss = loss_func(pos)
            losses.append(loss.item())
            loss.backward()
            opt.step()
        return {"param": {"E": E.item()}, "loss": float(np.mean(losses)), "points": pos.clone().detach()}

    def run_diff_optimization(self, parameters, n_train_frames, max_iters, loss_func=None):
        """Fit the parameters named in `parameters` ("E" and "nu" as scalars,
        "rho" per particle, starting from the given values) with AdamW (lr
        1e-3) and ReduceLROnPlateau (factor 0.1, patience 5), for at most
        max_iters iterations or until the learning rate drops below 1e-5.
        Returns {name: fitted tensor}."""
        if not self.initialized:
            self.initialize()
        start = {"x": self.x_t.clone(), "v": self.v_t.clone(), "E": self.E_t.clone(), "nu": self.nu_t.clone(),
                 "rho": self.rho_t.clone()}
        fitted = {name: self._leaf(parameters[name], name == "rho") for name in ("E", "nu", "rho")
                  if name in parameters}
        start.update(fitted)
        opt = torch.optim.AdamW(list(fitted.values()), lr=1e-3, weight_decay=0.)
        plateau = torch.optim.lr_scheduler.ReduceLROnPlateau(opt, mode="min", factor=0.1, patience=5)
        for _ in range(max_iters):
            opt.zero_grad()
            if self.optim_callback:
                self.optim_callback(self)
            pos = self._trail_positions(self.mpm_state, start["x"], start["v"], start["E"], start["nu"],
                                        start["rho"], n_train_frames)
            loss = loss_func(pos)
            loss.backward()
            opt.step()
            plateau.step(loss.item())
            if opt.param_groups[0]["lr"] < 1e-5:
                break
        return fitted
