"""State, model and boundary-condition objects of the MPM simulator.

Mirrors phys_sim/diff_simulator/warp_mpm/mpm_data_structure.py (same class
names, fields, method names and argument orders), backed by PyTorch device
tensors in the library's layout instead of Warp arrays:

* ``particle_x`` / ``particle_v`` are live ``[N, 3]`` views of the float4
  planes ``(x, y, z, mass)`` / ``(vx, vy, vz, 0)``; ``particle_mass`` is the
  live view of the fourth column of the x plane.
* ``particle_C``, ``particle_F_trial`` and ``particle_F`` are 3x3 fields
  stored as f9 planes; reading them returns an ``[N, 3, 3]`` copy and
  assigning packs a tensor back.
* the grid lives in the solver's context (``MPMWARPDiff``), not in the state.
"""
from __future__ import annotations

import ctypes
import math
from typing import Optional, Sequence, Union

import torch
from torch import Tensor

from . import _native as N

DTYPE = torch.float32


def _dev(device) -> torch.device:
    d = torch.device(device)
    if d.type != "cuda":
        raise ValueError(f"empm_b200 runs on CUDA devices only (got {device!r}); there is no CPU path")
    return d


def _stream_ptr(device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _f9_pack(dst: Tensor, m: Tensor) -> None:
    """Pack [N,3,3] (or [N,9]) into f9 planes (float4 A, float4 B, float C)."""
    n = m.shape[0]
    m = m.reshape(n, 9).to(dtype=DTYPE)
    dst[: 4 * n].view(n, 4).copy_(m[:, 0:4])
    dst[4 * n: 8 * n].view(n, 4).copy_(m[:, 4:8])
    dst[8 * n: 9 * n].copy_(m[:, 8])


def _f9_unpack(src: Tensor, n: int) -> Tensor:
    return torch.cat([src[: 4 * n].view(n, 4), src[4 * n: 8 * n].view(n, 4), src[8 * n: 9 * n].view(n, 1)],
                     dim=1).view(n, 3, 3)


def _f9_identity(dst: Tensor, n: int) -> None:
    dst.zero_()
    dst[: 4 * n].view(n, 4)[:, 0] = 1.0
    dst[4 * n: 8 * n].view(n, 4)[:, 0] = 1.0
    dst[8 * n: 9 * n] = 1.0


class MPMStateStruct:
    """Particle state (mpm_data_structure.py:13-387)."""

    def __init__(self):
        self.n_particles = 0
        self.device = None
        self.requires_grad = False
        self.grid_res = 10

    # -- allocation ---------------------------------------------------------
    def init(self, shape: Union[Sequence[int], int], device="cuda:0", requires_grad=False) -> None:
        n = int(shape if isinstance(shape, int) else shape[0])
        d = _dev(device)
        self.n_particles = n
        self.device = d
        self.requires_grad = requires_grad
        self._x4 = torch.zeros((n, 4), dtype=DTYPE, device=d)
        self._v4 = torch.zeros((n, 4), dtype=DTYPE, device=d)
        self._C = torch.zeros(9 * n, dtype=DTYPE, device=d)
        self._F_trial = torch.zeros(9 * n, dtype=DTYPE, device=d)
        self._F = torch.zeros(9 * n, dtype=DTYPE, device=d)
        self.particle_cov = torch.zeros(6 * n, dtype=DTYPE, device=d)
        self.particle_vol = torch.zeros(n, dtype=DTYPE, device=d)
        self.particle_density = torch.zeros(n, dtype=DTYPE, device=d)
        self.particle_selection = torch.zeros(n, dtype=torch.int32, device=d)
        self._has_selection = False

    def init_grid(self, grid_res: int, device="cuda:0", requires_grad=False):
        self.grid_res = int(grid_res)

    # -- live views / packed fields -------------------------------------------
    @property
    def particle_x(self) -> Tensor:
        return self._x4[:, :3]

    @particle_x.setter
    def particle_x(self, t: Tensor):
        self._x4[:, :3].copy_(t.reshape(-1, 3))

    @property
    def particle_v(self) -> Tensor:
        return self._v4[:, :3]

    @particle_v.setter
    def particle_v(self, t: Tensor):
        self._v4[:, :3].copy_(t.reshape(-1, 3))

    @property
    def particle_mass(self) -> Tensor:
        return self._x4[:, 3]

    @particle_mass.setter
    def particle_mass(self, t: Tensor):
        self._x4[:, 3].copy_(t.reshape(-1))

    @property
    def particle_C(self) -> Tensor:
        return _f9_unpack(self._C, self.n_particles)

    @particle_C.setter
    def particle_C(self, t: Tensor):
        _f9_pack(self._C, t)

    @property
    def particle_F_trial(self) -> Tensor:
        return _f9_unpack(self._F_trial, self.n_particles)

    @particle_F_trial.setter
    def particle_F_trial(self, t: Tensor):
        _f9_pack(self._F_trial, t)

    @property
    def particle_F(self) -> Tensor:
        return _f9_unpack(self._F, self.n_particles)

    @particle_F.setter
    def particle_F(self, t: Tensor):
        _f9_pack(self._F, t)

    @property
    def particle_stress(self) -> Tensor:
        raise AttributeError("particle_stress is not materialised: the fused P2G kernel computes the Kirchhoff "
                             "stress in registers and scatters it directly")

    # -- C ABI views ------------------------------------------------------------
    def _particles(self) -> N.EmpmParticles:
        return N.EmpmParticles(self._x4.data_ptr(), self._v4.data_ptr(), self._C.data_ptr(), self._F_trial.data_ptr())

    def _sel_ptr(self):
        return self.particle_selection.data_ptr() if self._has_selection else None

    # -- reference methods ----------------------------------------------------
    def from_torch(self, tensor_x: Tensor, tensor_volume: Tensor, tensor_cov: Optional[Tensor] = None,
                   tensor_velocity: Optional[Tensor] = None, n_grid: int = 100, grid_lim=1.0, device="cuda:0",
                   requires_grad=True):
        n = tensor_x.shape[0]
        assert tensor_x.shape[0] == tensor_volume.shape[0]
        if self.n_particles != n:
            self.init(n, device=device, requires_grad=requires_grad)
        self.init_grid(grid_res=n_grid, device=device, requires_grad=requires_grad)
        self.particle_x = tensor_x.detach().to(self.device, DTYPE)
        self.particle_vol.copy_(tensor_volume.detach().reshape(-1).to(self.device, DTYPE))
        if tensor_cov is not None:
            self.particle_cov.copy_(tensor_cov.detach().reshape(-1).to(self.device, DTYPE))
        if tensor_velocity is not None:
            self.particle_v = tensor_velocity.detach().to(self.device, DTYPE)
        _f9_identity(self._F_trial, n)

    def reset_state(self, tensor_x: Tensor, tensor_cov: Optional[Tensor] = None,
                    tensor_velocity: Optional[Tensor] = None, tensor_density: Optional[Tensor] = None,
                    selection_mask: Optional[Tensor] = None, device="cuda:0", requires_grad=True):
        n = self.n_particles
        if tensor_x is not None:
            self.particle_x = tensor_x.detach().to(self.device, DTYPE)
        if tensor_cov is not None:
            self.particle_cov.copy_(tensor_cov.detach().reshape(-1).to(self.device, DTYPE))
        if tensor_velocity is not None:
            self.particle_v = tensor_velocity.detach().to(self.device, DTYPE)
        if tensor_density is not None and selection_mask is not None:
            m = selection_mask.to(self.device).to(torch.int32) == 1
            self.particle_density[m] = tensor_density.detach().to(self.device, DTYPE).reshape(-1)[m]
        _f9_identity(self._F_trial, n)
        _f9_identity(self._F, n)
        self._C.zero_()

    def continue_from_torch(self, tensor_x: Tensor, tensor_velocity: Optional[Tensor] = None,
                            tensor_F: Optional[Tensor] = None, tensor_C: Optional[Tensor] = None,
                            device="cuda:0", requires_grad=True):
        if tensor_x is not None:
            self.particle_x = tensor_x.detach().to(self.device, DTYPE)
        if tensor_velocity is not None:
            self.particle_v = tensor_velocity.detach().to(self.device, DTYPE)
        if tensor_F is not None:
            _f9_pack(self._F_trial, tensor_F.detach().to(self.device, DTYPE))
        if tensor_C is not None:
            _f9_pack(self._C, tensor_C.detach().to(self.device, DTYPE))

    def set_require_grad(self, requires_grad=True):
        self.requires_grad = requires_grad

    def reset_density(self, tensor_density: Tensor, selection_mask: Optional[Tensor] = None, device="cuda:0",
                      requires_grad=True, update_mass=False):
        dens = tensor_density.detach().to(self.device, DTYPE).reshape(-1)
        if selection_mask is not None:
            m = selection_mask.to(self.device).to(torch.int32) == 1
            self.particle_density[m] = dens[m]
        else:
            self.particle_density.copy_(dens)
        if update_mass:
            self.update_mass()

    def update_mass(self):
        """mass = density * vol (get_float_array_product, mpm_data_structure.py:719-726)."""
        N.check(N.lib().empm_prepare(None, None, None, None, None, self.particle_density.data_ptr(),
                                     self.particle_vol.data_ptr(), self._x4.data_ptr(), self.n_particles,
                                     _stream_ptr(self.device)))

    def set_selection(self, selection: Tensor):
        """Set particle_selection (0 = simulated); the kernels skip the rest."""
        self.particle_selection.copy_(selection.to(self.device, torch.int32).reshape(-1))
        self._has_selection = bool((self.particle_selection != 0).any().item())

    def partial_clone(self, device="cuda:0", requires_grad=True):
        new = MPMStateStruct()
        new.init(self.n_particles, device=self.device, requires_grad=requires_grad)
        new.particle_vol.copy_(self.particle_vol)
        new.particle_density.copy_(self.particle_density)
        new._x4[:, 3].copy_(self._x4[:, 3])
        new.particle_selection.copy_(self.particle_selection)
        new._has_selection = self._has_selection
        new.init_grid(self.grid_res)
        _f9_identity(new._F_trial, self.n_particles)
        new.set_require_grad(requires_grad)
        return new


class MPMModelStruct:
    """Material model (mpm_data_structure.py:390-498)."""

    def __init__(self):
        self.grid_lim = 1.0
        self.n_particles = 0
        self.n_grid = 100
        self.dx = 0.01
        self.inv_dx = 100.0
        self.grid_dim_x = self.grid_dim_y = self.grid_dim_z = 100
        self.material = 0
        self.friction_angle = 25.0
        self.alpha = 0.0
        self.gravitational_accelaration = (0.0, 0.0, 0.0)
        self.hardening = 0.0
        self.xi = 0.0
        self.plastic_viscosity = 0.0
        self.softening = 0.1
        self.rpic_damping = 0.0
        self.grid_v_damping_scale = 1.1
        self.update_cov_with_F = 0
        self.device = None

    def init(self, shape: Union[Sequence[int], int], device="cuda:0", requires_grad=False) -> None:
        n = int(shape if isinstance(shape, int) else shape[0])
        d = _dev(device)
        self.device = d
        self.n_particles = n
        self.E = torch.zeros(n, dtype=DTYPE, device=d)
        self.nu = torch.zeros(n, dtype=DTYPE, device=d)
        self.mu = torch.zeros(n, dtype=DTYPE, device=d)
        self.lam = torch.zeros(n, dtype=DTYPE, device=d)
        self.yield_stress = torch.zeros(n, dtype=DTYPE, device=d)
        self.requires_grad = requires_grad

    def finalize_mu_lam(self, n_particles, device="cuda:0"):
        N.check(N.lib().empm_prepare(None, self.E.data_ptr(), self.nu.data_ptr(), self.mu.data_ptr(),
                                     self.lam.data_ptr(), None, None, None, int(n_particles),
                                     _stream_ptr(self.device)))

    def init_other_params(self, n_grid=100, grid_lim=1.0, device="cuda:0"):
        self.grid_lim = grid_lim
        self.n_grid = n_grid
        self.grid_dim_x = self.grid_dim_y = self.grid_dim_z = n_grid
        self.dx, self.inv_dx = self.grid_lim / self.n_grid, float(n_grid / grid_lim)
        self.update_cov_with_F = False
        self.material = 0
        self.plastic_viscosity = 0.0
        self.softening = 0.1
        self.friction_angle = 25.0
        sin_phi = math.sin(self.friction_angle / 180.0 * 3.14159265)
        self.alpha = math.sqrt(2.0 / 3.0) * 2.0 * sin_phi / (3.0 - sin_phi)
        self.gravitational_accelaration = (0.0, 0.0, 0.0)
        self.rpic_damping = 0.0
        self.grid_v_damping_scale = 1.1

    def from_torch(self, tensor_E: Tensor, tensor_nu: Tensor, device="cuda:0", requires_grad=False):
        self.E = tensor_E.detach().to(self.device or _dev(device), DTYPE).contiguous().clone()
        self.nu = tensor_nu.detach().to(self.E.device, DTYPE).contiguous().clone()
        self.finalize_mu_lam(n_particles=tensor_E.shape[0], device=device)

    def set_require_grad(self, requires_grad=True):
        self.requires_grad = requires_grad

    def _params(self) -> N.EmpmModelParams:
        p = N.EmpmModelParams()
        p.n_grid = int(self.n_grid)
        p.grid_lim = float(self.grid_lim)
        p.material = int(self.material)
        g = tuple(float(t) for t in self.gravitational_accelaration)
        p.gravity = N.F3(*g)
        p.rpic_damping = float(self.rpic_damping)
        p.grid_v_damping_scale = float(self.grid_v_damping_scale)
        p.softening = float(self.softening)
        p.hardening = float(self.hardening)
        p.xi = float(self.xi)
        p.plastic_viscosity = float(self.plastic_viscosity)
        p.alpha = float(self.alpha)
        return p


def _vec3(v, default=(0.0, 0.0, 0.0)):
    if v is None:
        return tuple(default)
    if isinstance(v, (int, float)):
        return (float(v),) * 3
    if isinstance(v, Tensor):
        v = v.detach().cpu().tolist()
    return tuple(float(t) for t in v)


class Dirichlet_collider:
    """Grid boundary-condition parameters (mpm_data_structure.py:502-537).

    Fields keep the reference's names and are read by the solver before each
    substep, so callers may mutate ``point``, ``velocity``, ``active`` ... between
    substeps as the reference's frame callbacks do.
    """

    def __init__(self):
        self.point = (0.0, 0.0, 0.0)
        self.normal = (0.0, 0.0, 0.0)
        self.direction = (0.0, 0.0, 0.0)
        self.start_time = 0.0
        self.end_time = 0.0
        self.active = False
        self.friction = 0.0
        self.surface_type = 0
        self.velocity = (0.0, 0.0, 0.0)
        self.angular_velocity = 0.0
        self.rot_axis = (0.0, 0.0, 0.0)
        self.threshold = 0.0
        self.reset = 0
        self.index = 0
        self.radius = 0.0
        self.size = (0.0, 0.0, 0.0)
        self.half_height = 0.0
        self.half_height_and_radius = (0.0, 0.0)
        # library-side identity of the closure this parameter block belongs to
        self._kind = 0
        self._shape = 0


class GridCollider:
    """enforce_grid_velocity_by_mask parameters (mpm_data_structure.py:540-548)."""

    def __init__(self):
        self.point = (0.0, 0.0, 0.0)
        self.normal = (0.0, 0.0, 0.0)
        self.direction = (0.0, 0.0, 0.0)
        self.start_time = 0.0
        self.end_time = 0.0
        self.mask = None
        self._kind = N.COLL_GRID_MASK
        self._shape = 0


class Impulse_modifier:
    """Particle impulse parameters (mpm_data_structure.py:551-564)."""

    def __init__(self):
        self.point = (0.0, 0.0, 0.0)
        self.normal = (0.0, 0.0, 0.0)
        self.start_time = 0.0
        self.end_time = 0.0
        self.force = (0.0, 0.0, 0.0)
        self.forceTimesDt = (0.0, 0.0, 0.0)
        self.numsteps = 0
        self.size = (0.0, 0.0, 0.0)
        self.mask = None
        self._kind = N.MOD_IMPULSE


class ParticleVelocityModifier:
    """Particle velocity modifier parameters (mpm_data_structure.py:602-621)."""

    def __init__(self):
        self.point = (0.0, 0.0, 0.0)
        self.normal = (0.0, 0.0, 0.0)
        self.half_height_and_radius = (0.0, 0.0)
        self.rotation_scale = 0.0
        self.translation_scale = 0.0
        self.size = (0.0, 0.0, 0.0)
        self.horizontal_axis_1 = (0.0, 0.0, 0.0)
        self.horizontal_axis_2 = (0.0, 0.0, 0.0)
        self.start_time = 0.0
        self.end_time = 0.0
        self.velocity = (0.0, 0.0, 0.0)
        self.mask = None
        self._kind = N.MOD_SET_VELOCITY
        # set_particle_mover extras
        self.rotation_axis = (0.0, 0.0, 0.0)
        self.rotation_center = (0.0, 0.0, 0.0)
        self.angular_velocity = 0.0


def compute_mu_lam_from_E_nu_clean(mu: Tensor, lam: Tensor, E: Tensor, nu: Tensor):
    """mu, lam from E, nu on the device (mpm_data_structure.py:624-633)."""
    N.check(N.lib().empm_prepare(None, E.data_ptr(), nu.data_ptr(), mu.data_ptr(), lam.data_ptr(), None, None,
                                 None, E.shape[0], _stream_ptr(E.device)))
