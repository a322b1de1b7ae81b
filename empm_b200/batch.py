"""Batched simulation of independent MPM instances in one launch sequence.

The reference evaluates a CMA-ES population one candidate at a time
(phys_sim/engine/trainer_warp_mpm.py:598-661): a full re-initialisation and
a serial ``advance_to`` per candidate. ``BatchedMPM`` keeps every member's
particles resident in one set of concatenated buffers (instance i at
[poff_i, poff_i + n_i)) and advances all of them with the same three kernels
per substep; rollouts run in CUDA-graph-captured blocks of substeps.

Per-instance boundary conditions are registered with the same factories as
``MPMWARPDiff`` (one solver object per instance holds the collider list and
builds that instance's step schedules).
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _native as N
from .mpm_data_structure import DTYPE, _f9_identity, _f9_pack, _f9_unpack, _stream_ptr
from .mpm_solver_diff import MATERIALS, MPMWARPDiff


@dataclass
class InstanceSpec:
    """One simulation instance of a batch (arrays on the host or device)."""
    x: np.ndarray
    vol: np.ndarray
    rho: np.ndarray
    E: np.ndarray
    nu: np.ndarray
    n_grid: int
    v: Optional[np.ndarray] = None
    yield_stress: Optional[np.ndarray] = None
    material: str = "jelly"
    grid_lim: float = 1.0
    gravity: Sequence[float] = (0.0, -9.8, 0.0)
    softening: float = 0.1
    hardening: float = 0.0
    xi: float = 0.0
    plastic_viscosity: float = 0.0
    friction_angle: float = 25.0
    rpic_damping: float = 0.0
    grid_v_damping_scale: float = 1.1
    colliders: List[dict] = field(default_factory=list)

    @property
    def n(self) -> int:
        return int(self.x.shape[0])


def register_colliders(solver: MPMWARPDiff, specs: List[dict]) -> None:
    """Register collider descriptions (dicts with a "kind") on a solver."""
    for c in specs:
        k = c["kind"]
        if k == "surface":
            solver.add_surface_collider(c["point"], c["normal"], c.get("surface", "sticky"), c.get("friction", 0.0),
                                        c.get("start_time", 0.0), c.get("end_time", 999.0))
        elif k == "cuboid":
            solver.set_velocity_on_cuboid(c["point"], c["size"], c["velocity"], c.get("start_time", 0.0),
                                          c.get("end_time", 999.0), c.get("reset", 0))
        elif k == "bbox":
            solver.add_bounding_box(c.get("start_time", 0.0), c.get("end_time", 999.0))
        elif k == "geometry":
            solver.add_geometry_collider({a: b for a, b in c.items() if a != "kind"})
        elif k == "grid_velocity":
            solver.set_grid_velocity_on_geometry({a: b for a, b in c.items() if a != "kind"})
        else:
            raise ValueError(f"unknown collider kind {k!r}")


def _params(spec: InstanceSpec) -> N.EmpmModelParams:
    if spec.material not in MATERIALS:
        raise TypeError("Undefined material type")
    p = N.EmpmModelParams()
    p.n_grid = int(spec.n_grid)
    p.grid_lim = float(spec.grid_lim)
    p.material = MATERIALS[spec.material]
    p.gravity = N.F3(*[float(g) for g in spec.gravity])
    p.rpic_damping = float(spec.rpic_damping)
    p.grid_v_damping_scale = float(spec.grid_v_damping_scale)
    p.softening = float(spec.softening)
    p.hardening = float(spec.hardening)
    p.xi = float(spec.xi)
    p.plastic_viscosity = float(spec.plastic_viscosity)
    sin_phi = math.sin(spec.friction_angle / 180.0 * 3.14159265)
    p.alpha = math.sqrt(2.0 / 3.0) * 2.0 * sin_phi / (3.0 - sin_phi)
    return p


class BatchedMPM:
    def __init__(self, instances: List[InstanceSpec], device="cuda:0", max_steps: int = 64):
        if not instances:
            raise ValueError("a batch needs at least one instance")
        self.device = torch.device(device)
        self.specs = list(instances)
        self.n_inst = len(instances)
        self.counts = [s.n for s in instances]
        self.poff = np.concatenate([[0], np.cumsum(self.counts)[:-1]]).astype(np.int64)
        self.n = int(sum(self.counts))
        n, dev = self.n, self.device
        self._x4 = [torch.zeros((n, 4), dtype=DTYPE, device=dev) for _ in range(2)]
        self._v4 = [torch.zeros((n, 4), dtype=DTYPE, device=dev) for _ in range(2)]
        self._C = [torch.zeros(9 * n, dtype=DTYPE, device=dev) for _ in range(2)]
        self._F = [torch.zeros(9 * n, dtype=DTYPE, device=dev) for _ in range(2)]
        self._Fe = torch.zeros(9 * n, dtype=DTYPE, device=dev)
        self.vol = torch.zeros(n, dtype=DTYPE, device=dev)
        self.density = torch.zeros(n, dtype=DTYPE, device=dev)
        self.E = torch.zeros(n, dtype=DTYPE, device=dev)
        self.nu = torch.zeros(n, dtype=DTYPE, device=dev)
        self.mu = torch.zeros(n, dtype=DTYPE, device=dev)
        self.lam = torch.zeros(n, dtype=DTYPE, device=dev)
        self.yield_stress = torch.zeros(n, dtype=DTYPE, device=dev)
        self.cur = 0
        self.time = 0.0
        self.use_graph = True
        self.resume_blocks = True   # blocks continue from the library's sorted state (empm_rollout_ex)
        self.sort_every = 32
        self.p2g_mode = 2
        self.g2p_tile = False
        self.tile_cap = 1024
        self.seg_cap = 4           # warp-aggregated P2G: longest same-cell run per reduction
        self.fuse = True           # fused G2P + stress + P2G between cell sorts
        self._opts = {}
        # per-instance collider lists / schedule builders
        self.solvers = []
        for s in instances:
            sv = MPMWARPDiff()
            sv.initialize(s.n, n_grid=s.n_grid, grid_lim=s.grid_lim, device=device)
            register_colliders(sv, s.colliders)
            self.solvers.append(sv)
        params = (N.EmpmModelParams * self.n_inst)(*[_params(s) for s in instances])
        counts = (ctypes.c_int * self.n_inst)(*self.counts)
        self.L = N.lib()
        ptr = ctypes.c_void_p()
        with torch.cuda.device(dev):
            N.check(self.L.empm_batch_create(params, counts, self.n_inst, max_steps, ctypes.byref(ptr)))
        self.ptr = ptr
        self._static = None
        self.load_state()

    # -- state ----------------------------------------------------------------
    def _sl(self, i):
        return slice(int(self.poff[i]), int(self.poff[i]) + self.counts[i])

    def load_state(self, instances: Optional[Sequence[int]] = None):
        """(Re)load positions, velocities and materials of the given instances
        (all by default) from their specs; C = 0, F = I."""
        idx = range(self.n_inst) if instances is None else instances
        dev = self.device
        b = self.cur
        for i in idx:
            s = self.specs[i]
            sl = self._sl(i)
            t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=DTYPE).to(dev, non_blocking=True)  # noqa
            self._x4[b][sl, :3] = t(s.x)
            self._v4[b][sl, :3] = t(s.v) if s.v is not None else 0.0
            self._v4[b][sl, 3] = 0.0
            self.vol[sl] = t(s.vol)
            self.density[sl] = t(s.rho)
            self.E[sl] = t(s.E)
            self.nu[sl] = t(s.nu)
            self.yield_stress[sl] = t(s.yield_stress) if s.yield_stress is not None else 0.0
        # C = 0 and F = I for the whole batch (per-instance planes are strided)
        if instances is None:
            self._C[b].zero_()
            _f9_identity(self._F[b], self.n)
        else:
            C = _f9_unpack(self._C[b], self.n).clone()
            F = _f9_unpack(self._F[b], self.n).clone()
            for i in idx:
                sl = self._sl(i)
                C[sl] = 0.0
                F[sl] = torch.eye(3, device=dev)
            _f9_pack(self._C[b], C)
            _f9_pack(self._F[b], F)
        self.prepare()

    def prepare(self):
        """mu, lam from E, nu and mass = density * vol for the whole batch."""
        N.check(self.L.empm_prepare(self.ptr, self.E.data_ptr(), self.nu.data_ptr(), self.mu.data_ptr(),
                                    self.lam.data_ptr(), self.density.data_ptr(), self.vol.data_ptr(),
                                    self._x4[self.cur].data_ptr(), self.n, _stream_ptr(self.device)), self.ptr)

    def set_material(self, i: int, E=None, nu=None, yield_stress=None):
        """Per-instance material (scalars or arrays); call prepare() after."""
        sl = self._sl(i)
        for name, val in (("E", E), ("nu", nu), ("yield_stress", yield_stress)):
            if val is not None:
                dst = getattr(self, name)
                dst[sl] = torch.as_tensor(val, dtype=DTYPE).to(self.device) if not isinstance(val, float) else val

    def positions(self, i: Optional[int] = None) -> torch.Tensor:
        x = self._x4[self.cur][:, :3]
        return x if i is None else x[self._sl(i)]

    def velocities(self, i: Optional[int] = None) -> torch.Tensor:
        v = self._v4[self.cur][:, :3]
        return v if i is None else v[self._sl(i)]

    def F_trial(self) -> torch.Tensor:
        return _f9_unpack(self._F[self.cur], self.n)

    # -- schedule -------------------------------------------------------------
    def _is_static(self) -> bool:
        for sv in self.solvers:
            if any(m is not None for m in sv.modify_bc):
                return False
            for p in sv.collider_params:
                if float(p.start_time) > 0.0 or float(p.end_time) < 999.0:
                    return False
            if sv.impulse_params or sv.particle_velocity_modifier_params:
                return False
        return True

    def _schedule(self, dt: float, n_steps: int):
        if self._is_static():
            if self._static is None or self._static[0] != dt:
                table = (N.EmpmStep * self.n_inst)()
                for i, sv in enumerate(self.solvers):
                    sv._fill_step(table[i], 0.0, dt)
                self._static = (dt, table)
            return self._static[1], 1
        table = (N.EmpmStep * (n_steps * self.n_inst))()
        for i, sv in enumerate(self.solvers):
            sv._check_masks()
            t = self.time
            for s in range(n_steps):
                sv._fill_step(table[s * self.n_inst + i], t, dt)
                sv._modify(t, dt)
                t = t + dt
        return table, n_steps

    def _apply_options(self):
        opts = {N.OPT_SORT_EVERY: int(self.sort_every), N.OPT_P2G_MODE: int(self.p2g_mode),
                N.OPT_G2P_TILE: int(bool(self.g2p_tile)), N.OPT_TILE_CAP: int(self.tile_cap),
                N.OPT_SEG_CAP: int(self.seg_cap), N.OPT_FUSE: int(bool(self.fuse))}
        for k, v in opts.items():
            if self._opts.get(k) != v:
                N.check(self.L.empm_ctx_set_option(self.ptr, k, v), self.ptr)
        self._opts = opts

    def _views(self, b):
        return N.EmpmParticles(self._x4[b].data_ptr(), self._v4[b].data_ptr(), self._C[b].data_ptr(),
                               self._F[b].data_ptr())

    def rollout(self, dt: float, n_steps: int, block: int = 50):
        """Advance every instance by n_steps substeps, `block` substeps per
        library call (one CUDA graph per block). With ``resume_blocks`` the
        blocks after the first continue from the library's cell-sorted state
        and only the last writes the particles back in their own order."""
        self._apply_options()
        mat = N.EmpmMaterial(self.vol.data_ptr(), self.mu.data_ptr(), self.lam.data_ptr(),
                             self.yield_stress.data_ptr(), None, self._Fe.data_ptr())
        done = 0
        stream = _stream_ptr(self.device)
        while done < n_steps:
            k = min(block, n_steps - done)
            table, n_tables = self._schedule(dt, k)
            a, b = self._views(self.cur), self._views(1 - self.cur)
            flags = block_flags(done, k, n_steps, self.use_graph, self.resume_blocks)
            with torch.cuda.device(self.device):
                N.check(self.L.empm_rollout_ex(self.ptr, a, b, mat, table, n_tables, k, flags, stream), self.ptr)
            if k % 2 == 1:
                self.cur = 1 - self.cur
            for _ in range(k):
                self.time = self.time + dt
            done += k

    def read_status(self) -> int:
        s = ctypes.c_uint32(0)
        N.check(self.L.empm_read_status(self.ptr, ctypes.byref(s), _stream_ptr(self.device)), self.ptr)
        return int(s.value)

    def kernel_timing(self, enable: bool, max_launches: int = 4096):
        N.check(self.L.empm_ctx_timing(self.ptr, int(enable), int(max_launches)), self.ptr)

    def kernel_times(self):
        """{kernel: (total_ms, launches)} for [stress_p2g, grid_update, g2p, g2p2g]."""
        return N.kernel_times(self.L, self.ptr)

    def __del__(self):
        try:
            if getattr(self, "ptr", None):
                self.L.empm_ctx_destroy(self.ptr)
                self.ptr = None
        except Exception:
            pass


def block_flags(done: int, k: int, n_steps: int, use_graph: bool, resume: bool) -> int:
    """empm_rollout_ex flags of the block of k substeps that starts after
    `done` of a rollout of n_steps: a graph when asked; with `resume`, every
    block but the first continues from the library's sorted state and every
    block but the last keeps its result there."""
    flags = N.ROLLOUT_GRAPH if use_graph else 0
    if resume:
        if done > 0:
            flags |= N.ROLLOUT_RESUME
        if done + k < n_steps:
            flags |= N.ROLLOUT_KEEP
    return flags


def single_instance(spec: InstanceSpec, device="cuda:0"):
    """(solver, model, state) of the reference-facing single-instance API for
    one instance spec: what a caller of MPMWARPDiff builds for one simulation."""
    from .mpm_data_structure import MPMModelStruct, MPMStateStruct

    dev = torch.device(device)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)  # noqa: E731
    n = spec.n
    st = MPMStateStruct()
    st.init(n, device=dev)
    st.from_torch(t(spec.x), t(spec.vol), None, t(spec.v) if spec.v is not None else None, n_grid=spec.n_grid,
                  grid_lim=spec.grid_lim, device=dev)
    st.reset_density(t(spec.rho), update_mass=True)
    md = MPMModelStruct()
    md.init(n, device=dev)
    md.init_other_params(n_grid=spec.n_grid, grid_lim=spec.grid_lim)
    md.gravitational_accelaration = tuple(spec.gravity)
    sv = MPMWARPDiff()
    sv.initialize(n, n_grid=spec.n_grid, grid_lim=spec.grid_lim, device=dev)
    sv.set_parameters_dict(md, st, {"material": spec.material, "softening": spec.softening,
                                    "plastic_viscosity": spec.plastic_viscosity,
                                    "friction_angle": spec.friction_angle, "rpic_damping": spec.rpic_damping,
                                    "grid_v_damping_scale": spec.grid_v_damping_scale})
    md.E.copy_(t(spec.E))
    md.nu.copy_(t(spec.nu))
    md.finalize_mu_lam(n)
    if spec.yield_stress is not None:
        md.yield_stress.copy_(t(spec.yield_stress))
    register_colliders(sv, spec.colliders)
    return sv, md, st
