"""CPU oracle for the MLS-MPM substep — TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import this module; it is the
checker, never the product path.

Parity status: the reference (EMPM, NVIDIA Warp 1.8.1) cannot run here
because Warp is not installable offline. The C restatement in
``mpm_oracle.c`` is pinned instead against golden vectors produced by running
the reference's *own* kernel source (phys_sim/diff_simulator/warp_mpm/
mpm_utils.py, mpm_solver_diff.py, mpm_data_structure.py) in FP64 under a
NumPy stand-in for the Warp runtime (``tests/golden/make_golden.py``), and
against physics known-answer tests. Warp's own GPU kernels and svd3 were
never run, so parity with them is unpinned.

The host-side orchestration below restates ``MPMWARPDiff.p2g2p_differentiable``
(mpm_solver_diff.py:165-291): time gates of every collider closure, the
``modify`` callbacks that move kinematic colliders after each substep
(:795-801, :860-866), and ``time += dt``.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")

# kinds shared with the library's numbering (see include/empm_b200.h)
SURFACE, GEOMETRY, GRID_VELOCITY, CUBOID_VELOCITY, BOUNDING_BOX, GRID_MASK = 1, 2, 3, 4, 5, 6
CUBE, SPHERE, CYLINDER, HALFSPACE = 1, 2, 3, 4
MOD_IMPULSE, MOD_IMPULSE_MASK, MOD_SET_VELOCITY, MOD_ROTATION, MOD_MOVER = 1, 2, 3, 4, 5


def build() -> None:
    """Compile the oracle libraries (gcc; see build_oracle.sh)."""
    import subprocess

    subprocess.run(["bash", os.path.join(_HERE, "build_oracle.sh")], check=True)


def _lib_struct(real):
    class OrModel(ctypes.Structure):
        _fields_ = [
            ("G", ctypes.c_int), ("grid_lim", real), ("dx", real), ("inv_dx", real),
            ("material", ctypes.c_int), ("gravity", real * 3),
            ("rpic_damping", real), ("grid_v_damping_scale", real),
            ("softening", real), ("hardening", real), ("xi", real),
            ("plastic_viscosity", real), ("alpha", real), ("pred32", ctypes.c_int),
        ]

    class OrCollider(ctypes.Structure):
        _fields_ = [
            ("kind", ctypes.c_int), ("gate", ctypes.c_int), ("shape", ctypes.c_int), ("surface_type", ctypes.c_int),
            ("point", real * 3), ("normal", real * 3), ("size", real * 3), ("velocity", real * 3),
            ("rot_axis", real * 3), ("angular_velocity", real), ("radius", real), ("half_height", real),
            ("friction", real), ("mask", ctypes.c_void_p),
        ]

    class OrModifier(ctypes.Structure):
        _fields_ = [
            ("kind", ctypes.c_int), ("gate", ctypes.c_int), ("vec", real * 3), ("point", real * 3),
            ("normal", real * 3), ("axis1", real * 3), ("axis2", real * 3), ("scale", real * 2),
            ("mask", ctypes.c_void_p),
        ]

    return OrModel, OrCollider, OrModifier


class _Lib:
    def __init__(self, path: str, real, np_real):
        if not os.path.exists(path):
            build()
        self.lib = ctypes.CDLL(path)
        self.real = real
        self.np_real = np_real
        self.OrModel, self.OrCollider, self.OrModifier = _lib_struct(real)
        P = ctypes.c_void_p
        M = ctypes.POINTER(self.OrModel)
        L = self.lib
        L.or_substep.argtypes = [M, ctypes.c_int] + [P] * 20 + [ctypes.c_int, P, ctypes.c_int, real]
        L.or_stress.argtypes = [M, ctypes.c_int, P, P, P, P, P, real, P, P]
        L.or_p2g.argtypes = [M, ctypes.c_int, P, P, P, P, P, P, P, real, P, P]
        L.or_grid_update.argtypes = [M, P, P, P, P, ctypes.c_int, real]
        L.or_g2p.argtypes = [M, ctypes.c_int, P, P, P, P, real, P, P, P, P]
        L.or_svd3.argtypes = [P, P, P, P]
        L.or_mu_lam.argtypes = [ctypes.c_int, P, P, P, P]
        L.or_restart.argtypes = [M, ctypes.c_int, P, P, P, P, P, P, P]
        L.or_num_threads.restype = ctypes.c_int
        for f in ("or_substep", "or_stress", "or_p2g", "or_grid_update", "or_g2p", "or_svd3", "or_mu_lam",
                  "or_restart"):
            getattr(L, f).restype = None


_LIBS = {}


def lib(precision: str = "fp64") -> _Lib:
    if precision not in _LIBS:
        if precision == "fp64":
            _LIBS[precision] = _Lib(os.path.join(_BUILD, "liboracle64.so"), ctypes.c_double, np.float64)
        elif precision == "fp32_omp":
            _LIBS[precision] = _Lib(os.path.join(_BUILD, "liboracle32_omp.so"), ctypes.c_float, np.float32)
        elif precision == "fp64_omp":
            _LIBS[precision] = _Lib(os.path.join(_BUILD, "liboracle64_omp.so"), ctypes.c_double, np.float64)
        else:
            raise ValueError(precision)
    return _LIBS[precision]


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def svd3(A: np.ndarray, precision: str = "fp64"):
    L = lib(precision)
    A = np.ascontiguousarray(A, dtype=L.np_real).reshape(3, 3)
    U = np.zeros((3, 3), L.np_real); s = np.zeros(3, L.np_real); V = np.zeros((3, 3), L.np_real)
    L.lib.or_svd3(_ptr(A), _ptr(U), _ptr(s), _ptr(V))
    return U, s, V


def stress(material: int, F_trial: np.ndarray, mu: np.ndarray, lam: np.ndarray, ys: np.ndarray, dt: float,
           softening: float = 0.1, hardening: float = 0.0, xi: float = 0.0, plastic_viscosity: float = 0.0,
           alpha: float = 0.0, precision: str = "fp64"):
    """Return map + Kirchhoff stress of n particles (compute_stress_from_F_trial,
    mpm_utils.py:602-665). Returns (F_elastic [n,9], stress [n,9], mu', lam', ys')."""
    L = lib(precision)
    R = L.np_real
    n = F_trial.shape[0]
    Ft = np.ascontiguousarray(F_trial, dtype=R).reshape(n, 9)
    mu = np.array(mu, dtype=R).reshape(n)
    lam = np.array(lam, dtype=R).reshape(n)
    ys = np.array(ys, dtype=R).reshape(n)
    Fe = np.zeros((n, 9), R)
    S = np.zeros((n, 9), R)
    m = L.OrModel()
    m.material = int(material)
    m.softening, m.hardening, m.xi = softening, hardening, xi
    m.plastic_viscosity, m.alpha = plastic_viscosity, alpha
    L.lib.or_stress(ctypes.byref(m), n, None, _ptr(Ft), _ptr(mu), _ptr(lam), _ptr(ys), R(dt), _ptr(Fe), _ptr(S))
    return Fe, S, mu, lam, ys


def restart(G: int, x: np.ndarray, mass: np.ndarray, target: np.ndarray, selection=None, grid_lim: float = 1.0,
            precision: str = "fp64", cov=None):
    """F_trial and positions after MPMWARPDiff.restart_and_compute_F_C.
    Returns (F_trial [n, 3, 3], x [n, 3]), plus the updated packed covariances
    [n, 6] when cov is given (update_cov_with_F)."""
    L = lib(precision)
    R = L.np_real
    n = x.shape[0]
    xs = np.ascontiguousarray(x, dtype=R).reshape(n, 3).copy()
    ms = np.ascontiguousarray(mass, dtype=R).reshape(n)
    tg = np.ascontiguousarray(target, dtype=R).reshape(n, 3)
    Ft = np.tile(np.eye(3, dtype=R).reshape(1, 9), (n, 1))
    m = L.OrModel()
    m.G, m.grid_lim, m.dx, m.inv_dx = int(G), grid_lim, grid_lim / G, float(G / grid_lim)
    sel = None if selection is None else np.ascontiguousarray(selection, dtype=np.int32)
    gm = np.zeros(G ** 3, R)
    gv = np.zeros(3 * G ** 3, R)
    cv = None if cov is None else np.ascontiguousarray(cov, dtype=R).reshape(n, 6).copy()
    L.lib.or_restart(ctypes.byref(m), n, _ptr(sel), _ptr(xs), _ptr(ms), _ptr(tg), _ptr(Ft), _ptr(gm), _ptr(gv),
                     _ptr(cv))
    if cv is not None:
        return Ft.reshape(n, 3, 3), xs, cv
    return Ft.reshape(n, 3, 3), xs


@dataclass
class OrColliderSpec:
    """One collider in registration order (fields as in Dirichlet_collider)."""
    kind: int
    shape: int = 0
    surface_type: int = 0
    point: tuple = (0.0, 0.0, 0.0)
    normal: tuple = (0.0, 0.0, 0.0)
    size: tuple = (0.0, 0.0, 0.0)
    velocity: tuple = (0.0, 0.0, 0.0)
    rot_axis: tuple = (1.0, 0.0, 0.0)
    angular_velocity: float = 0.0
    radius: float = 0.0
    half_height: float = 0.0
    friction: float = 0.0
    start_time: float = 0.0
    end_time: float = 999.0
    active: bool = True
    reset: int = 0
    mask: Optional[np.ndarray] = None   # int32 [G^3] for GRID_MASK


@dataclass
class OrModifierSpec:
    kind: int
    vec: tuple = (0.0, 0.0, 0.0)
    point: tuple = (0.0, 0.0, 0.0)
    normal: tuple = (0.0, 0.0, 0.0)
    axis1: tuple = (0.0, 0.0, 0.0)
    axis2: tuple = (0.0, 0.0, 0.0)
    scale: tuple = (0.0, 0.0)
    start_time: float = 0.0
    end_time: float = 999.0
    mask: Optional[np.ndarray] = None   # int32 [N]


class OracleSim:
    """Whole-rollout oracle: reference state semantics on the host, C kernels."""

    def __init__(self, x, v, vol, mass, E, nu, *, n_grid, grid_lim=1.0, material=0, gravity=(0.0, 0.0, 0.0),
                 yield_stress=None, softening=0.1, hardening=0.0, xi=0.0, plastic_viscosity=0.0,
                 friction_angle=25.0, rpic_damping=0.0, grid_v_damping_scale=1.1, selection=None,
                 precision="fp64", collider_f32=False):
        """collider_f32: keep the collider state as the reference's Warp
        structs keep it, in float32 (kinematic collider points are rounded to
        float32 after every move, mpm_solver_diff.py:795-801, 860-866), and
        evaluate the inside tests on float32 offsets (OrModel.pred32). The
        default keeps both in the oracle's precision."""
        self.L = lib(precision)
        R = self.L.np_real
        n = x.shape[0]
        self.n = n
        self.G = int(n_grid)
        self.x = np.ascontiguousarray(x, dtype=R).reshape(n, 3).copy()
        self.v = np.ascontiguousarray(v, dtype=R).reshape(n, 3).copy()
        self.C = np.zeros((n, 9), R)
        self.F_trial = np.tile(np.eye(3, dtype=R).reshape(1, 9), (n, 1))
        self.F = np.zeros((n, 9), R)
        self.stress = np.zeros((n, 9), R)
        self.vol = np.ascontiguousarray(vol, dtype=R).reshape(n).copy()
        self.mass = np.ascontiguousarray(mass, dtype=R).reshape(n).copy()
        E = np.broadcast_to(np.asarray(E, dtype=R), (n,)).copy()
        nu = np.broadcast_to(np.asarray(nu, dtype=R), (n,)).copy()
        self.mu = np.zeros(n, R); self.lam = np.zeros(n, R)
        self.L.lib.or_mu_lam(n, _ptr(E), _ptr(nu), _ptr(self.mu), _ptr(self.lam))
        self.ys = np.zeros(n, R) if yield_stress is None else np.broadcast_to(np.asarray(yield_stress, R), (n,)).copy()
        self.sel = None if selection is None else np.ascontiguousarray(selection, dtype=np.int32)
        self.time = 0.0
        sin_phi = np.sin(friction_angle / 180.0 * 3.14159265)
        alpha = np.sqrt(2.0 / 3.0) * 2.0 * sin_phi / (3.0 - sin_phi)
        m = self.L.OrModel()
        m.G = self.G
        m.grid_lim = grid_lim
        m.dx = grid_lim / self.G
        m.inv_dx = float(self.G / grid_lim)
        m.material = material
        m.gravity = (self.L.real * 3)(*gravity)
        m.rpic_damping = rpic_damping
        m.grid_v_damping_scale = grid_v_damping_scale
        m.softening = softening
        m.hardening = hardening
        m.xi = xi
        m.plastic_viscosity = plastic_viscosity
        m.alpha = alpha
        m.pred32 = 1 if collider_f32 else 0
        self.collider_f32 = bool(collider_f32)
        self.model = m
        g3 = self.G ** 3
        self.grid_m = np.zeros(g3, R)
        self.grid_v_in = np.zeros(3 * g3, R)
        self.grid_v_out = np.zeros(3 * g3, R)
        self.colliders: List[OrColliderSpec] = []
        self.modifiers: List[OrModifierSpec] = []

    # --- host-side gates (closures of mpm_solver_diff.py) -------------------
    def _collider_gate(self, c: OrColliderSpec, dt: float) -> int:
        t = self.time
        in_window = c.start_time <= t < c.end_time
        if c.kind in (SURFACE, CUBOID_VELOCITY, BOUNDING_BOX):
            if in_window:
                return 1
        elif c.kind in (GEOMETRY, GRID_VELOCITY):
            if in_window and c.active:
                return 1
        elif c.kind == GRID_MASK:
            return 1
        if c.kind in (GRID_VELOCITY, CUBOID_VELOCITY) and c.reset == 1 and t < c.end_time + 15.0 * dt:
            return 2
        return 0

    def _tables(self, dt: float):
        L = self.L
        nc, nm = len(self.colliders), len(self.modifiers)
        coll = (L.OrCollider * max(nc, 1))()
        for i, c in enumerate(self.colliders):
            o = coll[i]
            o.kind, o.gate, o.shape, o.surface_type = c.kind, self._collider_gate(c, dt), c.shape, c.surface_type
            for f in ("point", "normal", "size", "velocity", "rot_axis"):
                setattr(o, f, (L.real * 3)(*getattr(c, f)))
            o.angular_velocity, o.radius, o.half_height, o.friction = c.angular_velocity, c.radius, c.half_height, c.friction
            o.mask = None if c.mask is None else c.mask.ctypes.data
        mods = (L.OrModifier * max(nm, 1))()
        for i, md in enumerate(self.modifiers):
            o = mods[i]
            o.kind = md.kind
            o.gate = 1 if md.start_time <= self.time < md.end_time else 0
            for f in ("vec", "point", "normal", "axis1", "axis2"):
                setattr(o, f, (L.real * 3)(*getattr(md, f)))
            o.scale = (L.real * 2)(*md.scale)
            o.mask = None if md.mask is None else md.mask.ctypes.data
        return coll, nc, mods, nm

    def substep(self, dt: float) -> None:
        R = self.L.np_real
        n = self.n
        coll, nc, mods, nm = self._tables(dt)
        x1 = np.zeros_like(self.x); v1 = np.zeros_like(self.v)
        C1 = np.zeros_like(self.C); F1 = np.zeros_like(self.F_trial)
        self.L.lib.or_substep(ctypes.byref(self.model), n, _ptr(self.sel), _ptr(self.mu), _ptr(self.lam), _ptr(self.ys),
                              _ptr(self.vol), _ptr(self.mass), _ptr(self.x), _ptr(self.v), _ptr(self.C),
                              _ptr(self.F_trial), _ptr(self.F), _ptr(self.stress), _ptr(x1), _ptr(v1), _ptr(C1),
                              _ptr(F1), _ptr(self.grid_m), _ptr(self.grid_v_in), _ptr(self.grid_v_out),
                              coll, nc, mods, nm, R(dt))
        # modify callbacks after the collider kernels (mpm_solver_diff.py:277-278)
        for c in self.colliders:
            if c.kind in (GRID_VELOCITY, CUBOID_VELOCITY) and c.start_time <= self.time < c.end_time:
                c.point = tuple(p + dt * vv for p, vv in zip(c.point, c.velocity))
                if self.collider_f32:
                    c.point = tuple(float(np.float32(p)) for p in c.point)
        self.x, self.v, self.C, self.F_trial = x1, v1, C1, F1
        self.time = self.time + dt

    def rollout(self, dt: float, n_steps: int, callback=None):
        for s in range(n_steps):
            if callback is not None:
                callback(self, s)
            self.substep(dt)
        return self.x
