"""Seeded synthetic workloads of the benchmark configurations.

The reference publishes no benchmark inputs and its dataset is not
available, so every configuration is synthetic (numpy.random.default_rng):

  c1  plain forward: 20,000 particles uniform in [0.35, 0.65]^3, 48^3 grid,
      fixed-corotated jelly E=2e4 nu=0.3 rho=1e3, dt=2e-4 x 200 substeps,
      gravity (0,-9.8,0), sticky floor at y=3dx, slip walls (bounding box)
  c2  large single forward: 500,000 particles in two boxes, 128^3 grid,
      plasticine with per-particle E log-U[1e3,1e5], nu U[0.2,0.45],
      yield U[5e2,5e3], softening 0.1; a 0.1^3 box collider centred at
      (0.30, 0.45, 0.30) moves at (0,-0.5,0) for the first 500 substeps and
      (0,+0.5,0) after; dt=1e-4 x 1000 substeps; floor and walls as c1
  c3  differentiable: 200,000 particles in [0.35,0.65]^3, v0 ~ N(0, 0.05),
      96^3 grid, plasticine; target (E=3e4, nu=0.35, yield=2e3), guess
      (1e4, 0.25, 1e3); dt=2e-4 x 400 substeps, checkpoint every 20
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, List, Optional

import numpy as np


@dataclass
class Workload:
    name: str
    n: int
    G: int
    dt: float
    T: int
    material: str
    x: np.ndarray
    v: np.ndarray
    vol: np.ndarray
    rho: np.ndarray
    E: np.ndarray
    nu: np.ndarray
    ys: np.ndarray
    gravity: tuple = (0.0, -9.8, 0.0)
    colliders: List[dict] = field(default_factory=list)
    velocity_schedule: Optional[Callable[[int], tuple]] = None   # cuboid velocity per substep
    description: str = ""

    @property
    def particle_substeps(self) -> int:
        return self.n * self.T


def _floor_walls(G):
    return [dict(kind="surface", point=[0.0, 3.0 / G, 0.0], normal=[0.0, 1.0, 0.0], surface="sticky"),
            dict(kind="bbox")]


def c1(seed: int = 1, n: int = 20_000, G: int = 48, T: int = 200) -> Workload:
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.35, 0.65, (n, 3)).astype(np.float32)
    return Workload(
        name="c1", n=n, G=G, dt=2e-4, T=T, material="jelly", x=x, v=np.zeros((n, 3), np.float32),
        vol=np.full(n, np.float32(0.027 / n), np.float32), rho=np.full(n, np.float32(1e3), np.float32),
        E=np.full(n, np.float32(2e4), np.float32), nu=np.full(n, np.float32(0.3), np.float32),
        ys=np.zeros(n, np.float32), colliders=_floor_walls(G),
        description=f"plain forward: {n} particles, {G}^3 grid, jelly (FCR), dt=2e-4 x {T} substeps")


def c2(seed: int = 2, n: int = 500_000, G: int = 128, T: int = 1000) -> Workload:
    rng = np.random.default_rng(seed)
    h = n // 2
    x = np.concatenate([rng.uniform((0.15, 0.10, 0.15), (0.45, 0.40, 0.45), (h, 3)),
                        rng.uniform((0.55, 0.10, 0.55), (0.85, 0.40, 0.85), (n - h, 3))]).astype(np.float32)
    E = np.exp(rng.uniform(np.log(1e3), np.log(1e5), n)).astype(np.float32)
    nu = rng.uniform(0.2, 0.45, n).astype(np.float32)
    ys = rng.uniform(5e2, 5e3, n).astype(np.float32)
    half = T // 2
    colliders = _floor_walls(G)
    colliders.insert(1, dict(kind="cuboid", point=[0.30, 0.45, 0.30], size=[0.05, 0.05, 0.05],
                             velocity=[0.0, -0.5, 0.0]))
    return Workload(
        name="c2", n=n, G=G, dt=1e-4, T=T, material="plasticine", x=x, v=np.zeros((n, 3), np.float32),
        vol=np.full(n, np.float32(0.054 / n), np.float32), rho=np.full(n, np.float32(1e3), np.float32),
        E=E, nu=nu, ys=ys, colliders=colliders,
        velocity_schedule=lambda s: (0.0, -0.5, 0.0) if s < half else (0.0, 0.5, 0.0),
        description=f"large single forward: {n} particles in two boxes, {G}^3 grid, plasticine "
                    f"(von Mises + FCR), moving 0.1^3 box collider, dt=1e-4 x {T} substeps")


def c3(seed: int = 3, n: int = 200_000, G: int = 96, T: int = 400, guess: bool = True) -> Workload:
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.35, 0.65, (n, 3)).astype(np.float32)
    v = (rng.standard_normal((n, 3)) * 0.05).astype(np.float32)
    E, nu, ys = (1e4, 0.25, 1e3) if guess else (3e4, 0.35, 2e3)
    return Workload(
        name="c3", n=n, G=G, dt=2e-4, T=T, material="plasticine", x=x, v=v,
        vol=np.full(n, np.float32(0.027 / n), np.float32), rho=np.full(n, np.float32(1e3), np.float32),
        E=np.full(n, np.float32(E), np.float32), nu=np.full(n, np.float32(nu), np.float32),
        ys=np.full(n, np.float32(ys), np.float32), colliders=_floor_walls(G),
        description=f"differentiable rollout: {n} particles, {G}^3 grid, plasticine, dt=2e-4 x {T} substeps")


def build_product(w: Workload, device="cuda:0"):
    """(solver, model, state_a, state_b) of the reference-facing API for w."""
    import torch

    from .mpm_data_structure import MPMModelStruct, MPMStateStruct
    from .mpm_solver_diff import MPMWARPDiff

    dev = torch.device(device)

    def t(a):
        return torch.as_tensor(np.ascontiguousarray(a), device=dev)

    st = MPMStateStruct()
    st.init(w.n, device=dev)
    st.from_torch(t(w.x), t(w.vol), None, t(w.v), n_grid=w.G, device=dev)
    st.reset_density(t(w.rho), update_mass=True)
    md = MPMModelStruct()
    md.init(w.n, device=dev)
    md.init_other_params(n_grid=w.G)
    md.gravitational_accelaration = w.gravity
    solver = MPMWARPDiff()
    solver.initialize(w.n, n_grid=w.G, device=dev)
    solver.set_parameters_dict(md, st, {"material": w.material})
    md.E.copy_(t(w.E))
    md.nu.copy_(t(w.nu))
    md.finalize_mu_lam(w.n)
    md.yield_stress.copy_(t(w.ys))
    for c in w.colliders:
        if c["kind"] == "surface":
            solver.add_surface_collider(c["point"], c["normal"], c.get("surface", "sticky"), 0.0)
        elif c["kind"] == "cuboid":
            solver.set_velocity_on_cuboid(c["point"], c["size"], c["velocity"])
        elif c["kind"] == "bbox":
            solver.add_bounding_box()
        else:
            raise ValueError(c["kind"])
    other = st.partial_clone()
    return solver, md, st, other


def cuboid_callback(w: Workload, solver):
    """Host callback applying w.velocity_schedule to the cuboid collider."""
    if w.velocity_schedule is None:
        return None
    idx = [i for i, c in enumerate(w.colliders) if c["kind"] == "cuboid"]
    if not idx:
        return None
    k = idx[0]

    def cb(step):
        solver.collider_params[k].velocity = w.velocity_schedule(step)

    return cb


def c4(seed: int = 4, n_inst: int = 32, T: int = 300, n_lo: int = 20_000, n_hi: int = 300_000):
    """Batched CMA-ES population: n_inst plasticine instances, particle counts
    log-uniform in [n_lo, n_hi], grids from {48, 64, 96, 128}^3, each body a
    random sub-box; per-instance log E ~ N(log 2e4, 0.3^2), log yield ~
    N(log 2e3, 0.3^2), nu ~ N(0.3, 0.05) clipped to [0.2, 0.45];
    dt = 2e-4 x T substeps; sticky floor at y = 3 dx and slip walls."""
    from .batch import InstanceSpec

    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n_inst):
        n = int(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi))))
        G = int(rng.choice([48, 64, 96, 128]))
        side = float(np.clip((n / (8.0 * G ** 3)) ** (1.0 / 3.0), 0.15, 0.6))
        lo = rng.uniform(0.1, 0.9 - side, 3)
        x = (lo + side * rng.uniform(0.0, 1.0, (n, 3))).astype(np.float32)
        E = np.float32(np.exp(rng.normal(np.log(2e4), 0.3)))
        ys = np.float32(np.exp(rng.normal(np.log(2e3), 0.3)))
        nu = np.float32(np.clip(rng.normal(0.3, 0.05), 0.2, 0.45))
        specs.append(InstanceSpec(
            x=x, v=np.zeros((n, 3), np.float32), vol=np.full(n, np.float32(side ** 3 / n), np.float32),
            rho=np.full(n, np.float32(1e3), np.float32), E=np.full(n, E, np.float32), nu=np.full(n, nu, np.float32),
            yield_stress=np.full(n, ys, np.float32), n_grid=G, material="plasticine", gravity=(0.0, -9.8, 0.0),
            colliders=_floor_walls(G)))
    return specs, 2e-4, T


def c5_arrivals(seed: int = 5, rate: float = 20.0, seconds: float = 60.0, grad_fraction: float = 0.3):
    """Arrival schedule of the serving stream: Poisson arrivals at `rate`
    requests/s for `seconds`; a `grad_fraction` of them (30 %) are rollout +
    gradient, the rest rollouts; particles log-uniform in [10k, 1M], grids
    uniform in 48..160, substeps uniform in [50, 1000]. The same draws are made
    whatever grad_fraction is, so other fractions keep the same requests.
    Returns [(t_arrival_s, grad, n, G, T, seed)]."""
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t > seconds:
            return out
        grad = bool(rng.uniform() < grad_fraction)
        n = int(np.exp(rng.uniform(np.log(1e4), np.log(1e6))))
        G = int(rng.integers(48, 161))
        T = int(rng.integers(50, 1001))
        out.append((t, grad, n, G, T, int(rng.integers(1 << 31))))


def c5_request(grad: bool, n: int, G: int, T: int, seed: int, dt: float = 1e-4):
    """One serving request: a plasticine body in a random sub-box (about 8
    particles per cell, side clipped to [0.15, 0.6]) with the large single
    rollout's material distributions (E log-U[1e3,1e5], nu U[0.2,0.45], yield
    U[5e2,5e3] per particle), sticky floor and slip walls. A gradient
    request's loss is the mean squared distance of the final positions from
    the initial ones."""
    from .batch import InstanceSpec
    from .serving import Request

    rng = np.random.default_rng(seed)
    side = float(np.clip((n / (8.0 * G ** 3)) ** (1.0 / 3.0), 0.15, 0.6))
    lo = rng.uniform(0.1, 0.9 - side, 3)
    x = (lo + side * rng.uniform(0.0, 1.0, (n, 3))).astype(np.float32)
    spec = InstanceSpec(
        x=x, v=np.zeros((n, 3), np.float32), vol=np.full(n, np.float32(side ** 3 / n), np.float32),
        rho=np.full(n, np.float32(1e3), np.float32),
        E=np.exp(rng.uniform(np.log(1e3), np.log(1e5), n)).astype(np.float32),
        nu=rng.uniform(0.2, 0.45, n).astype(np.float32), yield_stress=rng.uniform(5e2, 5e3, n).astype(np.float32),
        n_grid=G, material="plasticine", gravity=(0.0, -9.8, 0.0), colliders=_floor_walls(G))
    return Request(spec=spec, n_substeps=T, dt=dt, grad=grad, target=x.copy() if grad else None)


def lbs_frame(seed: int = 6, n_bones: int = 200_000, n_gauss: int = 2_000_000):
    """One rendered frame of Gaussian motion interpolation (synthetic): the
    particles of a 200k-particle body (the differentiable rollout's size, in
    [0.35, 0.65]^3) turn 2 degrees about (0.3, 1, 0.2) around their centre,
    translate by (2, -4, 1) mm and jitter by N(0, 0.2 mm); 2M Gaussians with
    random unit quaternions fill [0.33, 0.67]^3. Returns float32 arrays
    (prev, cur, xyz, quat)."""
    rng = np.random.default_rng(seed)
    prev = rng.uniform(0.35, 0.65, (n_bones, 3))
    c = prev.mean(0)
    axis = np.array([0.3, 1.0, 0.2]) / np.linalg.norm([0.3, 1.0, 0.2])
    ang = np.deg2rad(2.0)
    K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    R = np.eye(3) + np.sin(ang) * K + (1 - np.cos(ang)) * K @ K
    cur = (prev - c) @ R.T + c + np.array([0.002, -0.004, 0.001]) + rng.normal(0, 2e-4, (n_bones, 3))
    xyz = rng.uniform(0.33, 0.67, (n_gauss, 3))
    q = rng.normal(size=(n_gauss, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    f = lambda a: np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
    return f(prev), f(cur), f(xyz), f(q)
