"""GPU parity tests: the CUDA substep (through the C ABI and the
reference-facing Python API) against the golden vectors of the reference's
own kernels and against the FP64 CPU oracle.

Tolerances (FP32 kernels vs FP64 references, unit-cube domain):
  * single-stage values: relative to the largest magnitude of the compared
    field, 1e-4 (stress, C) / 2e-5 (F, positions);
  * rollouts: positions within 1e-4 of the domain size (the accuracy gate).
"""
import ctypes
import json

import numpy as np
import pytest
import torch

from empm_b200 import MPMModelStruct, MPMStateStruct, MPMWARPDiff
from empm_b200 import _native as N
from oracle import oracle as O
from tests import scenarios as S
from tests.gpu_helpers import max_abs, product_from_rollout

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
POS_GATE = 1e-4


def _rel_close(a, b, rel, floor=1e-30, what=""):
    a = np.asarray(a.detach().double().cpu() if isinstance(a, torch.Tensor) else a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), floor)
    err = np.abs(a - b).max()
    assert err <= rel * scale, f"{what}: max abs err {err:.3e} > {rel:.1e} * {scale:.3e}"
    return err


def _params(material, G, softening=0.1, plastic_viscosity=0.0, alpha=0.0, gravity=(0.0, 0.0, 0.0), rpic=0.0,
            damping=1.1):
    p = N.EmpmModelParams()
    p.n_grid, p.grid_lim, p.material = G, 1.0, material
    p.gravity = N.F3(*gravity)
    p.rpic_damping, p.grid_v_damping_scale = rpic, damping
    p.softening, p.plastic_viscosity, p.alpha = softening, plastic_viscosity, alpha
    return p


def _t(a, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=DEV).contiguous()


@pytest.mark.parametrize("material", range(7))
def test_stress_kernel_vs_golden(golden, material):
    g = golden("kernel_stress")
    k = f"m{material}/"
    n = g[k + "F_trial"].shape[0]
    L = N.lib()
    p = _params(material, 8, float(g[k + "softening"]), float(g[k + "plastic_viscosity"]), float(g[k + "alpha"]))
    Ft = _t(g[k + "F_trial"].reshape(n, 9))
    mu, lam, ys = _t(g[k + "mu_in"]), _t(g[k + "lam_in"]), _t(g[k + "ys_in"])
    F = torch.empty(n, 9, device=DEV)
    Sg = torch.empty(n, 9, device=DEV)
    N.check(L.empm_debug_stress(p, Ft.data_ptr(), mu.data_ptr(), lam.data_ptr(), ys.data_ptr(), float(g[k + "dt"]),
                                F.data_ptr(), Sg.data_ptr(), n, torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    _rel_close(F, g[k + "F"].reshape(n, 9), 2e-5, 1.0, "F")
    _rel_close(Sg, g[k + "stress"].reshape(n, 9), 1e-4, 1.0, "stress")
    _rel_close(ys, g[k + "ys_out"], 1e-5, 1.0, "yield")
    _rel_close(mu, g[k + "mu_out"], 1e-6, 1.0, "mu")
    _rel_close(lam, g[k + "lam_out"], 1e-6, 1.0, "lam")


def _random_case(rng, n, G, material):
    x = rng.uniform(0.3, 0.7, (n, 3)).astype(np.float32)
    v = (rng.standard_normal((n, 3)) * 0.5).astype(np.float32)
    C = (rng.standard_normal((n, 3, 3)) * 3.0).astype(np.float32)
    scale = np.where(rng.uniform(size=n) < 0.5, 0.05, 0.25)[:, None, None]
    Ft = (np.eye(3)[None] + scale * rng.standard_normal((n, 3, 3))).astype(np.float32)
    E = np.exp(rng.uniform(np.log(1e3), np.log(1e5), n)).astype(np.float32)
    nu = rng.uniform(0.2, 0.45, n).astype(np.float32)
    ys = rng.uniform(5e2, 5e3, n).astype(np.float32)
    vol = np.full(n, np.float32(0.064 / n), np.float32)
    rho = np.full(n, np.float32(1e3), np.float32)
    return x, v, C, Ft, E, nu, ys, vol, rho


def _product_state(x, v, C, Ft, E, nu, ys, vol, rho, G, material, gravity, softening=0.1):
    n = x.shape[0]
    st = MPMStateStruct()
    st.init(n, device=DEV)
    st.from_torch(_t(x), _t(vol), None, _t(v), n_grid=G, device=DEV)
    st.particle_C = _t(C)
    st.particle_F_trial = _t(Ft)
    st.reset_density(_t(rho), update_mass=True)
    md = MPMModelStruct()
    md.init(n, device=DEV)
    md.init_other_params(n_grid=G)
    md.material = material
    md.softening = softening
    md.gravitational_accelaration = gravity
    md.E.copy_(_t(E))
    md.nu.copy_(_t(nu))
    md.finalize_mu_lam(n)
    md.yield_stress.copy_(_t(ys))
    return st, md


@pytest.mark.parametrize("material", [0, 1, 2, 3, 4, 5, 6])
def test_single_substep_vs_oracle(material):
    rng = np.random.default_rng(100 + material)
    n, G, dt = 3000, 24, 2e-4
    x, v, C, Ft, E, nu, ys, vol, rho = _random_case(rng, n, G, material)
    gravity = (0.0, -9.8, 0.0)
    # oracle
    sim = O.OracleSim(x, v, vol, rho.astype(np.float64) * vol, E, nu, n_grid=G, material=material, gravity=gravity,
                      yield_stress=ys, friction_angle=25.0)
    sim.C = C.reshape(n, 9).astype(np.float64).copy()
    sim.F_trial = Ft.reshape(n, 9).astype(np.float64).copy()
    specs = [dict(kind="surface", point=[0.0, 3.0 / G, 0.0], normal=[0.0, 1.0, 0.0]),
             dict(kind="cuboid", point=[0.5, 0.62, 0.5], size=[0.1, 0.05, 0.1], velocity=[0.0, -0.5, 0.0]),
             dict(kind="geometry", shape="sphere", center=[0.35, 0.4, 0.5], radius=0.06),
             dict(kind="bbox")]
    sim.colliders = S.oracle_colliders(specs)
    # product
    st, md = _product_state(x, v, C, Ft, E, nu, ys, vol, rho, G, material, gravity)
    solver = MPMWARPDiff()
    solver.initialize(n, n_grid=G)
    solver.add_surface_collider((0.0, 3.0 / G, 0.0), (0.0, 1.0, 0.0), "sticky", 0.0)
    solver.set_velocity_on_cuboid([0.5, 0.62, 0.5], [0.1, 0.05, 0.1], [0.0, -0.5, 0.0])
    solver.add_geometry_collider(dict(shape="sphere", center=[0.35, 0.4, 0.5], radius=0.06))
    solver.add_bounding_box()
    nxt = st.partial_clone()
    solver.p2g2p_differentiable(md, st, nxt, dt)
    sim.substep(dt)
    torch.cuda.synchronize()
    # grid velocities after the boundary conditions
    mom, vel = ctypes.c_void_p(), ctypes.c_void_p()
    N.check(N.lib().empm_ctx_grid(solver._ctx.ptr, ctypes.byref(mom), ctypes.byref(vel)))
    nb = (G + 3) // 4
    g_blk = _wrap_device(vel.value, 4 * nb ** 3 * 64).view(-1, 4).double().cpu().numpy()
    g_vel = g_blk[N.grid_dense_index(G).reshape(-1)]
    touched = sim.grid_m > 0   # only nodes in some particle's stencil are updated
    _rel_close(g_vel[:, 3], sim.grid_m, 1e-5, 1e-12, "node mass")
    _rel_close(g_vel[touched, :3].reshape(-1), sim.grid_v_out.reshape(-1, 3)[touched].reshape(-1), 1e-4, 1.0,
               "node velocity")
    _rel_close(st.particle_F.reshape(n, 9), sim.F, 2e-5, 1.0, "elastic F")
    _rel_close(md.yield_stress, sim.ys, 1e-5, 1.0, "yield")
    _rel_close(md.mu, sim.mu, 1e-6, 1.0, "mu")
    _rel_close(nxt.particle_v, sim.v, 1e-4, 1.0, "v")
    _rel_close(nxt.particle_C.reshape(n, 9), sim.C, 1e-4, 1.0, "C")
    _rel_close(nxt.particle_F_trial.reshape(n, 9), sim.F_trial, 2e-5, 1.0, "F_trial")
    assert max_abs(nxt.particle_x, sim.x) <= 1e-6
    assert solver.time == pytest.approx(dt)


def _wrap_device(ptr: int, n: int) -> torch.Tensor:
    """Wrap a raw device float pointer (owned by the library) as a tensor view."""
    class _Holder:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False), "version": 3}

    return torch.as_tensor(_Holder(), device=DEV)


ROLLOUTS = ["jelly", "plasticine", "metal", "sand", "foam", "snow", "neohookean", "damped"]


@pytest.mark.parametrize("key", ROLLOUTS)
def test_rollout_vs_golden(golden, key):
    d = golden("rollouts")
    mpm, s = product_from_rollout(d, key)
    traj = mpm.advance_to(s["n_frames"])
    torch.cuda.synchronize()
    err = max_abs(traj, d[f"{key}/traj"])
    assert err <= 2e-5, f"{key}: trajectory error {err:.3e}"
    st = mpm.mpm_state
    _rel_close(st.particle_v, d[f"{key}/v"], 1e-3, 1.0, "v")
    _rel_close(st.particle_F_trial.reshape(-1, 9), d[f"{key}/F_trial"].reshape(-1, 9), 1e-4, 1.0, "F_trial")
    _rel_close(mpm.mpm_model.yield_stress, d[f"{key}/ys_out"], 1e-4, 1.0, "yield")


def _c1_like(n, G, seed, material, T, dt, plastic=False, cuboid=False):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.35, 0.65, (n, 3)).astype(np.float32)
    v = np.zeros((n, 3), np.float32)
    vol = np.full(n, np.float32(0.027 / n), np.float32)
    rho = np.full(n, np.float32(1e3), np.float32)
    if plastic:
        E = np.exp(rng.uniform(np.log(1e3), np.log(1e5), n)).astype(np.float32)
        nu = rng.uniform(0.2, 0.45, n).astype(np.float32)
        ys = rng.uniform(5e2, 5e3, n).astype(np.float32)
    else:
        E = np.full(n, 2e4, np.float32)
        nu = np.full(n, 0.3, np.float32)
        ys = np.zeros(n, np.float32)
    return x, v, vol, rho, E, nu, ys


@pytest.mark.parametrize("case", ["jelly_c1", "plasticine_small"])
def test_rollout_vs_fp64_oracle(case):
    if case == "jelly_c1":
        n, G, T, dt, material, plastic, cub = 20000, 48, 200, 2e-4, 0, False, False
    else:
        n, G, T, dt, material, plastic, cub = 20000, 48, 200, 1e-4, 5, True, True
    x, v, vol, rho, E, nu, ys = _c1_like(n, G, 1, material, T, dt, plastic)
    gravity = (0.0, -9.8, 0.0)
    specs = [dict(kind="surface", point=[0.0, 3.0 / G, 0.0], normal=[0.0, 1.0, 0.0]), dict(kind="bbox")]
    if cub:
        specs.insert(1, dict(kind="cuboid", point=[0.5, 0.72, 0.5], size=[0.08, 0.05, 0.08], velocity=[0.0, -1.0, 0.0]))
    sim = O.OracleSim(x, v, vol, rho.astype(np.float64) * vol, E, nu, n_grid=G, material=material, gravity=gravity,
                      yield_stress=ys)
    sim.colliders = S.oracle_colliders(specs)
    sim.rollout(dt, T)
    from empm_b200 import WarpMPMWrapper
    mpm = WarpMPMWrapper(grid_size=G, frame_dt=dt * T, sim_dt=dt, device=DEV)
    mpm.gravity = list(gravity)
    mpm.material_params = {"material": "plasticine" if plastic else "jelly"}
    mpm.add_particles(_t(x), _t(v), float(vol[0]), _t(E), _t(nu), 1e3)
    mpm.surface_colliders.append([(0.0, 3.0 / G, 0.0), (0.0, 1.0, 0.0), "sticky", 0.0])
    if cub:
        mpm.moving_boundaries.append([[0.5, 0.72, 0.5], [0.08, 0.05, 0.08], [0.0, -1.0, 0.0], 0.0])
    mpm.initialize()
    mpm.mpm_solver.add_bounding_box()
    mpm.mpm_model.yield_stress.copy_(_t(ys))
    n_sub = int(mpm.frame_dt / mpm.sim_dt)
    assert n_sub == T
    traj = mpm.advance_to(1)
    torch.cuda.synchronize()
    err = max_abs(traj[-1], sim.x)
    moved = float(np.abs(sim.x - x).max())
    print(f"{case}: max |x_gpu - x_fp64| = {err:.3e} (max displacement {moved:.3e})")
    assert moved > 1e-3
    assert err <= POS_GATE


def test_conservation_full_size():
    """Mass and momentum conservation of P2G/G2P at the 500k-particle, 128^3 size."""
    n, G, dt = 500_000, 128, 1e-4
    rng = np.random.default_rng(2)
    x = np.concatenate([rng.uniform((0.15, 0.10, 0.15), (0.45, 0.40, 0.45), (n // 2, 3)),
                        rng.uniform((0.55, 0.10, 0.55), (0.85, 0.40, 0.85), (n // 2, 3))]).astype(np.float32)
    v = (rng.standard_normal((n, 3)) * 0.3).astype(np.float32)
    C = (rng.standard_normal((n, 3, 3)) * 2.0).astype(np.float32)
    Ft = (np.eye(3)[None] + 0.05 * rng.standard_normal((n, 3, 3))).astype(np.float32)
    E = np.exp(rng.uniform(np.log(1e3), np.log(1e5), n)).astype(np.float32)
    nu = rng.uniform(0.2, 0.45, n).astype(np.float32)
    ys = rng.uniform(5e2, 5e3, n).astype(np.float32)
    vol = np.full(n, np.float32(0.054 / n), np.float32)
    rho = np.full(n, np.float32(1e3), np.float32)
    st, md = _product_state(x, v, C, Ft, E, nu, ys, vol, rho, G, 5, (0.0, 0.0, 0.0))
    solver = MPMWARPDiff()
    solver.initialize(n, n_grid=G)
    nxt = st.partial_clone()
    solver.p2g2p_differentiable(md, st, nxt, dt)
    torch.cuda.synchronize()
    mom, vel = ctypes.c_void_p(), ctypes.c_void_p()
    N.check(N.lib().empm_ctx_grid(solver._ctx.ptr, ctypes.byref(mom), ctypes.byref(vel)))
    nb = (G + 3) // 4
    g = _wrap_device(vel.value, 4 * nb ** 3 * 64).view(-1, 4).double()
    m_p = st.particle_mass.double()
    assert float(g[:, 3].sum()) == pytest.approx(float(m_p.sum()), rel=1e-5)
    p_grid = (g[:, :3] * g[:, 3:4]).sum(0)
    p_part = (st.particle_v.double() * m_p[:, None]).sum(0)
    scale = float((st.particle_v.double().abs() * m_p[:, None]).sum())
    assert float((p_grid - p_part).abs().max()) <= 1e-5 * scale
    p_new = (nxt.particle_v.double() * m_p[:, None]).sum(0)
    assert float((p_new - p_part).abs().max()) <= 1e-5 * scale
    assert solver.read_status() & N.EMPM_STATUS_NAN == 0


def test_graph_and_stream_paths_agree():
    n, G, dt, T = 20000, 48, 2e-4, 40
    x, v, vol, rho, E, nu, ys = _c1_like(n, G, 3, 0, T, dt)
    outs = []
    for use_graph in (False, True, True):
        st, md = _product_state(x, v, np.zeros((n, 3, 3), np.float32), np.tile(np.eye(3, dtype=np.float32), (n, 1, 1)),
                                E, nu, ys, vol, rho, G, 0, (0.0, -9.8, 0.0))
        solver = MPMWARPDiff()
        solver.initialize(n, n_grid=G)
        solver.use_graph = use_graph
        solver.add_bounding_box()
        other = st.partial_clone()
        res = solver.rollout(md, st, other, dt, T)
        outs.append(res.particle_x.clone())
    torch.cuda.synchronize()
    assert max_abs(outs[0], outs[1]) <= 1e-5
    assert max_abs(outs[1], outs[2]) <= 1e-5


def test_status_word_flags_cfl_and_nan():
    n, G, dt = 256, 16, 1e-3
    rng = np.random.default_rng(5)
    x = rng.uniform(0.4, 0.6, (n, 3)).astype(np.float32)
    v = np.zeros((n, 3), np.float32)
    v[:, 0] = 200.0               # the whole body moves: |v| dt = 0.2 > dx = 1/16 after G2P
    Ft = np.tile(np.eye(3, dtype=np.float32), (n, 1, 1))
    Ft[1, 0, 0] = np.nan
    st, md = _product_state(x, v, np.zeros((n, 3, 3), np.float32), Ft, np.full(n, 1e4, np.float32),
                            np.full(n, 0.3, np.float32), np.zeros(n, np.float32), np.full(n, 1e-5, np.float32),
                            np.full(n, 1e3, np.float32), G, 0, (0.0, 0.0, 0.0))
    solver = MPMWARPDiff()
    solver.initialize(n, n_grid=G)
    nxt = st.partial_clone()
    solver.p2g2p_differentiable(md, st, nxt, dt)
    status = solver.read_status()
    assert status & N.EMPM_STATUS_CFL
    assert status & N.EMPM_STATUS_NAN
    assert solver.read_status() == 0   # reading clears the word


@pytest.mark.parametrize("sort_every,p2g_mode,g2p_tile,tile_cap,seg_cap", [
    (0, 0, False, 1024, 4),       # direct path
    (1, 2, True, 1024, 4),
    (4, 1, False, 1024, 4),
    (16, 0, True, 1024, 4),
    (16, 1, True, 1024, 4),
    (16, 2, False, 1024, 4),
    (16, 2, False, 1024, 1),      # every lane its own reduction
    (16, 2, False, 1024, 32),     # whole same-cell runs per reduction
    (16, 1, True, 64, 4),         # tiny tile: forces the fallback path for most chunks
])
def test_sorted_path_vs_oracle(sort_every, p2g_mode, g2p_tile, tile_cap, seg_cap):
    n, G, T, dt = 20000, 48, 120, 2e-4
    x, v, vol, rho, E, nu, ys = _c1_like(n, G, 11, 5, T, dt, plastic=True)
    v = (np.random.default_rng(12).standard_normal((n, 3)) * 0.5).astype(np.float32)
    gravity = (0.0, -9.8, 0.0)
    specs = [dict(kind="surface", point=[0.0, 3.0 / G, 0.0], normal=[0.0, 1.0, 0.0]),
             dict(kind="cuboid", point=[0.5, 0.68, 0.5], size=[0.08, 0.05, 0.08], velocity=[0.0, -1.0, 0.0]),
             dict(kind="bbox")]
    sim = O.OracleSim(x, v, vol, rho.astype(np.float64) * vol, E, nu, n_grid=G, material=5, gravity=gravity,
                      yield_stress=ys)
    sim.colliders = S.oracle_colliders(specs)
    sim.rollout(dt, T)
    st, md = _product_state(x, v, np.zeros((n, 3, 3), np.float32), np.tile(np.eye(3, dtype=np.float32), (n, 1, 1)),
                            E, nu, ys, vol, rho, G, 5, gravity)
    solver = MPMWARPDiff()
    solver.initialize(n, n_grid=G)
    solver.sort_every, solver.p2g_mode, solver.g2p_tile, solver.tile_cap = sort_every, p2g_mode, g2p_tile, tile_cap
    solver.seg_cap = seg_cap
    solver.add_surface_collider((0.0, 3.0 / G, 0.0), (0.0, 1.0, 0.0), "sticky", 0.0)
    solver.set_velocity_on_cuboid([0.5, 0.68, 0.5], [0.08, 0.05, 0.08], [0.0, -1.0, 0.0])
    solver.add_bounding_box()
    other = st.partial_clone()
    res = solver.rollout(md, st, other, dt, T)
    torch.cuda.synchronize()
    err = max_abs(res.particle_x, sim.x)
    print(f"sort_every={sort_every} p2g_mode={p2g_mode} g2p_tile={g2p_tile} cap={tile_cap}: max pos err {err:.3e}")
    assert err <= POS_GATE
    _rel_close(md.yield_stress, sim.ys, 2e-3, 1.0, "yield")
    _rel_close(res.particle_F_trial.reshape(n, 9), sim.F_trial, 2e-3, 1.0, "F_trial")
    assert solver.read_status() & (N.EMPM_STATUS_NAN | N.EMPM_STATUS_OUT_OF_BAND) == 0


def test_sorted_path_modifiers_and_selection():
    """Particle modifiers (masks indexed by the caller's particle order) and an
    unsimulated selection on the sorted path against the oracle."""
    n, G, T, dt = 4000, 24, 30, 2e-4
    rng = np.random.default_rng(21)
    x = rng.uniform(0.3, 0.7, (n, 3)).astype(np.float32)
    v = np.zeros((n, 3), np.float32)
    vol = np.full(n, np.float32(0.064 / n), np.float32)
    rho = np.full(n, np.float32(1e3), np.float32)
    E = np.full(n, np.float32(3e4), np.float32)
    nu = np.full(n, np.float32(0.3), np.float32)
    sel = (rng.uniform(size=n) < 0.05).astype(np.int32)
    st, md = _product_state(x, v, np.zeros((n, 3, 3), np.float32), np.tile(np.eye(3, dtype=np.float32), (n, 1, 1)),
                            E, nu, np.zeros(n, np.float32), vol, rho, G, 0, (0.0, -9.8, 0.0))
    st.set_selection(_t(sel, torch.int32))
    solver = MPMWARPDiff()
    solver.initialize(n, n_grid=G)
    solver.sort_every = 4
    solver.add_impulse_on_particles(st, force=[0.0, 0.0, 5e-3], dt=dt, point=[0.45, 0.45, 0.45], size=[0.1, 0.1, 0.1],
                                    num_dt=10)
    solver.enforce_particle_velocity_translation(st, point=[0.6, 0.6, 0.6], size=[0.08, 0.08, 0.08],
                                                 velocity=[0.3, 0.0, 0.0], start_time=0.0, end_time=0.004)
    mover_mask = (rng.uniform(size=n) < 0.2).astype(np.int32)
    solver.set_particle_mover(velocity=[0.0, 0.0, -0.01], angular_velocity=2.0, center=[0.5, 0.5, 0.5],
                              axis=[0.0, 1.0, 0.0], selection_mask=mover_mask, device=DEV)
    solver.add_bounding_box()
    other = st.partial_clone()
    res = solver.rollout(md, st, other, dt, T)
    torch.cuda.synchronize()
    sim = O.OracleSim(x, v, vol, rho.astype(np.float64) * vol, E, nu, n_grid=G, material=0, gravity=(0.0, -9.8, 0.0),
                      selection=sel)
    box = lambda p, s: (np.abs(x - np.array(p)) < np.array(s)).all(1).astype(np.int32)  # noqa: E731
    sim.modifiers = [
        O.OrModifierSpec(O.MOD_IMPULSE, vec=(0.0, 0.0, 5e-3), start_time=0.0, end_time=0.0 + dt * 10,
                         mask=box([0.45] * 3, [0.1] * 3)),
        O.OrModifierSpec(O.MOD_SET_VELOCITY, vec=(0.3, 0.0, 0.0), start_time=0.0, end_time=0.004,
                         mask=box([0.6] * 3, [0.08] * 3)),
        O.OrModifierSpec(O.MOD_MOVER, vec=(0.0, 0.0, -0.01), point=(0.5, 0.5, 0.5), normal=(0.0, 1.0, 0.0),
                         scale=(2.0, 0.0), mask=mover_mask),
    ]
    sim.colliders = S.oracle_colliders([dict(kind="bbox")])
    sim.rollout(dt, T)
    err = max_abs(res.particle_x, sim.x)
    print(f"modifiers+selection: max pos err {err:.3e}")
    assert err <= POS_GATE
    assert float(res.particle_x[torch.from_numpy(sel).bool().to(DEV)].abs().max()) == 0.0
