"""Generate golden vectors by running the reference's own simulator source.

Run where the reference checkout is available (read-only) at
/root/reference. The machines that run the GPU tests do not have it, so the
outputs are committed as tests/golden/*.npz:

    python tests/golden/make_golden.py [--reference /root/reference]

The reference modules phys_sim/diff_simulator/warp_mpm/{mpm_data_structure,
mpm_utils, mpm_solver_diff, warp_mpm_wrapper}.py are imported unmodified.
Two of their imports are replaced because they need the Warp runtime, which
is not installable offline:
  * ``warp`` -> tests/golden/warp_shim (FP64 NumPy restatement of the Warp
    builtins the code calls; see its docstring);
  * ``warp_utils`` -> a stub whose from_torch_safe copies the tensor (the
    reference's version aliases the torch storage through a raw pointer).
``pyvista`` and ``matplotlib`` (used only for PLY export and plots) are stubbed.

Each fixture stores the scenario (JSON) and the inputs/outputs in float64.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_reference(ref_root: str):
    sys.path.insert(0, os.path.join(HERE, "warp_shim"))
    import torch
    import warp as wp  # the shim

    wu = types.ModuleType("warp_utils")

    def from_torch_safe(t, dtype=None, requires_grad=None, grad=None):
        if dtype is None:
            dtype = float
        return wp.from_numpy(t.detach().cpu().numpy(), dtype=dtype, requires_grad=bool(requires_grad))

    class MyTape(wp.Tape):
        pass

    class CondTape:
        def __init__(self, tape, cond=True):
            self.tape = tape

        def __enter__(self):
            return self

        def __exit__(self, *a):
            pass

    wu.from_torch_safe = from_torch_safe
    wu.MyTape = MyTape
    wu.CondTape = CondTape
    sys.modules["warp_utils"] = wu
    for name in ("pyvista", "matplotlib", "matplotlib.pyplot"):
        sys.modules.setdefault(name, types.ModuleType(name))
    src = os.path.join(ref_root, "phys_sim", "diff_simulator", "warp_mpm")
    sys.path.insert(0, src)
    pkg = types.ModuleType("warp_mpm")
    pkg.__path__ = [src]
    sys.modules["warp_mpm"] = pkg
    ref = types.SimpleNamespace()
    ref.wp = wp
    ref.torch = torch
    ref.ds = importlib.import_module("mpm_data_structure")
    ref.utils = importlib.import_module("mpm_utils")
    ref.solver = importlib.import_module("mpm_solver_diff")
    ref.wrapper = importlib.import_module("warp_mpm.warp_mpm_wrapper")
    ref.root = ref_root
    return ref


def f32(a):
    return np.asarray(a, dtype=np.float32).astype(np.float64)


# ---------------------------------------------------------------------------
# per-kernel fixtures
# ---------------------------------------------------------------------------
def make_state(ref, n, G, grid_lim=1.0):
    wp = ref.wp
    st = ref.ds.MPMStateStruct()
    st.init(n, device="cpu", requires_grad=False)
    st.init_grid(G, device="cpu")
    model = ref.ds.MPMModelStruct()
    model.init(n, device="cpu")
    model.init_other_params(n_grid=G, grid_lim=grid_lim, device="cpu")
    return st, model


def kernel_stress(ref, rng):
    wp = ref.wp
    out = {}
    n = 48
    for material in range(7):
        st, model = make_state(ref, n, 8)
        model.material = material
        model.softening = 0.1
        model.plastic_viscosity = 2.0
        sin_phi = wp.sin(35.0 / 180.0 * 3.14159265)
        model.alpha = wp.sqrt(2.0 / 3.0) * 2.0 * sin_phi / (3.0 - sin_phi)
        scale = np.where(np.arange(n) < n // 2, 0.05, 0.35)[:, None, None]
        Ft = np.eye(3)[None] + scale * rng.standard_normal((n, 3, 3))
        Ft = f32(Ft)
        E = f32(np.exp(rng.uniform(np.log(1e3), np.log(1e5), n)))
        nu = f32(rng.uniform(0.2, 0.45, n))
        ys = f32(rng.uniform(5e2, 5e3, n))
        st.particle_F_trial.data[...] = Ft
        model.E.data[...] = E
        model.nu.data[...] = nu
        model.yield_stress.data[...] = ys
        wp.launch(ref.utils.compute_mu_lam_from_E_nu, dim=n, inputs=[st, model])
        mu0, lam0 = model.mu.data.copy(), model.lam.data.copy()
        dt = 2e-4
        wp.launch(ref.utils.compute_stress_from_F_trial, dim=n, inputs=[st, model, dt])
        out[f"m{material}"] = dict(
            material=material, dt=dt, softening=0.1, plastic_viscosity=2.0, alpha=model.alpha,
            F_trial=Ft, E=E, nu=nu, mu_in=mu0, lam_in=lam0, ys_in=ys,
            F=st.particle_F.data.copy(), stress=st.particle_stress.data.copy(),
            mu_out=model.mu.data.copy(), lam_out=model.lam.data.copy(), ys_out=model.yield_stress.data.copy(),
        )
    return out


def kernel_p2g(ref, rng):
    wp = ref.wp
    out = {}
    n, G = 96, 12
    for tag, rpic in (("apic", 0.0), ("rpic", 0.3), ("pic", -1.0)):
        st, model = make_state(ref, n, G)
        model.rpic_damping = rpic
        x = f32(rng.uniform(0.3, 0.7, (n, 3)))
        v = f32(rng.standard_normal((n, 3)) * 0.3)
        C = f32(rng.standard_normal((n, 3, 3)) * 2.0)
        S = rng.standard_normal((n, 3, 3)) * 1e3
        S = f32(0.5 * (S + np.transpose(S, (0, 2, 1))))
        vol = f32(rng.uniform(0.5, 1.5, n) * 1e-4)
        mass = f32(vol * 1e3)
        for name, arr in (("particle_x", x), ("particle_v", v), ("particle_C", C), ("particle_stress", S),
                          ("particle_vol", vol), ("particle_mass", mass)):
            getattr(st, name).data[...] = arr
        dt = 1e-4
        wp.launch(ref.utils.zero_grid, dim=(G, G, G), inputs=[st, model])
        wp.launch(ref.utils.p2g_apic_with_stress, dim=n, inputs=[st, model, dt])
        out[tag] = dict(G=G, rpic=rpic, dt=dt, x=x, v=v, C=C, stress=S, vol=vol, mass=mass,
                        grid_m=st.grid_m.data.copy(), grid_v_in=st.grid_v_in.data.copy())
    return out


def collider_suite(ref, solver, G, dx):
    """Register one collider of every kind on `solver` (MPMWARPDiff); returns specs."""
    specs = []
    solver.add_surface_collider((0.0, 3 * dx, 0.0), (0.0, 1.0, 0.0), "sticky", 0.0)
    specs.append(dict(kind="surface", point=[0.0, 3 * dx, 0.0], normal=[0.0, 1.0, 0.0], surface="sticky"))
    solver.add_surface_collider((0.0, 0.0, 0.2), (0.3, 0.0, 1.0), "slip", 0.0)
    specs.append(dict(kind="surface", point=[0.0, 0.0, 0.2], normal=[0.3, 0.0, 1.0], surface="slip"))
    solver.add_surface_collider((0.8, 0.0, 0.0), (-1.0, 0.0, 0.0), "cut", 0.0)
    specs.append(dict(kind="surface", point=[0.8, 0.0, 0.0], normal=[-1.0, 0.0, 0.0], surface="cut"))
    geos = [
        dict(shape="cube", center=[0.5, 0.5, 0.5], size=[0.1, 0.05, 0.08]),
        dict(shape="sphere", center=[0.3, 0.6, 0.4], radius=0.12),
        dict(shape="cylinder", center=[0.6, 0.3, 0.6], axis=[0.0, 1.0, 1.0], radius=0.1, half_height=0.15),
        dict(shape="halfspace", point=[0.0, 0.0, 0.9], normal=[0.0, 0.0, -1.0], surface="separate"),
    ]
    for g in geos:
        solver.add_geometry_collider(dict(g))
        specs.append(dict(kind="geometry", **g))
    solver.set_grid_velocity_on_geometry(dict(shape="cube", center=[0.45, 0.42, 0.5], size=[0.1, 0.06, 0.1],
                                              velocity=[0.2, -0.3, 0.1], angular_velocity=2.0,
                                              rot_axis=[0.0, 0.0, 1.0]))
    specs.append(dict(kind="grid_velocity", shape="cube", center=[0.45, 0.42, 0.5], size=[0.1, 0.06, 0.1],
                      velocity=[0.2, -0.3, 0.1], angular_velocity=2.0, rot_axis=[0.0, 0.0, 1.0]))
    solver.set_velocity_on_cuboid([0.55, 0.62, 0.45], ref.wp.vec3(0.08, 0.05, 0.08), [0.0, -0.5, 0.0])
    specs.append(dict(kind="cuboid", point=[0.55, 0.62, 0.45], size=[0.08, 0.05, 0.08], velocity=[0.0, -0.5, 0.0]))
    solver.add_bounding_box()
    specs.append(dict(kind="bbox"))
    return specs


def kernel_grid(ref, rng):
    wp = ref.wp
    torch = ref.torch
    G = 16
    st, model = make_state(ref, 1, G)
    dx = model.dx
    model.gravitational_accelaration = wp.vec3(0.0, -9.8, 0.0)
    m = rng.uniform(0.0, 2e-3, (G, G, G))
    m[rng.uniform(size=(G, G, G)) < 0.3] = 0.0
    m = f32(m)
    vin = f32(rng.standard_normal((G, G, G, 3)) * 1e-3)
    mask = (rng.uniform(size=(G, G, G)) < 0.05).astype(np.int32)
    out = {}
    for tag, damping, with_coll in (("plain", 1.1, False), ("damped_colliders", 0.98, True)):
        st.grid_m.data[...] = m
        st.grid_v_in.data[...] = vin
        st.grid_v_out.data[...] = 0.0
        solver = ref.solver.MPMWARPDiff()
        solver.initialize(1, n_grid=G, device="cpu")
        specs = collider_suite(ref, solver, G, dx) if with_coll else []
        if with_coll:
            solver.enforce_grid_velocity_by_mask(torch.from_numpy(mask))
            specs.append(dict(kind="grid_mask"))
        dt = 2e-4
        solver.time = 0.0
        wp.launch(ref.utils.grid_normalization_and_gravity, dim=(G, G, G), inputs=[st, model, dt])
        if damping < 1.0:
            wp.launch(ref.utils.add_damping_via_grid, dim=(G, G, G), inputs=[st, damping])
        for k in range(len(solver.grid_postprocess)):
            wp.launch(solver.grid_postprocess[k], dim=(G, G, G),
                      inputs=[solver.time, dt, st, model, solver.collider_params[k]])
        out[tag] = dict(G=G, dt=dt, damping=damping, gravity=[0.0, -9.8, 0.0], grid_m=m, grid_v_in=vin, mask=mask,
                        colliders=json.dumps(specs), grid_v_out=st.grid_v_out.data.copy())
    return out


def kernel_g2p(ref, rng):
    wp = ref.wp
    n, G = 96, 12
    st, model = make_state(ref, n, G)
    nxt, _ = make_state(ref, n, G)
    x = f32(rng.uniform(0.25, 0.75, (n, 3)))
    x[0] = [2.05 / G, 0.5, 0.5]                 # lands in the low clamp band
    F = f32(np.eye(3)[None] + 0.1 * rng.standard_normal((n, 3, 3)))
    gv = f32(rng.standard_normal((G, G, G, 3)) * 0.5)
    gv[:, :, :, 0] -= 4.0                         # push particle 0 below 2 dx
    st.particle_x.data[...] = x
    st.particle_F.data[...] = F
    st.grid_v_out.data[...] = gv
    dt = 2e-3
    wp.launch(ref.utils.g2p_differentiable, dim=n, inputs=[st, nxt, model, dt])
    return {"g2p": dict(G=G, dt=dt, x=x, F=F, grid_v_out=gv, x_out=nxt.particle_x.data.copy(),
                        v_out=nxt.particle_v.data.copy(), C_out=nxt.particle_C.data.copy(),
                        F_out=nxt.particle_F_trial.data.copy())}


def kernel_restart(ref, rng):
    """MPMWARPDiff.restart_and_compute_F_C (mpm_solver_diff.py:1214-1262): F
    from a displacement field scattered to the grid and gathered back."""
    wp = ref.wp
    n, G = 80, 12
    st, model = make_state(ref, n, G)
    x = f32(rng.uniform(0.3, 0.7, (n, 3)))
    target = f32(x + 0.02 * rng.standard_normal((n, 3)))
    mass = f32(rng.uniform(0.5, 1.5, n) * 1e-4)
    st.particle_x.data[...] = x
    st.particle_mass.data[...] = mass
    solver = ref.solver.MPMWARPDiff()
    solver.initialize(n, n_grid=G, device="cpu")
    solver.restart_and_compute_F_C(model, st, wp.from_numpy(target, dtype=wp.vec3), device="cpu")
    out = {"restart": dict(G=G, x=x, target=target, mass=mass, F_out=st.particle_F_trial.data.copy(),
                           x_out=st.particle_x.data.copy())}
    # the same with the PhysGaussian covariance update switched on
    st, model = make_state(ref, n, G)
    st.particle_x.data[...] = x
    st.particle_mass.data[...] = mass
    A = rng.standard_normal((n, 3, 3)) * 1e-2
    S = A @ np.transpose(A, (0, 2, 1)) + 1e-4 * np.eye(3)
    cov = f32(np.stack([S[:, 0, 0], S[:, 0, 1], S[:, 0, 2], S[:, 1, 1], S[:, 1, 2], S[:, 2, 2]], 1).reshape(-1))
    st.particle_cov.data[...] = cov
    model.update_cov_with_F = True
    solver = ref.solver.MPMWARPDiff()
    solver.initialize(n, n_grid=G, device="cpu")
    solver.restart_and_compute_F_C(model, st, wp.from_numpy(target, dtype=wp.vec3), device="cpu")
    out["restart_cov"] = dict(G=G, x=x, target=target, mass=mass, cov=cov, F_out=st.particle_F_trial.data.copy(),
                              cov_out=st.particle_cov.data.copy())
    return out


# ---------------------------------------------------------------------------
# rollouts through WarpMPMWrapper (the reference's public API)
# ---------------------------------------------------------------------------
def rollout(ref, rng, *, material, n, G, frame_dt, sim_dt, n_frames, gravity, E, nu, rho, yield_stress=None,
            v0_scale=0.0, box=(0.35, 0.65), cuboid=None, bbox=True, floor=True, extra_params=None, per_particle=False,
            grid_mover=None):
    torch = ref.torch
    lo, hi = box
    x = f32(rng.uniform(lo, hi, (n, 3)))
    v = f32(rng.standard_normal((n, 3)) * v0_scale)
    vol = float(np.float32(((hi - lo) ** 3) / n))
    mpm = ref.wrapper.WarpMPMWrapper(grid_size=G, grid_lim=1.0, frame_dt=frame_dt, sim_dt=sim_dt, device="cpu")
    mpm.gravity = list(gravity)
    params = dict(ref.wrapper.material_gallery[material])
    if extra_params:
        params.update(extra_params)
    mpm.material_params = params
    if per_particle:
        E_arr = f32(np.exp(rng.uniform(np.log(E[0]), np.log(E[1]), n)))
        nu_arr = f32(rng.uniform(nu[0], nu[1], n))
    else:
        E_arr = np.full(n, float(np.float32(E)))
        nu_arr = np.full(n, float(np.float32(nu)))
    mpm.add_particles(torch.from_numpy(x), torch.from_numpy(v), vol, torch.from_numpy(E_arr),
                      torch.from_numpy(nu_arr), float(rho))
    dx = 1.0 / G
    specs = []
    if floor:
        mpm.surface_colliders.append([(0.0, 3 * dx, 0.0), (0.0, 1.0, 0.0), "sticky", 0.0])
        specs.append(dict(kind="surface", point=[0.0, 3 * dx, 0.0], normal=[0.0, 1.0, 0.0], surface="sticky"))
    if cuboid is not None:
        mpm.moving_boundaries.append([cuboid["point"], cuboid["size"], cuboid["velocity"], 0.0])
        specs.append(dict(kind="cuboid", **cuboid))
    if grid_mover is not None:
        mpm.grid_geometry_movers.append(dict(grid_mover))
        specs.append(dict(kind="grid_velocity", **grid_mover))
    mpm.initialize()
    if bbox:
        mpm.mpm_solver.add_bounding_box()
        specs.append(dict(kind="bbox"))
    ys_arr = None
    if yield_stress is not None:
        if isinstance(yield_stress, tuple):
            ys_arr = f32(rng.uniform(yield_stress[0], yield_stress[1], n))
            mpm.mpm_model.yield_stress.data[...] = ys_arr
        else:
            ys_arr = np.full(n, float(yield_stress))
    ys_in = mpm.mpm_model.yield_stress.data.copy()
    traj = mpm.advance_to(n_frames).numpy()
    st = mpm.mpm_state
    model = mpm.mpm_model
    scen = dict(material=material, n=n, G=G, frame_dt=frame_dt, sim_dt=sim_dt, n_frames=n_frames,
                n_substeps=int(frame_dt / sim_dt), gravity=list(gravity), rho=float(rho), vol=vol,
                params={k: v for k, v in params.items()}, colliders=specs,
                damping=float(model.grid_v_damping_scale), rpic=float(model.rpic_damping))
    return dict(scenario=json.dumps(scen), x0=x, v0=v, E=E_arr, nu=nu_arr, ys_in=ys_in, traj=traj,
                x=st.particle_x.data.copy(), v=st.particle_v.data.copy(), C=st.particle_C.data.copy(),
                F_trial=st.particle_F_trial.data.copy(), ys_out=model.yield_stress.data.copy(),
                mu_out=model.mu.data.copy(), lam_out=model.lam.data.copy())


def rollouts(ref, rng):
    out = {}
    g = (0.0, -9.8, 0.0)
    out["jelly"] = rollout(ref, rng, material="jelly", n=256, G=16, frame_dt=1e-3, sim_dt=2e-4, n_frames=3,
                           gravity=g, E=2e4, nu=0.3, rho=1e3, v0_scale=0.3)
    out["plasticine"] = rollout(ref, rng, material="plasticine", n=256, G=16, frame_dt=1e-3, sim_dt=2e-4,
                                n_frames=4, gravity=g, E=(1e3, 1e5), nu=(0.2, 0.45), rho=1e3, per_particle=True,
                                yield_stress=(5e2, 5e3), v0_scale=1.5,
                                cuboid=dict(point=[0.5, 0.68, 0.5], size=[0.1, 0.06, 0.1], velocity=[0.0, -2.0, 0.0]))
    for mat in ("metal", "sand", "foam", "snow", "neo-hookean"):
        extra = {"yield_stress": 3e3} if mat in ("metal", "foam") else None
        if mat == "foam":
            extra["plastic_viscosity"] = 0.5
        out[mat.replace("-", "")] = rollout(ref, rng, material=mat, n=160, G=12, frame_dt=1e-3, sim_dt=2.5e-4,
                                            n_frames=2, gravity=g, E=(5e3, 5e4), nu=(0.25, 0.4), rho=1e3,
                                            per_particle=True, v0_scale=1.0, extra_params=extra)
    out["damped"] = rollout(ref, rng, material="jelly", n=200, G=16, frame_dt=1e-3, sim_dt=2.5e-4, n_frames=2,
                            gravity=g, E=3e4, nu=0.3, rho=1e3, v0_scale=0.5,
                            extra_params={"rpic_damping": 0.2, "grid_v_damping_scale": 0.98},
                            grid_mover=dict(shape="sphere", center=[0.5, 0.66, 0.5], radius=0.08,
                                            velocity=[0.0, -1.0, 0.0], end_time=0.0012, reset=1))
    return out


def inplace(ref, rng):
    """The in-place substep MPMWARPDiff.p2g2p (mpm_solver_diff.py:293-429):
    g2p with atomic_add on x and the PhysGaussian covariance update
    (mpm_utils.py:441-499), then clip_particle_x (:582-599). Plasticine with
    a moving cuboid, an impulse modifier, unsimulated particles and
    update_cov_with_F on."""
    torch, wp = ref.torch, ref.wp
    out = {}
    for tag, cov_on in (("cov", True), ("nocov", False)):
        n, G, dt, T = 220, 16, 2e-4, 6
        x = f32(rng.uniform(0.3, 0.7, (n, 3)))
        v = f32(rng.standard_normal((n, 3)) * 2.5)
        vol = float(np.float32(0.4 ** 3 / n))
        E = f32(np.exp(rng.uniform(np.log(2e3), np.log(5e4), n)))
        nu = f32(rng.uniform(0.2, 0.45, n))
        mpm = ref.wrapper.WarpMPMWrapper(grid_size=G, grid_lim=1.0, frame_dt=dt, sim_dt=dt, device="cpu")
        mpm.gravity = [0.0, -9.8, 0.0]
        mpm.material_params = dict(ref.wrapper.material_gallery["plasticine"])
        mpm.add_particles(torch.from_numpy(x), torch.from_numpy(v), vol, torch.from_numpy(E), torch.from_numpy(nu),
                          1e3)
        mpm.surface_colliders.append([(0.0, 3.0 / G, 0.0), (0.0, 1.0, 0.0), "sticky", 0.0])
        cub = dict(point=[0.5, 0.74, 0.5], size=[0.1, 0.06, 0.1], velocity=[0.0, -2.0, 0.0])
        mpm.moving_boundaries.append([cub["point"], cub["size"], cub["velocity"], 0.0])
        mpm.initialize()
        mpm.mpm_solver.add_bounding_box()
        st, model, solver = mpm.mpm_state, mpm.mpm_model, mpm.mpm_solver
        ys = f32(rng.uniform(5e2, 5e3, n))
        model.yield_stress.data[...] = ys
        imp = dict(force=[0.0, 0.0, 2e-3], point=[0.45, 0.45, 0.45], size=[0.1, 0.1, 0.1], num_dt=4)
        solver.add_impulse_on_particles(st, force=imp["force"], dt=dt, point=imp["point"], size=imp["size"],
                                        num_dt=imp["num_dt"], device="cpu")
        sel = (rng.uniform(size=n) < 0.1).astype(np.int32)
        st.particle_selection.data[...] = sel
        A = rng.standard_normal((n, 3, 3)) * 1e-2
        S = A @ np.transpose(A, (0, 2, 1)) + 1e-4 * np.eye(3)
        cov = f32(np.stack([S[:, 0, 0], S[:, 0, 1], S[:, 0, 2], S[:, 1, 1], S[:, 1, 2], S[:, 2, 2]], 1).reshape(-1))
        st.particle_cov.data[...] = cov
        model.update_cov_with_F = cov_on
        for step in range(T):
            solver.p2g2p(model, st, step, dt, device="cpu")
        scen = dict(n=n, G=G, dt=dt, T=T, vol=vol, rho=1e3, gravity=[0.0, -9.8, 0.0], cuboid=cub, impulse=imp,
                    update_cov=cov_on)
        out[tag] = dict(scenario=json.dumps(scen), x0=x, v0=v, E=E, nu=nu, ys_in=ys, sel=sel, cov0=cov,
                        x=st.particle_x.data.copy(), v=st.particle_v.data.copy(), C=st.particle_C.data.copy(),
                        F_trial=st.particle_F_trial.data.copy(), F=st.particle_F.data.copy(),
                        cov=st.particle_cov.data.copy(), ys_out=model.yield_stress.data.copy(),
                        mu_out=model.mu.data.copy(), lam_out=model.lam.data.copy())
    return out


def load_dynamic_utils(ref_root: str):
    """third_party/gaussian_splatting/dynamic_utils.py, unmodified. It imports
    kornia (0.8.1, not installed here) at module level; a stub module stands in
    whose rotation_matrix_to_quaternion raises, so interpolate_motions_speedup
    takes its own mat2quat fallback (dynamic_utils.py:474-478)."""
    kornia = types.ModuleType("kornia")
    geometry = types.ModuleType("kornia.geometry")
    conversions = types.ModuleType("kornia.geometry.conversions")

    def rotation_matrix_to_quaternion(*a, **k):
        raise NotImplementedError("kornia is not installed")

    conversions.rotation_matrix_to_quaternion = rotation_matrix_to_quaternion
    geometry.conversions = conversions
    kornia.geometry = geometry
    sys.modules.update({"kornia": kornia, "kornia.geometry": geometry, "kornia.geometry.conversions": conversions})
    path = os.path.join(ref_root, "third_party", "gaussian_splatting")
    sys.path.insert(0, path)
    try:
        return importlib.import_module("dynamic_utils")
    finally:
        sys.path.remove(path)


def lbs(ref, rng):
    """Gaussian motion interpolation cases (float32 tensors, CPU)."""
    import torch
    du = load_dynamic_utils(ref.root)
    t = lambda a: torch.as_tensor(np.asarray(a, np.float32))
    out = {}

    def rot_about(axis, ang):
        axis = np.asarray(axis, np.float64) / np.linalg.norm(axis)
        K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
        return np.eye(3) + np.sin(ang) * K + (1 - np.cos(ang)) * K @ K

    def random_quats(n):
        q = rng.normal(size=(n, 4))
        return q / np.linalg.norm(q, axis=1, keepdims=True)

    # 1. generic: a blob of bones turning 20 degrees, translating, with noise
    nb, ng = 600, 3000
    bones = rng.uniform(0.3, 0.7, size=(nb, 3))
    c = bones.mean(0)
    R = rot_about([0.3, 1.0, 0.2], np.deg2rad(20.0))
    motions = (bones - c) @ R.T + c + np.array([0.01, -0.02, 0.005]) - bones + rng.normal(0, 1e-3, (nb, 3))
    gauss = rng.uniform(0.28, 0.72, size=(ng, 3))
    quat = random_quats(ng)
    bones_t, motions_t, gauss_t, quat_t = t(bones), t(motions), t(gauss), t(quat)
    relations = du.get_topk_indices(bones_t, K=16)
    weights, widx = du.knn_weights_sparse(bones_t, gauss_t, K=16)
    weights2 = du.calc_weights_vals_from_indices(bones_t, gauss_t, widx)
    xyz, rot, _ = du.interpolate_motions_speedup(bones=bones_t, motions=motions_t, relations=relations, xyz=gauss_t,
                                                 quat=quat_t, weights=weights2, weights_indices=widx, device="cpu")
    dense_w = du.knn_weights(bones_t, gauss_t, K=16)
    xyz_d, rot_d, _ = du.interpolate_motions(bones=bones_t, motions=motions_t, relations=relations, xyz=gauss_t,
                                             quat=quat_t, weights=dense_w, device="cpu")
    out["generic"] = dict(bones=bones_t.numpy(), motions=motions_t.numpy(), gauss=gauss_t.numpy(),
                          quat=quat_t.numpy(), relations=relations.numpy(), knn_weights=weights.numpy(),
                          knn_idx=widx.numpy(), weights=weights2.numpy(), xyz=xyz.numpy(), rot=rot.numpy(),
                          xyz_dense=xyz_d.numpy(), rot_dense=rot_d.numpy())

    # 2. dense default weights (inverse distance to every bone)
    nb2, ng2 = 120, 400
    b2 = bones[:nb2]
    m2 = motions[:nb2]
    g2 = gauss[:ng2]
    rel2 = du.get_topk_indices(t(b2), K=8)
    xyz2, rot2, w2 = du.interpolate_motions(bones=t(b2), motions=t(m2), relations=rel2, xyz=t(g2), quat=t(quat[:ng2]),
                                            device="cpu")
    out["dense_default"] = dict(bones=t(b2).numpy(), motions=t(m2).numpy(), gauss=t(g2).numpy(),
                                quat=t(quat[:ng2]).numpy(), relations=rel2.numpy(), xyz=xyz2.numpy(),
                                rot=rot2.numpy(), weights=w2.numpy())

    # 3-5. rank-deficient bones, with hand-built relations. Line bones sit on
    #    the x axis at dyadic positions and move onto the y axis, so their F is
    #    exactly rank 1 (axis e_y).
    def line_case(n_line, extra):
        tt = np.arange(n_line) / 64.0
        line = np.stack([0.25 + tt, np.full(n_line, 0.5), np.full(n_line, 0.5)], 1)
        line_m = np.stack([-tt, tt, np.zeros(n_line)], 1)
        bb = np.concatenate([line, extra[0]]) if extra is not None else line
        mm = np.concatenate([line_m, extra[1]]) if extra is not None else line_m
        return bb, mm

    gen_b = bones[:40]
    gen_m = motions[:40]
    # 3. every bone rank 1
    bb, mm = line_case(24, None)
    rel = np.array([[j for j in range(24) if j != i][:8] for i in range(24)])
    case = {"rank1_all": (bb, mm, rel)}
    # 4. exactly one rank-1 bone among generic ones: its rotation goes to all
    bb, mm = line_case(10, (gen_b, gen_m))
    gen_rel = du.get_topk_indices(t(gen_b), K=8).numpy() + 10
    rel = np.concatenate([np.array([[j for j in range(10) if j != 0][:8]]),
                          np.tile(gen_rel[:1], (9, 1)), gen_rel])
    case["rank1_one"] = (bb, mm, rel)
    # 5. two rank-1 bones: every bone gets the identity
    rel5 = rel.copy()
    rel5[1] = np.array([j for j in range(10) if j != 1][:8])
    case["rank1_two"] = (bb, mm, rel5)
    # 6. rank-0 bones (all neighbours coincide with the bone): identity everywhere
    b6 = np.concatenate([gen_b, np.repeat(gen_b[:1], 4, 0)])
    m6 = np.concatenate([gen_m, np.repeat(gen_m[:1], 4, 0)])
    rel6 = np.concatenate([du.get_topk_indices(t(gen_b), K=4).numpy(), np.array([[41, 42, 43, 40]] * 4)])
    rel6[0] = [40, 41, 42, 43]
    case["rank0_some"] = (b6, m6, rel6)
    for name, (bb_, mm_, rel_) in case.items():
        g = rng.uniform(0.2, 0.8, size=(200, 3))
        q = random_quats(200)
        w, wi = du.knn_weights_sparse(t(bb_), t(g), K=4)
        xyz_c, rot_c, _ = du.interpolate_motions_speedup(bones=t(bb_), motions=t(mm_),
                                                         relations=torch.as_tensor(rel_), xyz=t(g), quat=t(q),
                                                         weights=w, weights_indices=wi, device="cpu")
        out[name] = dict(bones=t(bb_).numpy(), motions=t(mm_).numpy(), relations=np.asarray(rel_), gauss=t(g).numpy(),
                         quat=t(q).numpy(), weights=w.numpy(), knn_idx=wi.numpy(), xyz=xyz_c.numpy(),
                         rot=rot_c.numpy())

    # 7. the quaternion helpers on random rotations, including near-180-degree ones
    Rs = np.stack([rot_about(rng.normal(size=3), a) for a in
                   np.concatenate([rng.uniform(0, np.pi, 200), np.pi - rng.uniform(0, 1e-3, 20)])])
    Rs_t = t(Rs)
    q50 = t(random_quats(50))
    out["quat"] = dict(R=Rs_t.numpy(), mat2quat=du.mat2quat(Rs_t).numpy(), quat_in=q50.numpy(),
                       quat2mat=du.quat2mat(q50).numpy())
    return out


def save(name, d):
    flat = {}
    for key, val in d.items():
        for k, v in val.items():
            flat[f"{key}/{k}"] = np.asarray(v)
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **flat)
    print("wrote", path, sum(a.nbytes for a in flat.values()) // 1024, "KiB raw")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--only", default="")
    args = ap.parse_args()
    ref = load_reference(args.reference)
    jobs = dict(kernel_stress=kernel_stress, kernel_p2g=kernel_p2g, kernel_grid=kernel_grid,
                kernel_g2p=kernel_g2p, rollouts=rollouts, kernel_restart=kernel_restart, lbs=lbs, inplace=inplace)
    for i, (name, fn) in enumerate(jobs.items()):
        if args.only and name != args.only:
            continue
        rng = np.random.default_rng(1000 + i)
        save(name, fn(ref, rng))


if __name__ == "__main__":
    main()
