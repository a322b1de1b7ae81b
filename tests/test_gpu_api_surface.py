"""The rest of the reference-facing API on the GPU, against the FP64 oracle.

* MPMDifferentiableSimulationTrail (interface.py:20-251) with its quirks: a
  scalar E is scaled by 1e6 and its gradient is taken with respect to the
  scaled value (:70), the record gradients are summed over time and injected
  at the final state (:176-197), and a scalar parameter's gradient is the
  mean over particles (:210-236). Checked directly and through
  WarpMPMWrapper.run_diff_optimization (one AdamW step equals the step the
  oracle's central difference predicts).
* MPMDifferentiableSimulationClean (interface.py:777-986): gradients of the
  full state against central differences; the covariance output is the
  final partial clone's (zeros), as in the reference.
* A graph can be backpropagated twice (retain_graph) until the next
  differentiable forward pass on the same solver, then a backward raises.
* The particle and grid modifiers that had no GPU parity test:
  enforce_particle_velocity_rotation, enforce_particle_velocity_by_mask,
  add_impulse_on_particles_with_mask, release_particles_sequentially
  (mpm_solver_diff.py:1041-1212, 1353-1410) and
  enforce_grid_velocity_by_mask (:1264-1289), on the sorted rollout path and
  the per-substep path. The oracle gets the masks from a NumPy restatement of
  the reference's selection kernels (mpm_utils.py:758-808) and, for the
  layered release, the 50 separate modifiers the reference registers.

Bars: positions within 1e-4 of the domain of the FP64 oracle; gradients
within 1e-3 relative of central differences.
"""
import numpy as np
import pytest
import torch

from empm_b200 import MPMModelStruct, MPMStateStruct, MPMWARPDiff
from empm_b200.interface import (MPMDifferentiableSimulation, MPMDifferentiableSimulationClean,
                                 MPMDifferentiableSimulationTrail)
from empm_b200.warp_mpm_wrapper import WarpMPMWrapper
from oracle import oracle as O
from oracle.specs import oracle_colliders
from tests.gpu_helpers import max_abs

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
POS_GATE = 1e-4
GRAD_RTOL = 1e-3
FLOOR_WALLS = lambda G: [dict(kind="surface", point=[0.0, 3.0 / G, 0.0], normal=[0.0, 1.0, 0.0]),  # noqa: E731
                         dict(kind="bbox")]


def _t(a, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=DEV)


def _body(n=600, G=16, seed=4, speed=0.3, lo=0.35, side=0.3):
    rng = np.random.default_rng(seed)
    return dict(n=n, G=G, x=(lo + side * rng.uniform(size=(n, 3))).astype(np.float32),
                v=(speed * rng.standard_normal((n, 3))).astype(np.float32),
                vol=np.full(n, np.float32(side ** 3 / n), np.float32), rho=np.full(n, np.float32(1e3), np.float32),
                nu=np.full(n, np.float32(0.3), np.float32), gravity=(0.0, -9.8, 0.0))


def _product(b, material="jelly"):
    n, G = b["n"], b["G"]
    st = MPMStateStruct()
    st.init(n, device=DEV)
    st.from_torch(_t(b["x"]), _t(b["vol"]), None, _t(b["v"]), n_grid=G, device=DEV)
    st.reset_density(_t(b["rho"]), update_mass=True)
    md = MPMModelStruct()
    md.init(n, device=DEV)
    md.init_other_params(n_grid=G)
    md.gravitational_accelaration = b["gravity"]
    sv = MPMWARPDiff()
    sv.initialize(n, n_grid=G, device=DEV)
    sv.set_parameters_dict(md, st, {"material": material})
    md.E.fill_(2e4)
    md.nu.fill_(0.3)
    md.finalize_mu_lam(n)
    sv.add_surface_collider((0.0, 3.0 / G, 0.0), (0.0, 1.0, 0.0), "sticky", 0.0)
    sv.add_bounding_box()
    return st, md, sv


def _oracle(b, E, nu=None, x=None, v=None, mass=None, modifiers=(), colliders=None, mask=None, C=None, F=None):
    n = b["n"]
    sim = O.OracleSim(b["x"] if x is None else x, b["v"] if v is None else v, b["vol"],
                      b["vol"].astype(np.float64) * b["rho"] if mass is None else mass, E,
                      b["nu"] if nu is None else nu, n_grid=b["G"], material=0, gravity=b["gravity"])
    if C is not None:
        sim.C = np.ascontiguousarray(C, np.float64).reshape(n, 9)
    if F is not None:
        sim.F_trial = np.ascontiguousarray(F, np.float64).reshape(n, 9)
    sim.colliders = oracle_colliders(FLOOR_WALLS(b["G"]) if colliders is None else colliders, mask=mask)
    sim.modifiers = list(modifiers)
    return sim


# ---------------------------------------------------------------------------
# Trail: quirks of the trainer's autograd Function
# ---------------------------------------------------------------------------
SUB, T_TRAIL, DT = 4, 8, 2e-4


def _trail_fd(b, W_sum, E_pa, h_rel=1e-3, direction=None, what="E"):
    """Central difference of L' = sum(W_sum * x_T) in E (Pa), nu, v0, the
    density along a direction, or the Lame parameters (log scale), by the FP64
    oracle."""
    def L(mu_scale=1.0, lam_scale=1.0, **kw):
        sim = _oracle(b, **kw)
        sim.mu *= mu_scale
        sim.lam *= lam_scale
        sim.rollout(DT, T_TRAIL)
        return float((W_sum * sim.x).sum())
    if what == "E":
        h = h_rel * E_pa
        return (L(E=E_pa + h) - L(E=E_pa - h)) / (2 * h)
    if what == "nu":
        h = h_rel * 0.3
        return (L(E=E_pa, nu=np.full(b["n"], 0.3 + h)) - L(E=E_pa, nu=np.full(b["n"], 0.3 - h))) / (2 * h)
    if what in ("log_mu", "log_lam"):
        k = what[4:] + "_scale"
        return (L(E=E_pa, **{k: 1.0 + h_rel}) - L(E=E_pa, **{k: 1.0 - h_rel})) / (2 * h_rel)
    if what == "v":
        h = 1e-4
        v = b["v"].astype(np.float64)
        return (L(E=E_pa, v=v + h * direction) - L(E=E_pa, v=v - h * direction)) / (2 * h)
    if what == "rho":
        h = 1e-3
        rho = b["rho"].astype(np.float64)
        m = lambda s: b["vol"].astype(np.float64) * (rho + s * direction)  # noqa: E731
        return (L(E=E_pa, mass=m(h)) - L(E=E_pa, mass=m(-h))) / (2 * h)
    raise ValueError(what)


def test_trail_function_quirks_vs_central_differences():
    """Trail's quirks are checked against a tape of the same rollout, up to the
    order of the atomic reductions
    (the gradient in E is taken in the 1e6-scaled Pascals, a 0-d E or nu gets
    the mean over particles, and the record gradients are summed and injected
    at the final state), and its gradients against central differences of
    the FP64 oracle (bar 1e-3). The parameter gradients are sums over
    particles of terms of both signs; a sum that cancels by a factor kappa
    (sum of |terms| over |sum|, printed) loses that factor in relative
    accuracy, so its bar is 1e-3 x kappa. dL/dE and dL/dnu are also split
    into their shear (mu) and bulk (lam) parts, checked one at a time."""
    from empm_b200.adjoint import CheckpointedRollout, prepare_adjoint

    b = _body()
    n = b["n"]
    st, md, sv = _product(b)
    rng = np.random.default_rng(50)
    W = 1.0 + 0.5 * rng.standard_normal((T_TRAIL // SUB, n, 3))
    E = torch.tensor(0.02, device=DEV, requires_grad=True)      # 0-d: 2e4 Pa after the 1e6 scale
    nu = torch.tensor(0.3, device=DEV, requires_grad=True)
    v0 = _t(b["v"]).requires_grad_(True)
    rho = _t(b["rho"]).requires_grad_(True)
    dmask = torch.ones(n, dtype=torch.bool, device=DEV)           # what run_diff_optimization passes
    pos = MPMDifferentiableSimulationTrail.apply(sv, st, md, SUB, DT, T_TRAIL, _t(b["x"]), v0, E, nu, rho, dmask,
                                                 None, DEV, True, 0)
    assert tuple(pos.shape) == (T_TRAIL // SUB, n, 3)
    # records after substeps 1 and 5 (next_state_list[::substep]) against the oracle
    sim = _oracle(b, E=2e4)
    recs = []
    for s in range(T_TRAIL):
        sim.substep(DT)
        if s % SUB == 0:
            recs.append(sim.x.copy())
    for r in range(len(recs)):
        assert max_abs(pos[r], recs[r]) <= POS_GATE
    (pos * _t(W)).sum().backward()
    torch.cuda.synchronize()
    W_sum = W.sum(0)            # injected at the final state

    # the same rollout on a tape of its own, with the summed weights at the final state
    st2, md2, sv2 = _product(b)
    md2.E.fill_(float(np.float32(0.02)) * 1e6)
    md2.finalize_mu_lam(n)
    tape = CheckpointedRollout(sv2, md2, st2, DT, T_TRAIL, checkpoint_every=20, record_every=SUB)
    tape.forward()
    res = tape.backward(g_x=_t(W_sum))
    g_E, g_nu, g_rho = prepare_adjoint(md2.E, md2.nu, res["mu"], res["lam"], st2.particle_vol, res["mass"])
    # shear and bulk parts: dL/dlog(mu) and dL/dlog(lam); dL/dE = (shear + bulk) / E and
    # dL/dnu = shear * dlog(mu)/dnu + bulk * dlog(lam)/dnu. Each is a sum over particles of
    # terms of both signs; kappa = sum |term| / |sum term| is the factor by which that sum
    # cancels, and by which the FP32 rounding of its terms is amplified in it.
    ts_mu = res["mu"].double() * md2.mu.double()
    ts_lam = res["lam"].double() * md2.lam.double()
    shear, bulk = float(ts_mu.sum()), float(ts_lam.sum())
    nu0 = float(np.float32(0.3))
    dmu, dlam = -1.0 / (1.0 + nu0), 1.0 / nu0 - 1.0 / (1.0 + nu0) + 2.0 / (1.0 - 2.0 * nu0)
    kap = lambda t: float(t.abs().sum()) / abs(float(t.sum()))  # noqa: E731
    kappa = {"E": kap(ts_mu + ts_lam), "nu": kap(dmu * ts_mu + dlam * ts_lam), "log mu (shear part)": kap(ts_mu),
             "log lam (bulk part)": kap(ts_lam)}
    print("Trail cancellation factors:", {k: round(v, 1) for k, v in kappa.items()})
    exact = {"E": (float(E.grad), float(g_E.double().sum()) / n), "nu": (float(nu.grad), float(g_nu.double().sum()) / n),
             "v0": (v0.grad, res["v"]), "density": (rho.grad, g_rho)}
    for name, (a, c) in exact.items():
        err = max_abs(a, c) if isinstance(a, torch.Tensor) else abs(a - c)
        scale = float(c.abs().max()) if isinstance(c, torch.Tensor) else abs(c)
        # The two runs differ only in the order of their atomic reductions (forward and
        # adjoint); measured gaps reach about 1e-5 x kappa, so the bar is ten times that,
        # still ten times tighter than the bar against central differences below.
        tol = 1e-4 * max(1.0, kappa.get(name, 1.0))
        print(f"Trail {name}: autograd vs tape {err:.2e} (scale {scale:.3e}, tolerance {tol:.1e} relative)")
        assert err <= tol * scale, name
    assert rho.grad.shape[0] == int(dmask.sum())           # restricted to density_change_mask

    # against central differences of the FP64 oracle
    dv = rng.standard_normal((n, 3))
    drho = rng.standard_normal(n)
    E_pa = float(np.float32(0.02)) * 1e6
    strict = {"log mu (shear part)": (shear, _trail_fd(b, W_sum, E_pa, what="log_mu")),
              "log lam (bulk part)": (bulk, _trail_fd(b, W_sum, E_pa, what="log_lam")),
              "v0": (float((v0.grad.double().cpu().numpy() * dv).sum()),
                     _trail_fd(b, W_sum, E_pa, direction=dv, what="v")),
              "density": (float((rho.grad.double().cpu().numpy() * drho).sum()),
                          _trail_fd(b, W_sum, E_pa, direction=drho, what="rho"))}
    for name, (an, fd) in strict.items():
        k = kappa.get(name, 1.0)
        print(f"Trail d/d{name}: adjoint {an: .6e} fd {fd: .6e} rel {abs(an - fd) / abs(fd):.2e} "
              f"(cancellation {k:.1f}x)")
        assert abs(an - fd) <= GRAD_RTOL * max(1.0, k) * abs(fd), name
    fd_E = _trail_fd(b, W_sum, E_pa, what="E") / n
    fd_nu = _trail_fd(b, W_sum, E_pa, what="nu") / n
    for name, an, fd, k in (("E (scaled, mean)", float(E.grad), fd_E, kappa["E"]),
                            ("nu (mean)", float(nu.grad), fd_nu, kappa["nu"])):
        rel = abs(an - fd) / abs(fd)
        print(f"Trail d/d{name}: autograd {an: .6e} fd {fd: .6e} rel {rel:.2e} (shear/bulk cancellation {k:.1f}x)")
        assert rel <= GRAD_RTOL * max(1.0, k), name


def test_run_diff_optimization_one_step_matches_the_fd_step():
    b = _body(seed=8)
    n, G = b["n"], b["G"]
    rng = np.random.default_rng(51)
    W = rng.standard_normal((T_TRAIL // SUB, n, 3))
    sim = WarpMPMWrapper(grid_size=G, frame_dt=SUB * DT, sim_dt=DT, device=DEV)
    sim.gravity = list(b["gravity"])
    sim.surface_colliders.append(((0.0, 3.0 / G, 0.0), (0.0, 1.0, 0.0), "sticky", 0.0))
    sim.add_particles(b["x"], v=b["v"], vol=b["vol"], E=2e4, nu=0.3, rho=1e3)
    sim.initialize()
    Wt = _t(W)
    out = sim.run_diff_optimization({"E": 0.02}, n_train_frames=T_TRAIL // SUB, max_iters=1,
                                    loss_func=lambda p: (p * Wt).sum())
    e_new = float(out["E"])
    # the oracle with the same colliders (sticky floor only: the facade registers no walls)
    fd = _trail_fd_floor(b, W.sum(0), 2e4) / n
    lr, eps = 1e-3, 1e-8
    e_expected = float(np.float32(0.02)) - lr * fd / (abs(fd) + eps)     # first AdamW step
    print(f"run_diff_optimization: E {0.02} -> {e_new:.9f}, expected {e_expected:.9f} (fd gradient {fd:.4e})")
    assert abs(e_new - e_expected) <= 1e-3 * lr + 1e-9


def _trail_fd_floor(b, W_sum, E_pa, h_rel=1e-3):
    floor = [dict(kind="surface", point=[0.0, 3.0 / b["G"], 0.0], normal=[0.0, 1.0, 0.0])]

    def L(E):
        sim = _oracle(b, E=E, colliders=floor)
        sim.rollout(DT, T_TRAIL)
        return float((W_sum * sim.x).sum())
    h = h_rel * E_pa
    return (L(E_pa + h) - L(E_pa - h)) / (2 * h)


# ---------------------------------------------------------------------------
# Clean: gradients of the whole state
# ---------------------------------------------------------------------------
def test_clean_function_gradients_and_cov_pass_through():
    b = _body(n=500, seed=12)
    n, T = b["n"], 8
    rng = np.random.default_rng(52)
    C0 = (0.5 * rng.standard_normal((n, 3, 3))).astype(np.float32)
    F0 = (np.eye(3)[None] + 0.05 * rng.standard_normal((n, 3, 3))).astype(np.float32)
    st, md, sv = _product(b)
    st.particle_cov.copy_(_t(rng.standard_normal(6 * n)))
    x = _t(b["x"]).requires_grad_(True)
    v = _t(b["v"]).requires_grad_(True)
    F = _t(F0).requires_grad_(True)
    C = _t(C0).requires_grad_(True)
    E = _t(np.full(n, 2e4, np.float32)).requires_grad_(True)      # per particle: no averaging
    nu = torch.tensor(0.3, device=DEV, requires_grad=True)
    rho = _t(b["rho"]).requires_grad_(True)
    xo, vo, Fo, Co, covo = MPMDifferentiableSimulationClean.apply(sv, st, md, DT, T, x, v, F, C, E, nu, rho, None,
                                                                  DEV, True, 0)
    # the states of the rollout are partial clones, which do not copy the
    # covariances, and g2p_differentiable leaves them alone (mpm_utils.py:578),
    # so the reference returns the clone's zeros
    assert tuple(covo.shape) == (n, 6) and float(covo.abs().max()) == 0.0
    wx, wv, wF = rng.standard_normal((n, 3)), rng.standard_normal((n, 3)), rng.standard_normal((n, 3, 3))
    ((xo * _t(wx)).sum() + (vo * _t(wv)).sum() + (Fo * _t(wF)).sum()).backward()
    torch.cuda.synchronize()

    def L(**kw):
        base = dict(E=np.full(n, 2e4), x=b["x"].astype(np.float64), v=b["v"].astype(np.float64),
                    C=C0.astype(np.float64), F=F0.astype(np.float64))
        base.update(kw)
        sim = _oracle(b, **base)
        sim.rollout(DT, T)
        return float((wx * sim.x).sum() + (wv * sim.v).sum() + (wF.reshape(n, 9) * sim.F_trial).sum())

    checks = []
    dE = rng.standard_normal(n) * 2e4
    checks.append(("E", float((E.grad.double().cpu().numpy() * dE).sum()),
                   (L(E=2e4 + 1e-3 * dE) - L(E=2e4 - 1e-3 * dE)) / 2e-3))
    checks.append(("nu (mean)", float(nu.grad) * n,
                   (L(nu=np.full(n, 0.3 + 3e-4)) - L(nu=np.full(n, 0.3 - 3e-4))) / 6e-4))
    for name, t, base, scale, key in (("x", x, b["x"], 1e-2, "x"), ("v", v, b["v"], 0.3, "v"),
                                      ("C", C, C0, 0.5, "C"), ("F", F, F0, 0.05, "F")):
        d = rng.standard_normal(base.shape) * scale
        h = 1e-4
        fd = (L(**{key: base.astype(np.float64) + h * d}) - L(**{key: base.astype(np.float64) - h * d})) / (2 * h)
        checks.append((name, float((t.grad.double().cpu().numpy() * d).sum()), fd))
    for name, an, fd in checks:
        print(f"Clean d/d{name}: autograd {an: .6e} fd {fd: .6e} rel {abs(an - fd) / abs(fd):.2e}")
        assert abs(an - fd) <= GRAD_RTOL * abs(fd), name


# ---------------------------------------------------------------------------
# tape lifetime: double backward until the next forward
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("store", [True, False])
def test_double_backward_until_the_next_forward(store):
    b = _body(n=400, seed=13)
    st, md, sv = _product(b)
    if not store:
        sv._context(md, b["n"], st.device, max_steps=8)
        import empm_b200.interface as I
        orig = I.CheckpointedRollout

        class _Ckpt(orig):
            def __init__(self, *a, **k):
                k["store"] = False
                super().__init__(*a, **k)
        I.CheckpointedRollout = _Ckpt
    try:
        v0 = _t(b["v"]).requires_grad_(True)
        E = torch.tensor(2e4, device=DEV, requires_grad=True)
        nu = torch.tensor(0.3, device=DEV)
        args = (sv, st, md, 4, DT, 8, _t(b["x"]), v0, E, nu, _t(b["rho"]), None, None, DEV, True, 0)
        x = MPMDifferentiableSimulation.apply(*args)
        loss = (x * x).sum()
        loss.backward(retain_graph=True)
        g1 = v0.grad.clone()
        v0.grad = None
        loss.backward(retain_graph=True)
        assert max_abs(v0.grad, g1) <= 1e-6 * float(g1.abs().max())
        MPMDifferentiableSimulation.apply(*args)        # the next forward on the same solver
        with pytest.raises(RuntimeError):
            loss.backward()
    finally:
        if not store:
            I.CheckpointedRollout = orig


# ---------------------------------------------------------------------------
# particle and grid modifiers without a GPU test so far
# ---------------------------------------------------------------------------
def _box(x, point, size):
    return (np.abs(x - np.array(point, np.float32)) < np.array(size, np.float32)).all(1).astype(np.int32)


def _cylinder(x, point, normal, hh_r):
    """selection_enforce_particle_velocity_cylinder (mpm_utils.py:787-808)."""
    nrm = np.array(normal, np.float64) / np.linalg.norm(normal)
    off = x.astype(np.float64) - np.array(point)
    vert = np.abs(off @ nrm)
    horiz = np.linalg.norm(off - (off @ nrm)[:, None] * nrm[None], axis=1)
    return ((vert < hh_r[0]) & (horiz < hh_r[1])).astype(np.int32)


def _rotation_axes(normal):
    """Horizontal axes of enforce_particle_velocity_rotation (mpm_solver_diff.py:1064-1075)."""
    n = np.array(normal, np.float64) / np.linalg.norm(normal)
    h1 = np.array([1.0, 1.0, 1.0])
    if abs(float(n @ h1)) < 0.01:
        h1 = np.array([0.72, 0.37, -0.67])
    h1 = h1 - (h1 @ n) * n
    h1 = h1 / np.linalg.norm(h1)
    return n, h1, np.cross(h1, n)


def _modifier_case(kind, b, st, sv):
    """Register one modifier kind on the solver; return the oracle's specs,
    colliders and grid mask."""
    x, n, G = b["x"], b["n"], b["G"]
    rng = np.random.default_rng(60)
    colliders, gmask = FLOOR_WALLS(G), None
    if kind == "rotation":
        pt, nr, hr = [0.5, 0.5, 0.5], [0.2, 1.0, 0.1], [0.1, 0.12]
        sv.enforce_particle_velocity_rotation(st, point=pt, normal=nr, half_height_and_radius=hr,
                                              rotation_scale=3.0, translation_scale=0.2, start_time=0.0,
                                              end_time=0.004)
        nn, a1, a2 = _rotation_axes(nr)
        specs = [O.OrModifierSpec(O.MOD_ROTATION, point=tuple(pt), normal=tuple(nn), axis1=tuple(a1),
                                  axis2=tuple(a2), scale=(3.0, 0.2), start_time=0.0, end_time=0.004,
                                  mask=_cylinder(x, pt, nr, hr))]
    elif kind == "by_mask":
        m = rng.integers(0, 3, n).astype(np.int32)          # only entries equal to 1 select
        sv.enforce_particle_velocity_by_mask(st, _t(m, torch.int32), velocity=[0.2, -0.1, 0.0], start_time=0.001,
                                             end_time=0.005)
        specs = [O.OrModifierSpec(O.MOD_SET_VELOCITY, vec=(0.2, -0.1, 0.0), start_time=0.001, end_time=0.005,
                                  mask=m)]
    elif kind == "impulse_with_mask":
        pm = _t(np.ones(n, np.int32), torch.int32)
        sv.add_impulse_on_particles_with_mask(st, force=[0.0, 30.0, 0.0], dt=DT, particle_mask=pm,
                                              point=[0.45, 0.5, 0.5], size=[0.1, 0.2, 0.2], end_time=0.003)
        # the reference re-selects the given mask with the box (mpm_solver_diff.py:1389-1394)
        specs = [O.OrModifierSpec(O.MOD_IMPULSE_MASK, vec=(0.0, 30.0, 0.0), start_time=0.0, end_time=0.003,
                                  mask=_box(x, [0.45, 0.5, 0.5], [0.1, 0.2, 0.2]))]
    elif kind == "release":
        sv.release_particles_sequentially(normal=[0, 1, 0], start_position=0.65, end_position=0.35, num_layers=10,
                                          start_time=0.0, end_time=0.006, mpm_state=st)
        specs = []
        portion, t_portion = abs(0.65 - 0.35) / 50, 0.006 / 50
        for i in range(50):   # the 50 translation modifiers the reference registers
            size = [1.0, portion * (50 - i), 1.0]
            specs.append(O.OrModifierSpec(O.MOD_SET_VELOCITY, vec=(0.0, 0.0, 0.0), start_time=0.0,
                                          end_time=t_portion * (i + 1), mask=_box(x, [1.0, 0.35, 1.0], size)))
    elif kind == "grid_mask":
        gm = np.zeros((G, G, G), np.int32)
        gm[:, 9:12, :] = 1
        gm[4:7, :, 10:] = 2
        sv.enforce_grid_velocity_by_mask(_t(gm, torch.int32))
        specs, gmask = [], gm
        colliders = colliders + [dict(kind="grid_mask")]
    else:
        raise ValueError(kind)
    return specs, colliders, gmask


@pytest.mark.parametrize("path", ["rollout", "substeps"])
@pytest.mark.parametrize("kind", ["rotation", "by_mask", "impulse_with_mask", "release", "grid_mask"])
def test_modifier_vs_oracle(kind, path):
    b = _body(n=3000, G=24, seed=14, speed=0.1, lo=0.3, side=0.4)
    T = 40
    st, md, sv = _product(b)
    specs, colliders, gmask = _modifier_case(kind, b, st, sv)
    if path == "rollout":
        res = sv.rollout(md, st, st.partial_clone(), DT, T)
    else:
        cur, nxt = st, st.partial_clone()
        for _ in range(T):
            sv.p2g2p_differentiable(md, cur, nxt, DT)
            cur, nxt = nxt, cur
        res = cur
    torch.cuda.synchronize()
    sim = _oracle(b, E=np.full(b["n"], 2e4), modifiers=specs, colliders=colliders, mask=gmask)
    moved = _oracle(b, E=np.full(b["n"], 2e4), colliders=FLOOR_WALLS(b["G"]))
    sim.rollout(DT, T)
    moved.rollout(DT, T)
    effect = float(np.abs(sim.x - moved.x).max())
    err = max_abs(res.particle_x, sim.x)
    print(f"{kind} ({path}): max position error {err:.2e}; the modifier moves particles by up to {effect:.2e}")
    assert effect > 1e-4              # the case exercises the modifier
    assert err <= POS_GATE
    assert sv.read_status() & 1 == 0
