"""Adjoint kernels against central finite differences of the FP64 oracle.

For a loss with random weights on the outputs, the GPU gradient projected on
a random direction d is compared with (L(p + h d) - L(p - h d)) / 2h, both
losses evaluated by the FP64 oracle at the same (FP32-representable) inputs.
The bar is a relative error of 1e-3, the gradient tolerance against finite
differences. The GPU differentiates its FP32 forward map, so the residual is
FP32 rounding plus the O(h^2) error of the difference quotient.
"""
import numpy as np
import pytest
import torch

from empm_b200 import MPMModelStruct, MPMStateStruct, MPMWARPDiff
from empm_b200 import _native as N
from empm_b200.adjoint import CheckpointedRollout
from empm_b200.batch import register_colliders
from empm_b200.interface import MPMDifferentiableSimulationWCheckpoint
from empm_b200.mpm_data_structure import _stream_ptr
from oracle import oracle as O
from oracle.specs import MATERIAL_IDS, oracle_colliders

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
GRAD_RTOL = 1e-3


def _t(a, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=DEV)


# ---------------------------------------------------------------------------
# constitutive update (return map + stress), per particle
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("material", [0, 5, 1, 3, 2, 6, 4])
def test_constitutive_adjoint_matches_fd(material):
    rng = np.random.default_rng(100 + material)
    n = 4096
    Ft = (np.eye(3)[None] + 0.12 * rng.standard_normal((n, 3, 3))).astype(np.float32).reshape(n, 9)
    E = np.exp(rng.uniform(np.log(1e3), np.log(1e5), n))
    nu = rng.uniform(0.2, 0.4, n)
    mu = (E / (2 * (1 + nu))).astype(np.float32)
    lam = (E * nu / ((1 + nu) * (1 - 2 * nu))).astype(np.float32)
    ys = (mu * rng.uniform(0.01, 0.3, n)).astype(np.float32)   # mix of yielding and elastic particles
    dt = np.float32(2e-4)
    alpha = float(np.sqrt(2.0 / 3.0) * 2.0 * np.sin(25 / 180 * np.pi) / (3.0 - np.sin(25 / 180 * np.pi)))
    visc = 10.0 if material == 3 else 0.0
    gF = rng.standard_normal((n, 9)).astype(np.float32)
    gS = (rng.standard_normal((n, 9)) / mu[:, None]).astype(np.float32)
    gmo = (rng.standard_normal(n) / mu).astype(np.float32)
    glo = (rng.standard_normal(n) / mu).astype(np.float32)
    gyo = (rng.standard_normal(n) / mu).astype(np.float32)

    params = N.EmpmModelParams()
    params.n_grid, params.grid_lim, params.material = 16, 1.0, material
    params.softening, params.alpha, params.plastic_viscosity = 0.1, alpha, visc
    tFt, tmu, tlam, tys = _t(Ft), _t(mu), _t(lam), _t(ys)
    tgF, tgS = _t(gF), _t(gS)
    g_mu, g_lam, g_ys = _t(gmo), _t(glo), _t(gyo)
    gFt = torch.zeros_like(tFt)
    N.check(N.lib().empm_debug_stress_adjoint(params, tFt.data_ptr(), tmu.data_ptr(), tlam.data_ptr(), tys.data_ptr(),
                                              float(dt), tgF.data_ptr(), tgS.data_ptr(), g_mu.data_ptr(),
                                              g_lam.data_ptr(), g_ys.data_ptr(), gFt.data_ptr(), n,
                                              _stream_ptr(DEV)))
    torch.cuda.synchronize()
    gFt, g_mu, g_lam, g_ys = (a.double().cpu().numpy() for a in (gFt, g_mu, g_lam, g_ys))

    dF = rng.standard_normal((n, 9))
    dmu, dlam, dys = mu * rng.standard_normal(n), lam * rng.standard_normal(n), ys * rng.standard_normal(n)

    def loss(h):
        Fe, S, m2, l2, y2 = O.stress(material, Ft.astype(np.float64) + h * dF, mu + h * dmu, lam + h * dlam,
                                     ys + h * dys, float(dt), softening=0.1, alpha=alpha, plastic_viscosity=visc)
        return (gF * Fe).sum(1) + (gS * S).sum(1) + gmo * m2 + glo * l2 + gyo * y2

    h = 1e-6
    fd = (loss(h) - loss(-h)) / (2 * h)
    an = (gFt * dF).sum(1) + g_mu * dmu + g_lam * dlam + g_ys * dys
    scale = np.abs(gFt * dF).sum(1) + np.abs(g_mu * dmu) + np.abs(g_lam * dlam) + np.abs(g_ys * dys)
    ok = np.isfinite(fd) & np.isfinite(an)
    rel = np.abs(fd - an)[ok] / np.maximum(scale[ok], 1e-30)
    print(f"material {material}: finite {ok.mean():.3f}, rel err median {np.median(rel):.2e} "
          f"p99 {np.quantile(rel, 0.99):.2e} max {rel.max():.2e}")
    assert ok.mean() > 0.99
    assert np.quantile(rel, 0.99) <= GRAD_RTOL
    assert np.median(rel) <= 1e-5


# ---------------------------------------------------------------------------
# whole substeps and checkpointed segments
# ---------------------------------------------------------------------------
def _problem(material, n, G, seed, floor=False, deform=0.05, speed=0.3):
    rng = np.random.default_rng(seed)
    lo, side = (0.12, 0.3) if floor else (0.35, 0.3)
    x = (lo + side * rng.uniform(size=(n, 3))).astype(np.float32)
    if floor:
        x[:, 1] = (0.1 + 0.15 * rng.uniform(size=n)).astype(np.float32)
    p = dict(
        material=material, G=G, n=n,
        x=x, v=(speed * rng.standard_normal((n, 3))).astype(np.float32),
        C=(2.0 * rng.standard_normal((n, 9))).astype(np.float32),
        F=(np.eye(3)[None] + deform * rng.standard_normal((n, 3, 3))).reshape(n, 9).astype(np.float32),
        vol=np.full(n, np.float32(side ** 3 / n), np.float32),
        E=np.exp(rng.uniform(np.log(5e3), np.log(5e4), n)).astype(np.float32),
        nu=rng.uniform(0.25, 0.4, n).astype(np.float32),
        gravity=(0.0, -9.8, 0.0),
        colliders=[dict(kind="surface", point=[0.0, 3.0 / G, 0.0], normal=[0.0, 1.0, 0.0]), dict(kind="bbox")],
    )
    p["mass"] = (p["vol"] * np.float32(1e3)).astype(np.float32)
    mu = p["E"] / (2 * (1 + p["nu"]))
    p["ys"] = (mu * rng.uniform(0.005, 0.05, n)).astype(np.float32) if material in (1, 5) else \
        np.zeros(n, np.float32)
    return p


def _setup(p, dt):
    """State, model and solver of problem p on the GPU."""
    n, G = p["n"], p["G"]
    st = MPMStateStruct()
    st.init(n, device=DEV)
    st.from_torch(_t(p["x"]), _t(p["vol"]), None, _t(p["v"]), n_grid=G, device=DEV)
    st.particle_C = _t(p["C"])
    st.particle_F_trial = _t(p["F"])
    st.particle_mass = _t(p["mass"])
    md = MPMModelStruct()
    md.init(n, device=DEV)
    md.init_other_params(n_grid=G)
    md.material = p["material"]
    md.gravitational_accelaration = p["gravity"]
    md.E.copy_(_t(p["E"]))
    md.nu.copy_(_t(p["nu"]))
    md.finalize_mu_lam(n)
    md.yield_stress.copy_(_t(p["ys"]))
    md.rpic_damping = p.get("rpic", 0.0)
    md.grid_v_damping_scale = p.get("damping", 1.1)
    if p.get("sel") is not None:
        st.set_selection(_t(p["sel"], torch.int32))
    sv = MPMWARPDiff()
    sv.initialize(n, n_grid=G, device=DEV)
    sv.sort_every = p.get("sort_every", 16)
    sv.adj_store = p.get("adj_store", True)
    sv.seg_cap = p.get("seg_cap", sv.seg_cap)
    for m in p.get("modifiers", []):
        if m["kind"] == "impulse":
            sv.add_impulse_on_particles(st, force=m["force"], dt=dt, point=m["point"], size=m["size"],
                                        num_dt=m["num_dt"])
        elif m["kind"] == "translation":
            sv.enforce_particle_velocity_translation(st, point=m["point"], size=m["size"], velocity=m["velocity"],
                                                     start_time=m["start_time"], end_time=m["end_time"])
        elif m["kind"] == "mover":
            sv.set_particle_mover(velocity=m["velocity"], angular_velocity=m["angular_velocity"], center=m["center"],
                                  axis=m["axis"], selection_mask=_t(m["mask"], torch.int32), device=DEV)
    register_colliders(sv, p["colliders"])
    return st, md, sv


def _gpu(p, dt, T, every, weights):
    n = p["n"]
    st, md, sv = _setup(p, dt)
    mu0, lam0 = md.mu.double().cpu().numpy(), md.lam.double().cpu().numpy()
    tape = CheckpointedRollout(sv, md, st, dt, T, checkpoint_every=every, store=p.get("tape_store"))
    tape.forward()
    if p.get("tape_store") is not None:
        assert tape.stored == p["tape_store"]
    wx, wv, wC, wF = weights
    res = tape.backward(g_x=_t(wx), g_v=_t(wv), g_C=_t(wC), g_F=_t(wF))
    torch.cuda.synchronize()
    return {k: v.double().cpu().numpy().reshape(n, -1) for k, v in res.items()}, mu0, lam0, tape


def _oracle_loss(p, mu, lam, dt, T, weights, d=None, h=0.0):
    d = d or {}
    g = lambda k, base: base + h * d[k] if k in d else base  # noqa: E731
    n = p["n"]
    sim = O.OracleSim(g("x", p["x"].astype(np.float64)), g("v", p["v"].astype(np.float64)), p["vol"],
                      g("mass", p["mass"].astype(np.float64)), p["E"], p["nu"], n_grid=p["G"],
                      material=p["material"], gravity=p["gravity"], yield_stress=g("ys", p["ys"].astype(np.float64)),
                      rpic_damping=p.get("rpic", 0.0), grid_v_damping_scale=p.get("damping", 1.1),
                      selection=p.get("sel"))
    sim.C = np.ascontiguousarray(g("C", p["C"].astype(np.float64)).reshape(n, 9))
    sim.F_trial = np.ascontiguousarray(g("F", p["F"].astype(np.float64)).reshape(n, 9))
    sim.mu = np.ascontiguousarray(g("mu", mu))
    sim.lam = np.ascontiguousarray(g("lam", lam))
    sim.colliders = oracle_colliders(p["colliders"])
    sim.modifiers = _oracle_modifiers(p, dt)
    sim.rollout(dt, T)
    wx, wv, wC, wF = weights
    return float((wx * sim.x).sum() + (wv * sim.v).sum() + (wC * sim.C).sum() + (wF * sim.F_trial).sum())


def _oracle_modifiers(p, dt):
    """The modifiers of p as the oracle's specs; masks from the initial positions,
    as the solver computes them when a modifier is registered."""
    x = p["x"]
    box = lambda c, sz: (np.abs(x - np.array(c)) < np.array(sz)).all(1).astype(np.int32)  # noqa: E731
    out = []
    for m in p.get("modifiers", []):
        if m["kind"] == "impulse":
            out.append(O.OrModifierSpec(O.MOD_IMPULSE, vec=tuple(m["force"]), start_time=0.0,
                                        end_time=dt * m["num_dt"], mask=box(m["point"], m["size"])))
        elif m["kind"] == "translation":
            out.append(O.OrModifierSpec(O.MOD_SET_VELOCITY, vec=tuple(m["velocity"]), start_time=m["start_time"],
                                        end_time=m["end_time"], mask=box(m["point"], m["size"])))
        elif m["kind"] == "mover":
            out.append(O.OrModifierSpec(O.MOD_MOVER, vec=tuple(m["velocity"]), point=tuple(m["center"]),
                                        normal=tuple(m["axis"]), scale=(m["angular_velocity"], 0.0),
                                        mask=np.ascontiguousarray(m["mask"], dtype=np.int32)))
    return out


def _check_directional(p, dt, T, every, seed, h_rel=1e-6, rtol=GRAD_RTOL):
    rng = np.random.default_rng(seed)
    n = p["n"]
    weights = (rng.standard_normal((n, 3)), rng.standard_normal((n, 3)), 0.01 * rng.standard_normal((n, 9)),
               rng.standard_normal((n, 9)))
    res, mu, lam, tape = _gpu(p, dt, T, every, weights)
    dirs = {
        "x": 0.01 * rng.standard_normal((n, 3)), "v": rng.standard_normal((n, 3)), "C": rng.standard_normal((n, 9)),
        "F": 0.1 * rng.standard_normal((n, 9)), "mu": mu * rng.standard_normal(n), "lam": lam * rng.standard_normal(n),
        "mass": p["mass"] * rng.standard_normal(n),
    }
    if p["material"] in (1, 5):
        dirs["ys"] = p["ys"] * rng.standard_normal(n)
    keymap = {"x": "x", "v": "v", "C": "C", "F": "F", "mu": "mu", "lam": "lam", "mass": "mass", "ys": "yield_stress"}
    out = {}
    for k, d in dirs.items():
        fd = (_oracle_loss(p, mu, lam, dt, T, weights, {k: d}, h_rel) -
              _oracle_loss(p, mu, lam, dt, T, weights, {k: d}, -h_rel)) / (2 * h_rel)
        an = float((res[keymap[k]].reshape(d.shape) * d).sum())
        out[k] = (an, fd)
        print(f"  d{k}: adjoint {an: .6e}  fd {fd: .6e}  rel {abs(an - fd) / max(abs(fd), 1e-30):.2e}")
    for k, (an, fd) in out.items():
        assert abs(an - fd) <= rtol * abs(fd) + 1e-9, k
    return tape


def test_single_substep_adjoint_jelly():
    p = _problem(0, n=800, G=16, seed=1)
    _check_directional(p, 2e-4, 1, 1, seed=11)


@pytest.mark.parametrize("sort_every", [16, 0])
def test_segment_adjoint_plasticine_yielding(sort_every):
    """Cell-sorted segments (sort_every > 0) and the caller-order path."""
    # strong initial deformation so that most particles are on the yield surface
    p = _problem(5, n=800, G=16, seed=2, deform=0.25, speed=0.5)
    p["sort_every"] = sort_every
    tape = _check_directional(p, 2e-4, 6, 4, seed=12)
    assert tape.bounds == [0, 4, 6]


@pytest.mark.parametrize("seg_cap", [1, 32])
def test_segment_adjoint_run_caps(seg_cap):
    """Same-cell runs capped at 1 or 32 lanes: the G2P adjoint's shuffle
    reduction takes its general form (the default cap of 4 has one with the
    rounds fixed at compile time), checked against finite differences."""
    p = _problem(5, n=800, G=16, seed=2, deform=0.25, speed=0.5)
    p["seg_cap"] = seg_cap
    _check_directional(p, 2e-4, 6, 4, seed=12)


def test_segment_adjoint_with_floor_contact():
    # strong deformation: most particles yield well clear of the yield surface, so
    # FP32 and FP64 take the same branch for them
    p = _problem(5, n=1000, G=24, seed=3, floor=True, deform=0.25, speed=0.5)
    p["v"][:, 1] = np.float32(-1.5)
    _check_directional(p, 2e-4, 12, 5, seed=13)


def test_segment_adjoint_modifiers_selection_damping():
    """Velocity modifiers (impulse, velocity override, mover), unsimulated
    particles, RPIC damping, grid damping and a moving cuboid collider."""
    dt = 2e-4
    p = _problem(0, n=900, G=16, seed=5, speed=0.3)
    rng = np.random.default_rng(55)
    p["sel"] = (rng.uniform(size=p["n"]) < 0.05).astype(np.int32)
    p["rpic"] = 0.3
    p["damping"] = 0.98
    p["colliders"] = [dict(kind="cuboid", point=[0.5, 0.62, 0.5], size=[0.06, 0.03, 0.06], velocity=[0.0, -0.5, 0.0]),
                      dict(kind="bbox")]
    p["modifiers"] = [
        dict(kind="impulse", force=[0.0, 0.0, 2e-3], point=[0.45, 0.45, 0.45], size=[0.08, 0.08, 0.08], num_dt=3),
        dict(kind="translation", point=[0.58, 0.45, 0.5], size=[0.05, 0.05, 0.05], velocity=[0.2, 0.0, 0.0],
             start_time=0.0, end_time=0.004),
        dict(kind="mover", velocity=[0.0, 0.0, -0.01], angular_velocity=2.0, center=[0.5, 0.5, 0.5],
             axis=[0.0, 1.0, 0.0], mask=(rng.uniform(size=p["n"]) < 0.2).astype(np.int32)),
    ]
    _check_directional(p, dt, 6, 4, seed=15)


@pytest.mark.parametrize("sort_every", [16, 0])
def test_segment_adjoint_store_matches_recompute(sort_every):
    """The three ways to run the reverse pass give the same gradients:
    - segments stored by the tape's forward pass (empm_segment_*);
    - checkpoints whose segments are re-run with the grids and elastic F kept;
    - checkpoints whose grids are recomputed in the reverse pass.
    They agree up to the order of the P2G's floating-point atomics, which a
    re-run does not repeat: a particle close to the yield surface can take the
    other branch, so the bound is on the norm of each gradient."""
    dt = 2e-4
    p = _problem(5, n=1000, G=24, seed=7, floor=True, deform=0.25, speed=0.5)
    p["v"][:, 1] = np.float32(-1.5)
    p["sort_every"] = sort_every
    p["modifiers"] = [dict(kind="impulse", force=[0.0, 0.0, 2e-3], point=[0.5, 0.3, 0.5], size=[0.1, 0.1, 0.1],
                           num_dt=3)]
    rng = np.random.default_rng(17)
    n = p["n"]
    weights = (rng.standard_normal((n, 3)), rng.standard_normal((n, 3)), 0.01 * rng.standard_normal((n, 9)),
               rng.standard_normal((n, 9)))
    outs = []
    for tape_store, adj_store in ((False, False), (False, True), (True, True)):
        p["tape_store"], p["adj_store"] = tape_store, adj_store
        res, _, _, _ = _gpu(p, dt, 12, 5, weights)
        outs.append(res)
    for name, other in (("checkpoint + grid store", outs[1]), ("stored tape", outs[2])):
        for k in outs[0]:
            a, b = other[k], outs[0][k]
            rel = float(np.linalg.norm(a - b)) / max(float(np.linalg.norm(b)), 1e-30)
            print(f"  {name} {k}: |a - recompute| / |recompute| = {rel:.2e}")
            assert rel <= 2e-3, (name, k, rel)


@pytest.mark.parametrize("store", [True, False])
@pytest.mark.parametrize("sort_every", [16, 0])
def test_segment_graphs_match_direct_launches(sort_every, store):
    """Stored segments capture their substep loops as CUDA graphs on first use
    and replay them on later passes of the pooled segments; checkpointed
    segments (re-run in the reverse pass) replay graphs cached in the context.
    Replayed passes, including one whose step tables changed (a later start
    time moves the impulse's gate), give the gradients of the same passes
    launched kernel by kernel, up to the order of the atomics."""
    dt, T, every = 2e-4, 10, 4
    p = _problem(5, n=1500, G=24, seed=21, floor=True, deform=0.25, speed=0.5)
    p["v"][:, 1] = np.float32(-1.0)
    p["sort_every"] = sort_every
    p["modifiers"] = [dict(kind="impulse", force=[0.0, 0.0, 2e-3], point=[0.3, 0.2, 0.3], size=[0.15, 0.15, 0.15],
                           num_dt=3)]
    n = p["n"]
    rng = np.random.default_rng(23)
    g_x = _t(rng.standard_normal((n, 3)))
    g_v = _t(rng.standard_normal((n, 3)))

    def run(graphs, t0, passes):
        st, md, sv = _setup(p, dt)
        sv.segment_graph = graphs
        x0, v0 = st.particle_x.clone(), st.particle_v.clone()
        mat0 = (md.mu.clone(), md.lam.clone(), md.yield_stress.clone())
        out = []
        for _ in range(passes):
            st.particle_x = x0
            st.particle_v = v0
            for dst, src in zip((md.mu, md.lam, md.yield_stress), mat0):
                dst.copy_(src)
            sv.time = t0
            tape = CheckpointedRollout(sv, md, st, dt, T, checkpoint_every=every, store=store)
            final = tape.forward()
            assert tape.stored == store
            res = tape.backward(g_x=g_x, g_v=g_v)
            torch.cuda.synchronize()
            out.append((final.particle_x.double().cpu().numpy(),
                        {k: v.double().cpu().numpy() for k, v in res.items()}))
            tape.release()
        return out

    for t0 in (0.0, 1.5 * dt):
        replayed = run(True, t0, 3)      # pass 1 may size the segments; later passes replay
        direct = run(False, t0, 1)[0]
        for xf, res in replayed[1:]:
            assert float(np.abs(xf - direct[0]).max()) <= 1e-5
            for k in res:
                a, b = res[k], direct[1][k]
                rel = float(np.linalg.norm(a - b)) / max(float(np.linalg.norm(b)), 1e-30)
                assert rel <= 2e-3, (t0, k, rel)


def test_fused_stored_forward_matches_separate_kernels():
    """The stored forward pass of a cell-sorted tape runs the G2P of one
    substep and the stress + P2G of the next as one kernel that writes the
    tape itself; with the separate kernels (EMPM_OPT_FUSE 0) the same rollout
    gives the same final state and gradients, up to the order of the atomics."""
    dt, T, every = 2e-4, 12, 5
    p = _problem(5, n=1500, G=24, seed=31, floor=True, deform=0.25, speed=0.5)
    p["v"][:, 1] = np.float32(-1.5)
    p["modifiers"] = [dict(kind="impulse", force=[0.0, 0.0, 2e-3], point=[0.3, 0.2, 0.3], size=[0.15, 0.15, 0.15],
                           num_dt=3)]
    n = p["n"]
    rng = np.random.default_rng(33)
    g_x = _t(rng.standard_normal((n, 3)))
    g_F = _t(rng.standard_normal((n, 9)))
    outs = []
    for fuse in (True, False):
        st, md, sv = _setup(p, dt)
        sv.fuse = fuse
        tape = CheckpointedRollout(sv, md, st, dt, T, checkpoint_every=every, store=True)
        final = tape.forward()
        res = tape.backward(g_x=g_x, g_F=g_F)
        torch.cuda.synchronize()
        outs.append((final.particle_x.double().cpu().numpy(), md.mu.double().cpu().numpy(),
                     {k: v.double().cpu().numpy() for k, v in res.items()}))
    (xa, mua, ra), (xb, mub, rb) = outs
    assert float(np.abs(xa - xb).max()) <= 1e-5
    assert float(np.abs(mua - mub).max()) <= 1e-5 * float(np.abs(mub).max())
    for k in rb:
        rel = float(np.linalg.norm(ra[k] - rb[k])) / max(float(np.linalg.norm(rb[k])), 1e-30)
        print(f"  fused vs separate {k}: {rel:.2e}")
        assert rel <= 2e-3, (k, rel)


@pytest.mark.parametrize("sort_every", [16, 0])
def test_checkpointed_segments_fd(sort_every):
    """Finite differences through checkpointed segments (re-run in the reverse
    pass), the path taken when the stored rollout does not fit."""
    p = _problem(5, n=800, G=16, seed=2, deform=0.25, speed=0.5)
    p["sort_every"] = sort_every
    p["tape_store"] = False
    _check_directional(p, 2e-4, 6, 4, seed=12)


def test_stored_forward_matches_rollout():
    """The stored forward pass ends where the plain rollout ends, and the
    budget decides between storing and checkpointing."""
    dt, T = 2e-4, 12
    p = _problem(5, n=1000, G=24, seed=9, floor=True, deform=0.25, speed=0.5)
    finals = []
    for store in (True, False):
        p["tape_store"] = store
        rng = np.random.default_rng(3)
        n = p["n"]
        w = (rng.standard_normal((n, 3)), rng.standard_normal((n, 3)), rng.standard_normal((n, 9)),
             rng.standard_normal((n, 9)))
        _, _, _, tape = _gpu(p, dt, T, 5, w)
        finals.append((tape.final.particle_x.double().cpu().numpy(), tape.final.particle_v.double().cpu().numpy(),
                       tape.model.mu.double().cpu().numpy()))
    for a, b in zip(finals[0], finals[1]):
        assert float(np.abs(a - b).max()) <= 1e-5 * max(1.0, float(np.abs(b).max()))
    # a budget of one byte: automatic mode checkpoints, forced storing refuses
    p["tape_store"] = None
    st, md, sv = _setup(p, dt)
    tape = CheckpointedRollout(sv, md, st, dt, T, checkpoint_every=5, store_budget=1)
    tape.forward()
    assert not tape.stored and len(tape.ckpts) == 3
    tape = CheckpointedRollout(sv, md, st, dt, T, checkpoint_every=5, store=True, store_budget=1)
    with pytest.raises(MemoryError):
        tape.forward()
    # released segments go to the context's pool and the next rollout takes
    # them (once a first pass has measured the touched blocks: segments sized
    # by the first guess are freed instead)
    tape = CheckpointedRollout(sv, md, st, dt, T, checkpoint_every=5, store=True)
    tape.forward()
    assert sv._ctx.touched_blocks is not None
    tape.release()
    tape = CheckpointedRollout(sv, md, st, dt, T, checkpoint_every=5, store=True)
    tape.forward()
    ctx = sv._ctx
    first = [sg.ptr.value for sg in tape.segments]
    tape.release()
    assert ctx.pooled(5) == 2 and ctx.pooled(2) == 1
    tape2 = CheckpointedRollout(sv, md, st, dt, T, checkpoint_every=5, store=True)
    tape2.forward()
    assert sorted(sg.ptr.value for sg in tape2.segments) == sorted(first)
    assert ctx.pooled(5) == 0 and ctx.pooled(2) == 0
    del tape2
    sv.release_tape_memory()
    assert ctx.pooled(5) == 0
    # a grid store too small for the touched blocks: the pass is repeated with
    # room for the observed counts and ends where the checkpointed pass ends
    q = _problem(5, n=2000, G=32, seed=9, deform=0.25, speed=0.5)   # ~64 touched blocks per substep
    n = q["n"]
    rng = np.random.default_rng(4)
    g = torch.as_tensor(rng.standard_normal((n, 3)).astype(np.float32), device=DEV)
    outs = []
    for store, hint in ((True, 1), (False, None)):
        st, md, sv = _setup(q, dt)
        if hint is not None:
            sv._context(md, n, st.device, max_steps=T).touched_blocks = hint
        tape = CheckpointedRollout(sv, md, st, dt, T, checkpoint_every=5, store=store)
        final = tape.forward()
        assert tape.stored == store
        if store:
            assert sv._ctx.touched_blocks > int(hint * 1.25) + 16
            assert all(sg.block_cap >= sv._ctx.touched_blocks for sg in tape.segments)
        res = tape.backward(g_x=g)
        outs.append((final.particle_x.double().cpu().numpy(), res["v"].double().cpu().numpy()))
    assert float(np.abs(outs[0][0] - outs[1][0]).max()) <= 1e-5
    rel = float(np.linalg.norm(outs[0][1] - outs[1][1])) / float(np.linalg.norm(outs[1][1]))
    assert rel <= 2e-3, rel


# ---------------------------------------------------------------------------
# the reference's autograd boundary
# ---------------------------------------------------------------------------
def test_wcheckpoint_function_gradients():
    p = _problem(5, n=600, G=16, seed=4, deform=0.1, speed=0.4)
    n, dt, T = p["n"], 2e-4, 8
    st = MPMStateStruct()
    st.init(n, device=DEV)
    st.from_torch(_t(p["x"]), _t(p["vol"]), None, _t(p["v"]), n_grid=p["G"], device=DEV)
    md = MPMModelStruct()
    md.init(n, device=DEV)
    md.init_other_params(n_grid=p["G"])
    md.material = 5
    md.gravitational_accelaration = p["gravity"]
    md.yield_stress.copy_(_t(p["ys"]))
    sv = MPMWARPDiff()
    sv.initialize(n, n_grid=p["G"], device=DEV)
    sv.checkpoint_every = 3
    register_colliders(sv, p["colliders"])
    x = _t(p["x"]).requires_grad_(True)
    v = _t(p["v"]).requires_grad_(True)
    F = _t(p["F"]).reshape(n, 3, 3).requires_grad_(True)
    C = _t(p["C"]).reshape(n, 3, 3).requires_grad_(True)
    E = torch.tensor(2e4, device=DEV, requires_grad=True)       # scalar: aggregated gradient
    nu = _t(p["nu"]).requires_grad_(True)                        # per particle
    rho = _t(np.full(n, 1e3, np.float32)).requires_grad_(True)
    rng = np.random.default_rng(40)
    wx, wv = rng.standard_normal((n, 3)), rng.standard_normal((n, 3))
    xo, vo, Fo, Co = MPMDifferentiableSimulationWCheckpoint.apply(sv, st, md, dt, T, x, v, F, C, E, nu, rho, None,
                                                                  DEV, True, 0)
    loss = (xo * _t(wx)).sum() + (vo * _t(wv)).sum()
    loss.backward()
    torch.cuda.synchronize()

    zero = lambda s: np.zeros(s)  # noqa: E731
    weights = (wx, wv, zero((n, 9)), zero((n, 9)))
    q = dict(p)
    q["E"] = np.full(n, np.float32(2e4), np.float32)
    q["mass"] = (p["vol"] * np.float32(1e3)).astype(np.float32)

    def oracle_loss(E_val=2e4, nu_arr=None, rho_arr=None, h=0.0, dx=None):
        r = dict(q)
        E_arr = np.full(n, E_val, np.float64)
        nu_a = q["nu"].astype(np.float64) if nu_arr is None else nu_arr
        mu = E_arr / (2 * (1 + nu_a))
        lam = E_arr * nu_a / ((1 + nu_a) * (1 - 2 * nu_a))
        if rho_arr is not None:
            r["mass"] = p["vol"].astype(np.float64) * rho_arr
        d = {} if dx is None else {"x": dx}
        return _oracle_loss(r, mu, lam, dt, T, weights, d, h)

    h = 1e-3   # relative step on E (E = 2e4)
    fd_E = (oracle_loss(E_val=2e4 * (1 + h)) - oracle_loss(E_val=2e4 * (1 - h))) / (2 * 2e4 * h)
    an_E = float(E.grad) * n      # the reference returns sum(dL/dE_p) / N for a scalar E
    dnu = rng.standard_normal(n) * 0.01
    fd_nu = (oracle_loss(nu_arr=q["nu"] + 1e-4 * dnu) - oracle_loss(nu_arr=q["nu"] - 1e-4 * dnu)) / 2e-4
    an_nu = float((nu.grad.double().cpu().numpy() * dnu).sum())
    drho = rng.standard_normal(n) * 1e3
    fd_rho = (oracle_loss(rho_arr=1e3 + 1e-6 * drho) - oracle_loss(rho_arr=1e3 - 1e-6 * drho)) / 2e-6
    an_rho = float((rho.grad.double().cpu().numpy() * drho).sum())
    ddx = rng.standard_normal((n, 3)) * 0.01
    fd_x = (oracle_loss(h=1e-6, dx=ddx) - oracle_loss(h=-1e-6, dx=ddx)) / 2e-6
    an_x = float((x.grad.double().cpu().numpy() * ddx).sum())
    for name, an, fd in (("E", an_E, fd_E), ("nu", an_nu, fd_nu), ("density", an_rho, fd_rho), ("x", an_x, fd_x)):
        print(f"  {name}: autograd {an: .6e}  fd {fd: .6e}  rel {abs(an - fd) / abs(fd):.2e}")
        assert abs(an - fd) <= GRAD_RTOL * abs(fd), name
    assert v.grad is not None and F.grad is not None and C.grad is not None
    assert E.grad.ndim == 0
