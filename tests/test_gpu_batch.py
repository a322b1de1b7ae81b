"""Batched engine on the GPU: every instance of a heterogeneous batch must
match the same instance simulated alone (single-instance path) and the FP64
oracle, within the FP32 tolerance of the tests (positions 1e-4 of the domain
against the oracle; 1e-5 between the two GPU paths, which differ only in the
order of the floating-point reductions)."""
import numpy as np
import pytest
import torch

from empm_b200 import MPMModelStruct, MPMStateStruct, MPMWARPDiff
from empm_b200.batch import BatchedMPM, InstanceSpec, register_colliders
from oracle import oracle as O
from oracle.specs import MATERIAL_IDS, oracle_colliders
from tests.gpu_helpers import max_abs

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _spec(rng, n, G, material, colliders, box=(0.3, 0.6), v_scale=0.3):
    lo, side = box
    x = (lo + side * rng.uniform(size=(n, 3))).astype(np.float32)
    return InstanceSpec(
        x=x, v=(rng.standard_normal((n, 3)) * v_scale).astype(np.float32),
        vol=np.full(n, np.float32(side ** 3 / n), np.float32), rho=np.full(n, np.float32(1e3), np.float32),
        E=np.exp(rng.uniform(np.log(5e3), np.log(5e4), n)).astype(np.float32),
        nu=rng.uniform(0.25, 0.4, n).astype(np.float32),
        yield_stress=rng.uniform(5e2, 3e3, n).astype(np.float32), n_grid=G, material=material,
        colliders=colliders)


def _specs(dynamic=False):
    rng = np.random.default_rng(31)
    floor = lambda G: [dict(kind="surface", point=[0.0, 3.0 / G, 0.0], normal=[0.0, 1.0, 0.0]),  # noqa: E731
                       dict(kind="bbox")]
    specs = [
        _spec(rng, 3000, 32, "plasticine", floor(32)),
        _spec(rng, 1200, 16, "jelly", floor(16), box=(0.35, 0.3)),
        _spec(rng, 5000, 48, "plasticine", floor(48), box=(0.2, 0.5)),
        _spec(rng, 800, 24, "neo-hookean", floor(24), box=(0.4, 0.25)),
    ]
    if dynamic:
        specs[2].colliders.insert(1, dict(kind="cuboid", point=[0.45, 0.74, 0.45], size=[0.08, 0.05, 0.08],
                                          velocity=[0.0, -1.0, 0.0]))
    return specs


def _alone(spec: InstanceSpec, dt, T):
    n = spec.n
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=DEV)  # noqa: E731
    st = MPMStateStruct()
    st.init(n, device=DEV)
    st.from_torch(t(spec.x), t(spec.vol), None, t(spec.v), n_grid=spec.n_grid, device=DEV)
    st.reset_density(t(spec.rho), update_mass=True)
    md = MPMModelStruct()
    md.init(n, device=DEV)
    md.init_other_params(n_grid=spec.n_grid)
    md.gravitational_accelaration = tuple(spec.gravity)
    sv = MPMWARPDiff()
    sv.initialize(n, n_grid=spec.n_grid, device=DEV)
    sv.set_parameters_dict(md, st, {"material": spec.material})
    md.E.copy_(t(spec.E))
    md.nu.copy_(t(spec.nu))
    md.finalize_mu_lam(n)
    md.yield_stress.copy_(t(spec.yield_stress))
    register_colliders(sv, spec.colliders)
    other = st.partial_clone()
    res = sv.rollout(md, st, other, dt, T)
    return res.particle_x.clone()


def _oracle(spec: InstanceSpec, dt, T):
    sim = O.OracleSim(spec.x, spec.v, spec.vol, spec.rho.astype(np.float64) * spec.vol, spec.E, spec.nu,
                      n_grid=spec.n_grid, material=MATERIAL_IDS[spec.material], gravity=tuple(spec.gravity),
                      yield_stress=spec.yield_stress)
    sim.colliders = oracle_colliders(spec.colliders)
    sim.rollout(dt, T)
    return sim.x


@pytest.mark.parametrize("dynamic", [False, True])
def test_batch_matches_each_instance_alone(dynamic):
    specs = _specs(dynamic)
    dt, T = 2e-4, 40
    batch = BatchedMPM(specs, device=DEV)
    batch.rollout(dt, T, block=20)
    torch.cuda.synchronize()
    for i, s in enumerate(specs):
        xa = _alone(s, dt, T)
        err = max_abs(batch.positions(i), xa)
        print(f"instance {i} ({s.material}, n={s.n}, G={s.n_grid}): batch vs alone {err:.2e}")
        assert err <= 1e-5
    # one instance against the FP64 oracle
    xo = _oracle(specs[2], dt, T)
    err = max_abs(batch.positions(2), xo)
    print(f"instance 2 vs FP64 oracle: {err:.2e}")
    assert err <= 1e-4
    assert batch.read_status() & 1 == 0


def test_batch_graph_reuse_and_reload():
    """Reloading the initial state and replaying the same blocks gives the same result."""
    specs = _specs()
    batch = BatchedMPM(specs, device=DEV)
    batch.rollout(2e-4, 30, block=10)
    x1 = batch.positions().clone()
    batch.cur = 0
    batch.time = 0.0
    batch.load_state()
    batch.rollout(2e-4, 30, block=10)
    torch.cuda.synchronize()
    assert max_abs(batch.positions(), x1) <= 1e-5


@pytest.mark.parametrize("sort_every,p2g_mode,seg_cap", [(0, 0, 4), (8, 2, 4), (8, 2, 2), (8, 2, 32), (8, 1, 4),
                                                   (32, 0, 4)])
def test_batch_launch_options_agree(sort_every, p2g_mode, seg_cap):
    specs = _specs()
    ref = BatchedMPM(specs, device=DEV)
    ref.rollout(2e-4, 24, block=12)
    b = BatchedMPM(specs, device=DEV)
    b.sort_every, b.p2g_mode, b.seg_cap = sort_every, p2g_mode, seg_cap
    b.rollout(2e-4, 24, block=12)
    torch.cuda.synchronize()
    assert max_abs(b.positions(), ref.positions()) <= 1e-5


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_resumed_blocks_match_written_back_blocks(use_graph):
    """Blocks that continue from the library's sorted state (one write-back at
    the end) end where blocks that write back and re-sort every time end."""
    specs = _specs(dynamic=True)
    runs = []
    for resume in (False, True):
        b = BatchedMPM(specs, device=DEV)
        b.use_graph = use_graph
        b.resume_blocks = resume
        b.sort_every = 16
        b.rollout(2e-4, 130, block=50)
        b.rollout(2e-4, 20, block=50)        # a second call starts from the caller's buffers again
        torch.cuda.synchronize()
        runs.append((b.positions().clone(), b.mu.clone(), b.yield_stress.clone(), b._Fe.clone()))
    for a, c in zip(runs[0], runs[1]):
        assert max_abs(a, c) <= 1e-5 * max(1.0, float(c.abs().max()))


def test_rollout_resume_needs_a_sorted_state():
    from empm_b200 import _native as N
    from empm_b200.mpm_data_structure import _stream_ptr

    specs = _specs()
    b = BatchedMPM(specs, device=DEV)
    b._apply_options()
    mat = N.EmpmMaterial(b.vol.data_ptr(), b.mu.data_ptr(), b.lam.data_ptr(), b.yield_stress.data_ptr(), None,
                         b._Fe.data_ptr())
    table, n_tables = b._schedule(2e-4, 4)
    rc = b.L.empm_rollout_ex(b.ptr, b._views(0), b._views(1), mat, table, n_tables, 4, N.ROLLOUT_RESUME,
                             _stream_ptr(b.device))
    assert rc == N.EMPM_ERR_INVALID
    assert "no sorted state" in N.last_error(b.ptr)
    # after a rollout that kept its state, resuming works
    b.rollout(2e-4, 4, block=4)
    rc = b.L.empm_rollout_ex(b.ptr, b._views(b.cur), b._views(1 - b.cur), mat, table, n_tables, 4,
                             N.ROLLOUT_RESUME, _stream_ptr(b.device))
    assert rc == N.EMPM_OK
    torch.cuda.synchronize()


def _rollout_with_holds(specs, fuse, holds, T=70, dt=2e-4, sort_every=16):
    """One library rollout of the batch (stream path) with per-substep hold
    flags: holds[i] = (first, last) substeps [first, last) in which instance i
    is held."""
    from empm_b200 import _native as N
    from empm_b200.mpm_data_structure import _stream_ptr

    b = BatchedMPM(specs, device=DEV)
    b.fuse, b.sort_every = fuse, sort_every
    b._apply_options()
    mat = N.EmpmMaterial(b.vol.data_ptr(), b.mu.data_ptr(), b.lam.data_ptr(), b.yield_stress.data_ptr(), None,
                         b._Fe.data_ptr())
    table = (N.EmpmStep * (T * b.n_inst))()
    for i, sv in enumerate(b.solvers):
        t = 0.0
        for s in range(T):
            sv._fill_step(table[s * b.n_inst + i], t, dt)
            sv._modify(t, dt)
            t += dt
    for i, (first, last) in holds.items():
        for s in range(first, last):
            table[s * b.n_inst + i].hold = 1
    N.check(b.L.empm_rollout_ex(b.ptr, b._views(0), b._views(1), mat, table, T, T, 0, _stream_ptr(DEV)), b.ptr)
    torch.cuda.synchronize()
    out = 1 if T % 2 else 0
    return (b._x4[out].clone(), b._v4[out].clone(), b._C[out].clone(), b._F[out].clone(), b._Fe.clone(),
            b.yield_stress.clone(), b.read_status())


@pytest.mark.parametrize("holds", [{}, {1: (23, 70)}, {0: (5, 70), 3: (40, 70)}, {2: (10, 30)}],
                         ids=["no-holds", "held-to-end", "two-held", "released"])
def test_fused_runs_match_separate_kernels(holds):
    """Rollouts with the fused G2P + stress + P2G runs equal the separate
    kernels (state, elastic F, material) up to FP32 reduction order, with
    instances held to the end of the rollout (the serving pattern) and with a
    hold that is released again (which runs the separate kernels)."""
    specs = _specs(dynamic=True)
    fused = _rollout_with_holds(specs, True, holds)
    plain = _rollout_with_holds(specs, False, holds)
    # tolerances of the other parity tests: positions 1e-5 between GPU paths,
    # fields relative to their largest magnitude (1e-4 for C, whose run-to-run
    # spread under a different reduction order is about 3e-5 here even with
    # identical kernels: see the "released" case, which runs the separate
    # kernels in both modes)
    tol = {"x": 1e-5, "v": 1e-5, "C": 1e-4, "F_trial": 2e-5, "F_elastic": 2e-5, "yield": 1e-5}
    for name, a, c in zip(("x", "v", "C", "F_trial", "F_elastic", "yield"), fused[:6], plain[:6]):
        scale = max(1.0, float(c.abs().max()))
        err = max_abs(a, c)
        print(f"{holds}: {name} fused vs separate {err:.2e} (scale {scale:.3g})")
        assert err <= tol[name] * scale, name
    assert fused[6] & 1 == 0 and plain[6] & 1 == 0
