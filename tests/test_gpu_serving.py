"""The request loop on the GPU. Each result must be the same alone and in a
mix of concurrent requests: 1e-5 of the domain for positions (the tolerance
between two GPU paths that differ only in reduction order) and 1e-4 relative
for gradients. Also checked: a forward result against the FP64 oracle
(1e-4), a request's gradient against the single-instance differentiable
rollout, a Poisson stream of mixed requests, and host-injected faults."""
import time

import numpy as np
import pytest
import torch

from empm_b200 import MPMModelStruct, MPMStateStruct, MPMWARPDiff
from empm_b200.adjoint import CheckpointedRollout, prepare_adjoint
from empm_b200.batch import InstanceSpec, register_colliders
from empm_b200.serving import Capacity, MPMServer, Request, grid_blocks
from oracle import oracle as O
from oracle.specs import oracle_colliders

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _spec(rng, n, G):
    lo = rng.uniform(0.2, 0.45, 3)
    side = rng.uniform(0.15, 0.3)
    x = (lo + side * rng.uniform(size=(n, 3))).astype(np.float32)
    x[:, 1] = (0.15 + (x[:, 1] - lo[1])).astype(np.float32)
    return InstanceSpec(
        x=x, v=(0.2 * rng.standard_normal((n, 3))).astype(np.float32),
        vol=np.full(n, np.float32(side ** 3 / n), np.float32), rho=np.full(n, np.float32(1e3), np.float32),
        E=np.exp(rng.uniform(np.log(1e3), np.log(1e5), n)).astype(np.float32),
        nu=rng.uniform(0.2, 0.45, n).astype(np.float32),
        yield_stress=rng.uniform(5e2, 5e3, n).astype(np.float32), n_grid=G, material="plasticine",
        colliders=[dict(kind="surface", point=[0.0, 3.0 / G, 0.0], normal=[0.0, 1.0, 0.0]), dict(kind="bbox")])


def _request(seed, n, G, T, grad=False):
    rng = np.random.default_rng(seed)
    s = _spec(rng, n, G)
    tgt = (s.x + np.float32(0.01) * rng.standard_normal((n, 3)).astype(np.float32)) if grad else None
    return Request(spec=s, n_substeps=T, dt=1e-4, grad=grad, target=tgt)


def _server(**kw):
    cap = Capacity(particles=kw.pop("particles", 120_000), blocks=kw.pop("blocks", 60_000),
                   instances=kw.pop("instances", 16), ckpt_bytes=kw.pop("ckpt", 2 << 30),
                   adjoint_particles=kw.pop("adjoint_particles", 40_000), adjoint_blocks=grid_blocks(64))
    return MPMServer(capacity=cap, device=DEV, **kw).start()


def _single_gradient(req: Request):
    """The same loss through the single-instance differentiable rollout."""
    s = req.spec
    n = s.n
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=DEV)  # noqa: E731
    st = MPMStateStruct()
    st.init(n, device=DEV)
    st.from_torch(t(s.x), t(s.vol), None, t(s.v), n_grid=s.n_grid, device=DEV)
    st.reset_density(t(s.rho), update_mass=True)
    md = MPMModelStruct()
    md.init(n, device=DEV)
    md.init_other_params(n_grid=s.n_grid)
    md.gravitational_accelaration = tuple(s.gravity)
    sv = MPMWARPDiff()
    sv.initialize(n, n_grid=s.n_grid, device=DEV)
    sv.set_parameters_dict(md, st, {"material": s.material})
    md.E.copy_(t(s.E))
    md.nu.copy_(t(s.nu))
    md.finalize_mu_lam(n)
    md.yield_stress.copy_(t(s.yield_stress))
    register_colliders(sv, s.colliders)
    tape = CheckpointedRollout(sv, md, st, req.dt, req.n_substeps, checkpoint_every=20)
    x = tape.forward().particle_x
    diff = x - t(req.target)
    res = tape.backward(g_x=2.0 * diff / n)
    gE, gnu, _ = prepare_adjoint(md.E, md.nu, res["mu"], res["lam"])
    return (float((diff * diff).sum(1).mean()), res["v"].cpu().numpy(), float(gE.sum()), float(gnu.sum()),
            float(res["yield_stress"].sum()))


def test_results_same_alone_and_in_the_mix():
    R = _request(1, 5000, 32, 120)
    Rg = _request(2, 3000, 24, 80, grad=True)
    srv = _server()
    try:
        alone = srv.submit(R).wait(120)
        alone_g = srv.submit(Rg).wait(120)
    finally:
        srv.stop(timeout=300)
    assert alone.status == "ok" and alone_g.status == "ok", (alone.error, alone_g.error)

    srv = _server()
    try:
        others = [srv.submit(_request(10 + i, n, G, T, grad=(i % 3 == 2)))
                  for i, (n, G, T) in enumerate([(8000, 48, 150), (2000, 16, 60), (12000, 40, 90)])]
        time.sleep(0.02)
        tk = srv.submit(R)
        others += [srv.submit(_request(20 + i, n, G, T, grad=(i == 1)))
                   for i, (n, G, T) in enumerate([(4000, 24, 200), (6000, 32, 70)])]
        tkg = srv.submit(Rg)
        others.append(srv.submit(_request(30, 1500, 20, 40)))
        mix, mix_g = tk.wait(300), tkg.wait(300)
        rest = [o.wait(300) for o in others]
    finally:
        srv.stop(timeout=300)
    assert mix.status == "ok" and mix_g.status == "ok"
    assert all(r.status == "ok" for r in rest), [r.error for r in rest]
    err = float(np.abs(mix.x - alone.x).max())
    print(f"forward request: max |x_mix - x_alone| = {err:.2e}")
    assert err <= 1e-5
    errg = float(np.abs(mix_g.x - alone_g.x).max())
    print(f"gradient request: max |x_mix - x_alone| = {errg:.2e}, loss {alone_g.loss:.6e} / {mix_g.loss:.6e}")
    assert errg <= 1e-5
    for k in ("E", "nu", "yield_stress"):
        a, b = alone_g.grads[k], mix_g.grads[k]
        print(f"  dL/d{k}: alone {a: .6e} mix {b: .6e}")
        assert abs(a - b) <= 1e-4 * max(abs(a), 1e-30), k
    gv_scale = float(np.abs(alone_g.grads["v0"]).max())
    assert float(np.abs(mix_g.grads["v0"] - alone_g.grads["v0"]).max()) <= 1e-4 * gv_scale

    # the forward request against the FP64 oracle
    s = R.spec
    sim = O.OracleSim(s.x, s.v, s.vol, s.rho.astype(np.float64) * s.vol, s.E, s.nu, n_grid=s.n_grid, material=5,
                      gravity=tuple(s.gravity), yield_stress=s.yield_stress)
    sim.colliders = oracle_colliders(s.colliders)
    sim.rollout(R.dt, R.n_substeps)
    err_o = float(np.abs(alone.x - sim.x).max())
    print(f"forward request vs FP64 oracle: {err_o:.2e}")
    assert err_o <= 1e-4

    # the gradient request against the single-instance differentiable rollout
    loss, gv, gE, gnu, gys = _single_gradient(Rg)
    print(f"single-instance tape: loss {loss:.6e}, dL/dE {gE:.6e}, dL/dnu {gnu:.6e}, dL/dyield {gys:.6e}")
    assert abs(alone_g.loss - loss) <= 1e-5 * loss
    for a, b in ((alone_g.grads["E"], gE), (alone_g.grads["nu"], gnu), (alone_g.grads["yield_stress"], gys)):
        assert abs(a - b) <= 1e-4 * max(abs(b), 1e-30)
    assert float(np.abs(alone_g.grads["v0"] - gv).max()) <= 1e-4 * float(np.abs(gv).max())


def test_poisson_stream_of_mixed_requests():
    rng = np.random.default_rng(77)
    srv = _server()
    tickets = []
    try:
        t_next = time.monotonic()
        for i in range(24):
            t_next += rng.exponential(1.0 / 40.0)
            while time.monotonic() < t_next:
                time.sleep(0.001)
            n = int(np.exp(rng.uniform(np.log(1000), np.log(20000))))
            G = int(rng.integers(16, 49))
            T = int(rng.integers(20, 160))
            tickets.append(srv.submit(_request(100 + i, n, G, T, grad=bool(rng.uniform() < 0.3))))
        results = [t.wait(300) for t in tickets]
        stats = dict(srv.stats)
    finally:
        srv.stop(timeout=300)
    assert all(r.status == "ok" for r in results), [r.error for r in results if r.status != "ok"]
    lat = np.array([r.latency_s for r in results])
    print(f"{len(results)} requests: p50 {np.percentile(lat, 50) * 1e3:.1f} ms, p99 {np.percentile(lat, 99) * 1e3:.1f} ms, "
          f"blocks {stats['blocks']}, relayouts {stats['relayouts']}")
    expected = sum(t.req.spec.n * t.req.n_substeps for t in tickets)
    assert stats["particle_substeps"] == expected
    for r, t in zip(results, tickets):
        assert r.x.shape == (t.req.spec.n, 3) and np.isfinite(r.x).all()
        if t.req.grad:
            assert np.isfinite(r.grads["v0"]).all() and np.isfinite(r.loss)


def test_host_injected_faults():
    srv = _server(instances=2)

    def hook(t):
        if t.req.spec.n == 1234:
            raise RuntimeError("injected worker fault")

    srv.fault_hook = hook
    try:
        with pytest.raises(ValueError):
            srv.submit(Request(spec=_request(1, 100, 16, 10).spec, n_substeps=0, dt=1e-4))   # malformed
        huge = srv.submit(_request(2, 130_000, 16, 10))                                    # over capacity
        long1 = srv.submit(_request(3, 2000, 16, 400))
        faulty = srv.submit(_request(4, 1234, 16, 30))
        good = srv.submit(_request(5, 1500, 16, 30))
        late = _request(6, 1000, 16, 30)
        late.deadline_s = 1e-3                                   # waits behind the others: times out
        late_t = srv.submit(late)
        cancelled = srv.submit(_request(7, 1000, 16, 30))
        cancelled.cancel()
        res = {k: t.wait(120) for k, t in (("huge", huge), ("long", long1), ("faulty", faulty), ("good", good),
                                           ("late", late_t), ("cancelled", cancelled))}
    finally:
        srv.stop(timeout=300)
    print({k: (r.status, r.error) for k, r in res.items()})
    assert res["huge"].status == "rejected"
    assert res["faulty"].status == "error" and "injected" in res["faulty"].error
    assert res["long"].status == "ok" and res["good"].status == "ok"
    assert res["late"].status == "timeout"
    assert res["cancelled"].status == "cancelled"
