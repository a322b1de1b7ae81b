"""Device training losses and the batched CMA-ES driver.

Chamfer distance against an FP64 brute force (relative 1e-5, FP32 sums of
squared distances); its gradient against the analytic gradient at the FP64
nearest neighbours (relative 1e-5) and against central differences; the
driver's per-candidate loss the same in a generation as alone (1e-5 relative,
reduction order only); and CMA-ES on the batched engine recovering the
material of a synthetic trajectory."""
import numpy as np
import pytest
import torch

from empm_b200.batch import BatchedMPM, InstanceSpec
from empm_b200.cma_driver import PopulationEvaluator, denormalize, train_cma
from empm_b200.losses import chamfer_distance, chamfer_pairs, tracking_loss

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _ref_chamfer(x, y):
    d = ((x[:, None, :] - y[None, :, :]) ** 2).sum(-1)
    return d.min(1).mean() + d.min(0).mean(), d.argmin(1), d.argmin(0)


def _pairs(rng, sizes):
    xs = [rng.uniform(0, 1, (a, 3)) for a, _ in sizes]
    ys = [rng.uniform(0, 1, (b, 3)) for _, b in sizes]
    return xs, ys


def test_chamfer_pairs_matches_brute_force():
    rng = np.random.default_rng(0)
    sizes = [(1, 1), (300, 1000), (1000, 300), (2000, 2000), (517, 33), (33, 517)]
    xs, ys = _pairs(rng, sizes)
    t = lambda a: torch.as_tensor(np.concatenate(a), dtype=torch.float32, device=DEV)  # noqa: E731
    got = chamfer_pairs(t(xs), [a for a, _ in sizes], t(ys), [b for _, b in sizes]).double().cpu().numpy()
    for (x, y), g in zip(zip(xs, ys), got):
        ref = _ref_chamfer(x.astype(np.float32).astype(np.float64), y.astype(np.float32).astype(np.float64))[0]
        assert abs(g - ref) <= 1e-5 * ref, (g, ref)
    loss, none = chamfer_distance(t(xs[3]).reshape(1, 2000, 3), t(ys[3]).reshape(1, 2000, 3))
    assert none is None and abs(float(loss) - got[3]) <= 1e-6 * got[3]


def test_chamfer_gradient():
    rng = np.random.default_rng(1)
    sizes = [(400, 700), (900, 250), (64, 64)]
    xs, ys = _pairs(rng, sizes)
    w = rng.uniform(0.5, 2.0, len(sizes))
    x = torch.as_tensor(np.concatenate(xs), dtype=torch.float32, device=DEV).requires_grad_(True)
    y = torch.as_tensor(np.concatenate(ys), dtype=torch.float32, device=DEV)
    per = chamfer_pairs(x, [a for a, _ in sizes], y, [b for _, b in sizes])
    (per * torch.as_tensor(w, dtype=torch.float32, device=DEV)).sum().backward()
    g = x.grad.double().cpu().numpy()
    # analytic gradient at the FP64 nearest neighbours
    ref, o = [], 0
    for (xa, ya), wp in zip(zip(xs, ys), w):
        xa = xa.astype(np.float32).astype(np.float64)
        ya = ya.astype(np.float32).astype(np.float64)
        _, nx, ny = _ref_chamfer(xa, ya)
        gx = 2 * wp * (xa - ya[nx]) / len(xa)
        np.add.at(gx, ny, 2 * wp * (xa[ny] - ya) / len(ya))
        ref.append(gx)
    ref = np.concatenate(ref)
    assert np.abs(g - ref).max() <= 1e-5 * np.abs(ref).max()
    # central differences of the FP64 loss on a few coordinates
    for k in (3, 500, 1100):
        for c in range(3):
            h = 1e-6
            vals = []
            for s in (h, -h):
                xs2 = [a.astype(np.float32).astype(np.float64).copy() for a in xs]
                i, row = k, 0
                while i >= len(xs2[row]):
                    i -= len(xs2[row])
                    row += 1
                xs2[row][i, c] += s
                vals.append(sum(wp * _ref_chamfer(a, b.astype(np.float32).astype(np.float64))[0]
                                for a, b, wp in zip(xs2, ys, w)))
            fd = (vals[0] - vals[1]) / (2 * h)
            assert abs(fd - g[k, c]) <= 1e-4 * np.abs(ref).max()


def _body(n=2500, G=32, seed=3):
    rng = np.random.default_rng(seed)
    x = np.stack([0.35 + 0.25 * rng.uniform(size=n), 0.1 + 0.2 * rng.uniform(size=n),
                  0.35 + 0.25 * rng.uniform(size=n)], 1).astype(np.float32)
    v = np.zeros((n, 3), np.float32)
    v[:, 1] = -1.0
    return InstanceSpec(x=x, v=v, vol=np.full(n, np.float32(0.25 * 0.2 * 0.25 / n), np.float32),
                        rho=np.full(n, np.float32(1e3), np.float32), E=np.full(n, np.float32(2e4), np.float32),
                        nu=np.full(n, np.float32(0.3), np.float32), n_grid=G, material="jelly",
                        colliders=[dict(kind="surface", point=[0.0, 3.0 / G, 0.0], normal=[0.0, 1.0, 0.0]),
                                   dict(kind="bbox")])


def _target(base, params, dt, spf, frames):
    phys = denormalize(params)
    b = BatchedMPM([base], device=DEV)
    b.set_material(0, E=phys["E"], nu=phys["nu"])
    b.prepare()
    out = [b.positions().clone()]
    for _ in range(frames):
        b.rollout(dt, spf, block=spf)
        out.append(b.positions().clone())
    return torch.stack(out)


def test_generation_loss_equals_candidate_alone():
    base = _body()
    tgt = _target(base, {"E": 0.02, "nu": 0.3}, 2e-4, 20, 5)
    ev = PopulationEvaluator(base, tgt, 2e-4, 20)
    P = np.array([[0.01, 0.25], [0.02, 0.3], [0.05, 0.35], [0.08, 0.2]])
    together = ev(P)
    alone = np.array([PopulationEvaluator(base, tgt, 2e-4, 20)(P[i:i + 1])[0] for i in range(len(P))])
    print("generation:", together, "alone:", alone)
    assert np.allclose(together, alone, rtol=1e-5, atol=1e-6)
    assert together[1] < together[0] and together[1] < together[2]      # the true parameters score best
    # the tracking term alone, through the public helper
    assert float(tracking_loss(tgt[1], tgt[1])) == 0.0


def test_cma_recovers_material_on_the_batched_engine():
    base = _body()
    truth = {"E": 0.02, "nu": 0.3}
    tgt = _target(base, truth, 2e-4, 20, 5)
    ev = PopulationEvaluator(base, tgt, 2e-4, 20)
    first = ev(np.array([[0.06, 0.2]]))[0]
    es = train_cma(ev, [0.06, 0.2], sigma0=1 / 6, iterations=12, popsize=12, seed=42)
    best_x, best_f, n_eval, n_iter = es.result
    print(f"start loss {first:.4f}; best {best_f:.5f} at E={best_x[0]:.4f} nu={best_x[1]:.4f} after {n_eval} evals")
    assert n_iter == 12 and ev.evaluations == 1 + 12 * 12
    assert best_f < 0.1 * first
    assert abs(best_x[0] - truth["E"]) < 0.25 * abs(0.06 - truth["E"])
