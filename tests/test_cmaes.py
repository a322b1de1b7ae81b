"""CMA-ES (no GPU): convergence on standard test functions, box bounds,
determinism under a seed, and per-candidate vs whole-generation evaluation."""
import numpy as np

from empm_b200.cmaes import CMAES


def test_sphere_unbounded():
    es = CMAES(3.0 * np.ones(5), 1.0, seed=1)
    es.optimize_batch(lambda P: (P ** 2).sum(axis=1), 200)
    assert es.best_f < 1e-10
    assert np.abs(es.best_x).max() < 1e-4


def test_rosenbrock_2d():
    f = lambda P: (1 - P[:, 0]) ** 2 + 100 * (P[:, 1] - P[:, 0] ** 2) ** 2  # noqa: E731
    es = CMAES([-1.0, 1.5], 0.5, seed=3)
    es.optimize_batch(f, 300)
    assert es.best_f < 1e-8
    assert np.allclose(es.best_x, [1.0, 1.0], atol=1e-3)


def test_box_bounds_like_the_trainer():
    # the trainer's setting: 2 normalised parameters in [0, 1], sigma 1/6, seed 42
    target = np.array([0.3, 0.8])
    es = CMAES([0.5, 0.5], 1 / 6, bounds=(0.0, 1.0), seed=42)
    seen = []
    es.optimize_batch(lambda P: (seen.append(P.copy()) or ((P - target) ** 2).sum(axis=1)), 60)
    assert all(((P >= 0) & (P <= 1)).all() for P in seen)      # only feasible points are evaluated
    assert np.allclose(es.best_x, target, atol=1e-3)


def test_optimum_on_the_boundary():
    es = CMAES([0.5, 0.5], 1 / 6, bounds=(0.0, 1.0), seed=7)
    es.optimize_batch(lambda P: ((P - np.array([1.3, 0.5])) ** 2).sum(axis=1), 80)
    assert abs(es.best_x[0] - 1.0) < 1e-3 and abs(es.best_x[1] - 0.5) < 1e-3


def test_seeded_runs_are_identical_and_batch_equals_per_candidate():
    f = lambda p: float(((p - 0.25) ** 2).sum())  # noqa: E731
    a = CMAES([0.6, 0.6, 0.6], 0.2, bounds=(0.0, 1.0), seed=42).optimize(f, 25)
    b = CMAES([0.6, 0.6, 0.6], 0.2, bounds=(0.0, 1.0), seed=42).optimize_batch(
        lambda P: [f(p) for p in P], 25)
    assert a.best_f == b.best_f and np.array_equal(a.best_x, b.best_x)
    assert np.array_equal(a.mean, b.mean) and a.sigma == b.sigma
    assert a.result[2] == 25 * a.lam and a.result[3] == 25
