"""CMA-ES with an ask/tell interface, for evaluating whole populations at once.

The reference trainer drives ``cma.CMAEvolutionStrategy`` (pinned
``cma==4.3.0``, not installed here) through ``es.optimize``, one candidate
evaluation after another (phys_sim/engine/trainer_warp_mpm.py:593-663). This is
an implementation of the published algorithm, (mu/mu_w, lambda)-CMA-ES with
cumulative step-size adaptation and rank-one plus rank-mu covariance updates,
with the default parameters of N. Hansen, "The CMA Evolution Strategy: A
Tutorial" (arXiv:1604.00772, Table 1). ``optimize_batch`` hands a whole
generation to one call, so the batched engine can roll every candidate out in
one launch sequence.

Box bounds: a candidate outside the box is evaluated at its projection onto
the box, and its fitness gets a quadratic penalty on the distance to it.
pycma's default instead evaluates a smooth transform of the point, so the two
are the same algorithm but not the same sample sequence.
"""
from __future__ import annotations

import math
from typing import Callable, Optional, Sequence, Tuple

import numpy as np


class CMAES:
    def __init__(self, x0: Sequence[float], sigma0: float, bounds: Optional[Tuple[float, float]] = None,
                 popsize: Optional[int] = None, seed: Optional[int] = None, penalty: float = 1e3):
        self.n = n = len(x0)
        self.mean = np.asarray(x0, dtype=np.float64).copy()
        self.sigma = float(sigma0)
        self.bounds = bounds
        self.penalty = penalty
        self.rng = np.random.default_rng(seed)
        self.lam = int(popsize) if popsize else 4 + int(3 * math.log(n))
        self.mu = self.lam // 2
        w = math.log(self.lam / 2 + 0.5) - np.log(np.arange(1, self.mu + 1))
        self.weights = w / w.sum()
        self.mueff = 1.0 / float((self.weights ** 2).sum())
        self.cs = (self.mueff + 2) / (n + self.mueff + 5)
        self.ds = 1 + 2 * max(0.0, math.sqrt((self.mueff - 1) / (n + 1)) - 1) + self.cs
        self.cc = (4 + self.mueff / n) / (n + 4 + 2 * self.mueff / n)
        self.c1 = 2 / ((n + 1.3) ** 2 + self.mueff)
        self.cmu = min(1 - self.c1, 2 * (self.mueff - 2 + 1 / self.mueff) / ((n + 2) ** 2 + self.mueff))
        self.chi_n = math.sqrt(n) * (1 - 1 / (4 * n) + 1 / (21 * n * n))
        self.pc = np.zeros(n)
        self.ps = np.zeros(n)
        self.C = np.eye(n)
        self.B = np.eye(n)
        self.D = np.ones(n)
        self.countiter = 0
        self.countevals = 0
        self.best_x: Optional[np.ndarray] = None
        self.best_f = math.inf
        self._asked: Optional[np.ndarray] = None

    # -- sampling ------------------------------------------------------------------
    def ask(self) -> np.ndarray:
        """The next generation, [popsize, n] (unconstrained points)."""
        z = self.rng.standard_normal((self.lam, self.n))
        y = z @ (self.B * self.D).T
        self._asked = self.mean + self.sigma * y
        return self._asked.copy()

    def feasible(self, X: np.ndarray) -> np.ndarray:
        """Points at which the candidates are evaluated (projected into the box)."""
        if self.bounds is None:
            return np.asarray(X, dtype=np.float64)
        return np.clip(X, self.bounds[0], self.bounds[1])

    def penalised(self, X: np.ndarray, f: Sequence[float]) -> np.ndarray:
        f = np.asarray(f, dtype=np.float64)
        if self.bounds is None:
            return f
        return f + self.penalty * ((X - self.feasible(X)) ** 2).sum(axis=1)

    # -- update --------------------------------------------------------------------
    def tell(self, X: np.ndarray, f: Sequence[float]) -> None:
        """Update from the candidates X (as returned by ask) and their raw
        fitness at feasible(X) (lower is better)."""
        X = np.asarray(X, dtype=np.float64)
        raw = np.asarray(f, dtype=np.float64)
        fit = self.penalised(X, raw)
        self.countevals += len(raw)
        k = int(np.argmin(raw))
        if raw[k] < self.best_f:
            self.best_f = float(raw[k])
            self.best_x = self.feasible(X[k:k + 1])[0].copy()
        order = np.argsort(fit)[: self.mu]
        Y = (X[order] - self.mean) / self.sigma
        yw = self.weights @ Y
        self.mean = self.mean + self.sigma * yw
        inv_sqrt_C = self.B @ np.diag(1.0 / self.D) @ self.B.T
        self.ps = (1 - self.cs) * self.ps + math.sqrt(self.cs * (2 - self.cs) * self.mueff) * (inv_sqrt_C @ yw)
        self.countiter += 1
        norm_ps = float(np.linalg.norm(self.ps))
        hsig = norm_ps / math.sqrt(1 - (1 - self.cs) ** (2 * self.countiter)) < (1.4 + 2 / (self.n + 1)) * self.chi_n
        self.pc = (1 - self.cc) * self.pc + (math.sqrt(self.cc * (2 - self.cc) * self.mueff) * yw if hsig else 0.0)
        rank_mu = (Y.T * self.weights) @ Y
        delta = (1 - hsig) * self.cc * (2 - self.cc)
        self.C = ((1 - self.c1 - self.cmu) * self.C + self.c1 * (np.outer(self.pc, self.pc) + delta * self.C) +
                  self.cmu * rank_mu)
        self.sigma *= math.exp((self.cs / self.ds) * (norm_ps / self.chi_n - 1))
        self.C = (self.C + self.C.T) / 2
        d2, self.B = np.linalg.eigh(self.C)
        self.D = np.sqrt(np.maximum(d2, 1e-20))

    # -- drivers -----------------------------------------------------------------------
    def optimize(self, func: Callable[[np.ndarray], float], iterations: int,
                 callback: Optional[Callable[["CMAES"], None]] = None) -> "CMAES":
        """One evaluation per candidate, as cma's es.optimize does."""
        return self.optimize_batch(lambda P: [func(p) for p in P], iterations, callback)

    def optimize_batch(self, func_batch: Callable[[np.ndarray], Sequence[float]], iterations: int,
                       callback: Optional[Callable[["CMAES"], None]] = None) -> "CMAES":
        """func_batch receives the feasible points of a whole generation,
        [popsize, n], and returns their fitness."""
        for _ in range(iterations):
            X = self.ask()
            f = func_batch(self.feasible(X))
            self.tell(X, f)
            if callback is not None:
                callback(self)
        return self

    @property
    def result(self) -> Tuple[Optional[np.ndarray], float, int, int]:
        """(best x, best fitness, evaluations, iterations)."""
        return self.best_x, self.best_f, self.countevals, self.countiter
