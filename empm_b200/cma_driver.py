"""CMA-ES over material parameters, one batched rollout per generation.

The reference trainer (phys_sim/engine/trainer_warp_mpm.py:566-663) optimises
the normalised parameters ["E", "nu"] in [0, 1] with CMA-ES (sigma 1/6,
seed 42). Each candidate costs a full re-initialisation and a serial
``advance_to``. Its loss (``loss_func``, :617-642) is

    1e3 * sum over frames t < n_frames of ( chamfer(pred_t[vis_t], target_t[vis_t])
                                           + ||pred_t[valid_t] - target_t[valid_t]|| / n_valid_t )

with E denormalised as value * 1e6 (``denormalize_param``, :314-330).

``PopulationEvaluator`` evaluates a whole generation at once: every candidate
is one instance of a ``BatchedMPM`` built from the same base body, all of
them advance together frame by frame, and the chamfer terms of every
(candidate, frame) pair come from one ``chamfer_pairs`` launch.
"""
from __future__ import annotations

from dataclasses import replace
from typing import Callable, Dict, Optional, Sequence

import numpy as np
import torch
from torch import Tensor

from .batch import BatchedMPM, InstanceSpec
from .cmaes import CMAES
from .losses import chamfer_pairs

SCALES = {"E": 1e6}       # denormalisation of the reference trainer; other keys are used as given


def denormalize(params: Dict[str, float]) -> Dict[str, float]:
    return {k: float(v) * SCALES.get(k, 1.0) for k, v in params.items()}


class PopulationEvaluator:
    """Loss of every candidate of a generation, from one batched rollout.

    base: the body (initial state, material kind, colliders); target: [F+1, N, 3]
    observed positions per frame (frame 0 is the initial state); visible /
    valid: optional [F+1, N] masks of the chamfer and tracking terms."""

    def __init__(self, base: InstanceSpec, target: Tensor, dt: float, substeps_per_frame: int,
                 param_keys: Sequence[str] = ("E", "nu"), visible: Optional[Tensor] = None,
                 valid: Optional[Tensor] = None, device="cuda:0", block: int = 50):
        self.base = base
        self.device = torch.device(device)
        self.target = target.to(self.device, torch.float32)
        self.n_frames = self.target.shape[0] - 1
        self.dt = float(dt)
        self.spf = int(substeps_per_frame)
        self.keys = list(param_keys)
        self.visible = None if visible is None else visible.to(self.device).bool()
        self.valid = None if valid is None else valid.to(self.device).bool()
        self.block = block
        self.batch: Optional[BatchedMPM] = None
        self.evaluations = 0

    def _batch(self, lam: int) -> BatchedMPM:
        if self.batch is None or self.batch.n_inst != lam:
            self.batch = BatchedMPM([replace(self.base) for _ in range(lam)], device=self.device)
        return self.batch

    def rollout(self, P: np.ndarray) -> Tensor:
        """Positions of every candidate per frame, [F+1, lambda, N, 3]."""
        lam, n = P.shape[0], self.base.n
        b = self._batch(lam)
        b.cur, b.time = 0, 0.0
        b.load_state()
        for i, p in enumerate(np.asarray(P, dtype=np.float64)):
            phys = denormalize(dict(zip(self.keys, p)))
            b.set_material(i, E=phys.get("E"), nu=phys.get("nu"), yield_stress=phys.get("ys"))
        b.prepare()
        frames = [b.positions().reshape(lam, n, 3).clone()]
        for _ in range(self.n_frames):
            b.rollout(self.dt, self.spf, block=min(self.spf, self.block))
            frames.append(b.positions().reshape(lam, n, 3).clone())
        self.evaluations += lam
        return torch.stack(frames)

    def losses(self, frames: Tensor) -> Tensor:
        """The trainer's loss per candidate from [F+1, lambda, N, 3] positions."""
        F, lam = self.n_frames, frames.shape[1]
        pred = frames[:F]                                        # frames t < n_frames
        tgt = self.target[:F]
        xs, ys, xc, yc = [], [], [], []
        for t in range(F):
            m = None if self.visible is None else self.visible[t]
            yt = tgt[t] if m is None else tgt[t][m]
            for i in range(lam):
                xt = pred[t, i] if m is None else pred[t, i][m]
                xs.append(xt)
                ys.append(yt)
                xc.append(xt.shape[0])
                yc.append(yt.shape[0])
        cham = chamfer_pairs(torch.cat(xs), xc, torch.cat(ys), yc).reshape(F, lam)
        if self.valid is None:
            diff = pred - tgt[:, None]
            n_valid = torch.full((F, 1), float(frames.shape[2]), device=self.device)
        else:
            v = self.valid[:F, None, :, None].to(pred.dtype)
            diff = (pred - tgt[:, None]) * v
            n_valid = self.valid[:F].sum(1, keepdim=True).clamp(min=1).to(pred.dtype)
        track = diff.pow(2).sum(dim=(2, 3)).sqrt() / n_valid
        return 1e3 * (cham + track).sum(0)

    def __call__(self, P: np.ndarray) -> np.ndarray:
        with torch.no_grad():
            return self.losses(self.rollout(P)).double().cpu().numpy()


def train_cma(evaluator: Callable[[np.ndarray], np.ndarray], x0: Sequence[float], sigma0: float = 1 / 6,
              iterations: int = 20, bounds=(0.0, 1.0), seed: int = 42, popsize: Optional[int] = None,
              callback=None) -> CMAES:
    """The trainer's train_cma with whole-generation evaluation."""
    es = CMAES(x0, sigma0, bounds=bounds, popsize=popsize, seed=seed)
    return es.optimize_batch(evaluator, iterations, callback)
