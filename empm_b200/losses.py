"""Training losses of the reference trainer, on the device.

* ``chamfer_distance`` mirrors pytorch3d's (point_reduction "mean",
  batch_reduction "mean"), which the trainer calls per frame
  (phys_sim/engine/trainer_warp_mpm.py:542-561, 617-642, 745-765).
* ``chamfer_pairs`` scores many (prediction, target) pairs, e.g. every
  population member and frame of a CMA-ES generation, in one launch
  (``empm_chamfer``). It is differentiable in the predictions
  (``empm_chamfer_backward``); the targets are data.
* ``tracking_loss`` is the trainer's tracking term: ||pred - target|| / n over
  the valid points (trainer_warp_mpm.py:551-561).
"""
from __future__ import annotations

from typing import Optional, Sequence, Tuple

import numpy as np
import torch
from torch import Tensor

from . import _native as N
from .mpm_data_structure import _stream_ptr


def _offsets(counts: Sequence[int], device) -> Tuple[Tensor, int]:
    off = np.concatenate([[0], np.cumsum(np.asarray(counts, dtype=np.int64))]).astype(np.int32)
    return torch.as_tensor(off, device=device), int(max(counts) if len(counts) else 0)


class _ChamferPairs(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x: Tensor, y: Tensor, x_counts, y_counts):
        dev = x.device
        x = x.detach().float().contiguous()
        y = y.detach().float().contiguous().to(dev)
        n_pairs = len(x_counts)
        x_off, max_nx = _offsets(x_counts, dev)
        y_off, max_ny = _offsets(y_counts, dev)
        s_xy = torch.empty(n_pairs, dtype=torch.float32, device=dev)
        s_yx = torch.empty_like(s_xy)
        nn_x = torch.empty(x.shape[0], dtype=torch.int32, device=dev)
        nn_y = torch.empty(y.shape[0], dtype=torch.int32, device=dev)
        N.check(N.lib().empm_chamfer(x.data_ptr(), x_off.data_ptr(), x.shape[0], max_nx, y.data_ptr(),
                                     y_off.data_ptr(), y.shape[0], max_ny, n_pairs, s_xy.data_ptr(), s_yx.data_ptr(),
                                     nn_x.data_ptr(), nn_y.data_ptr(), _stream_ptr(dev)))
        nx = torch.as_tensor(np.maximum(np.asarray(x_counts), 1), dtype=torch.float32, device=dev)
        ny = torch.as_tensor(np.maximum(np.asarray(y_counts), 1), dtype=torch.float32, device=dev)
        ctx.save_for_backward(x, y, x_off, y_off, nn_x, nn_y, nx, ny)
        return s_xy / nx + s_yx / ny

    @staticmethod
    def backward(ctx, g: Tensor):
        x, y, x_off, y_off, nn_x, nn_y, nx, ny = ctx.saved_tensors
        dev = x.device
        g = g.float().contiguous()
        g_xy = (g / nx).contiguous()
        g_yx = (g / ny).contiguous()
        grad = torch.zeros_like(x)
        scratch = torch.empty(max(x.shape[0], y.shape[0], 1), dtype=torch.int32, device=dev)
        N.check(N.lib().empm_chamfer_backward(x.data_ptr(), x_off.data_ptr(), x.shape[0], y.data_ptr(),
                                              y_off.data_ptr(), y.shape[0], g.shape[0], nn_x.data_ptr(),
                                              nn_y.data_ptr(), g_xy.data_ptr(), g_yx.data_ptr(), grad.data_ptr(),
                                              scratch.data_ptr(), _stream_ptr(dev)))
        return grad, None, None, None


def chamfer_pairs(x: Tensor, x_counts: Sequence[int], y: Tensor, y_counts: Sequence[int]) -> Tensor:
    """Chamfer distance of each (x, y) pair: x rows grouped by x_counts, y rows
    by y_counts (same number of pairs). Returns [n_pairs]."""
    if len(x_counts) != len(y_counts) or len(x_counts) == 0:
        raise ValueError("x_counts and y_counts must list the same, non-zero number of pairs")
    if x.shape != (int(sum(x_counts)), 3) or y.shape != (int(sum(y_counts)), 3):
        raise ValueError("x and y must be [sum(counts), 3]")
    if x.device.type != "cuda":
        raise ValueError("chamfer_pairs runs on CUDA tensors")
    return _ChamferPairs.apply(x, y, list(map(int, x_counts)), list(map(int, y_counts)))


def chamfer_distance(x: Tensor, y: Tensor) -> Tuple[Tensor, None]:
    """pytorch3d.loss.chamfer_distance(x, y) for [B, N, 3] / [B, M, 3] (or
    [N, 3] / [M, 3]) point clouds: mean over the batch of (mean_x min_y |x-y|^2
    + mean_y min_x |x-y|^2). Returns (loss, None) as pytorch3d does without normals."""
    if x.dim() == 2:
        x, y = x.unsqueeze(0), y.unsqueeze(0)
    B, n, m = x.shape[0], x.shape[1], y.shape[1]
    per = chamfer_pairs(x.reshape(B * n, 3), [n] * B, y.reshape(B * m, 3), [m] * B)
    return per.mean(), None


def tracking_loss(pred: Tensor, target: Tensor, valid: Optional[Tensor] = None) -> Tensor:
    """||pred - target|| / n over the valid points (the trainer's tracking term)."""
    if valid is not None:
        pred, target = pred[valid], target[valid]
    n = max(int(pred.shape[0]), 1)
    return (pred - target).norm() / n
