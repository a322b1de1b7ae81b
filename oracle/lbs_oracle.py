"""CPU oracle for the Gaussian motion interpolation — TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py``
may import this module; it is the checker, never the product path.

A NumPy (FP64) restatement of third_party/gaussian_splatting/dynamic_utils.py:
  * ``knn``               get_topk_indices (:248-265), knn_weights_sparse (:295-302)
  * ``idw_weights``       calc_weights_vals_from_indices (:282-292)
  * ``bone_rotations``    the bone fit of interpolate_motions(_speedup)
                          (:315-409), including how the reference assigns
                          rank-deficient batches to all bones
  * ``quat_mat2quat``     mat2quat (:25-64)
  * ``quat_kornia``       kornia 0.8.1 rotation_matrix_to_quaternion, the
                          conversion the sparse path imports (:465-475); kornia
                          is not installed here, so this is the published
                          algorithm restated (trace > 0 picks w as pivot, else
                          the largest diagonal entry; eps 1e-8 under the root,
                          divisors clamped at the smallest normal float)
  * ``blend_sparse``      the Gaussian stage of interpolate_motions_speedup (:428-483)
  * ``blend_dense``       the Gaussian stage of interpolate_motions (:165-216)

Parity: pinned against tests/golden/lbs.npz, produced by running the
reference's own dynamic_utils functions (torch, CPU) on seeded inputs
(tests/golden/make_golden.py, job ``lbs``). kornia is stubbed there so the
sparse path takes its mat2quat fallback; the kornia restatement is checked
against mat2quat where both use the w pivot (rotations below 120 degrees).
The sign of a rank-1 bone's axis (U[:, 0] of the SVD) depends on the SVD
implementation, so ``bone_rotations`` returns both candidates for those bones.
"""
from __future__ import annotations

from typing import Optional, Tuple

import numpy as np

EPS_F32 = float(np.finfo(np.float32).eps)
TINY_F32 = float(np.finfo(np.float32).tiny)


def knn(queries: np.ndarray, points: np.ndarray, k: int, exclude_self: bool = False,
        chunk: int = 2048) -> Tuple[np.ndarray, np.ndarray]:
    """Indices [n, k] (nearest first; ties by index) and distances of the k
    nearest points of every query."""
    q = np.asarray(queries, np.float64)
    p = np.asarray(points, np.float64)
    idx = np.empty((q.shape[0], k), np.int64)
    dist = np.empty((q.shape[0], k), np.float64)
    for s in range(0, q.shape[0], chunk):
        qq = q[s:s + chunk]
        d2 = ((qq[:, None, :] - p[None, :, :]) ** 2).sum(-1)
        if exclude_self:
            d2[np.arange(qq.shape[0]), np.arange(s, s + qq.shape[0])] = np.inf
        order = np.argsort(d2, axis=1, kind="stable")[:, :k]
        idx[s:s + chunk] = order
        dist[s:s + chunk] = np.sqrt(np.take_along_axis(d2, order, 1))
    return idx, dist


def idw_weights(bones: np.ndarray, pts: np.ndarray, idx: np.ndarray) -> np.ndarray:
    """w = 1 / (|x - b| + 1e-6), normalised over each row (:282-292)."""
    d = np.linalg.norm(np.asarray(pts, np.float64)[:, None] - np.asarray(bones, np.float64)[idx], axis=2)
    v = 1.0 / (d + 1e-6)
    return v / v.sum(1, keepdims=True)


def _rank1_rotation(axis: np.ndarray) -> np.ndarray:
    """Rotation taking e_x onto axis about axis x e_x (:369-393)."""
    x = np.array([1.0, 0.0, 0.0])
    perp = np.cross(axis, x)
    n = np.linalg.norm(perp)
    if n < 1e-6:
        return np.eye(3)
    perp = perp / n
    third = np.cross(x, perp)
    third_after = np.cross(axis, perp)
    X = np.stack([x, perp, third], axis=-1)
    Y = np.stack([axis, perp, third_after], axis=-1)
    return Y @ X.T


def bone_fit(bones: np.ndarray, motions: np.ndarray, relations: np.ndarray):
    """Per bone: F (:323-329), rank as torch.linalg.matrix_rank counts it
    (singular values above 3 eps_f32 s_max), the proper rotation closest to F
    (:340-360) and, for rank 1, the two candidate rank-1 rotations (axis sign)
    and whether the small singular values pass allclose(., 0) (atol 1e-8);
    the rank-1 candidates of other bones are left at I."""
    b = np.asarray(bones, np.float64)
    m = np.asarray(motions, np.float64)
    old = b[relations] - b[:, None]
    new = (b[relations] + m[relations]) - (b[:, None] + m[:, None])
    F = np.einsum("nja,njb->nab", new, old)
    U, S, Vt = np.linalg.svd(F)
    tol = 3 * EPS_F32 * S[:, :1]
    rank = (S > tol).sum(1)
    d = np.sign(np.linalg.det(U) * np.linalg.det(Vt))
    d[d == 0] = 1.0
    D = np.zeros((len(b), 3, 3))
    D[:, 0, 0] = 1
    D[:, 1, 1] = 1
    D[:, 2, 2] = d
    R_kabsch = U @ D @ Vt
    r1_pos = np.broadcast_to(np.eye(3), R_kabsch.shape).copy()
    r1_neg = r1_pos.copy()
    for i in np.nonzero(rank == 1)[0]:
        r1_pos[i] = _rank1_rotation(U[i, :, 0])
        r1_neg[i] = _rank1_rotation(-U[i, :, 0])
    close = np.all(np.abs(S[:, 1:]) <= 1e-8, axis=1)
    return dict(F=F, S=S, rank=rank, R_kabsch=R_kabsch, R_rank1=(r1_pos, r1_neg), close=close)


def bone_rotations(bones: np.ndarray, motions: np.ndarray, relations: np.ndarray) -> Tuple[np.ndarray, str]:
    """Final rotation per bone [n, 2, 3, 3] (two candidates that differ only
    for rank-1 bones, by the axis sign) and the case taken (:337-407)."""
    fit = bone_fit(bones, motions, relations)
    n = len(bones)
    rank = fit["rank"]
    n1 = int((rank == 1).sum())
    n23 = int((rank >= 2).sum())
    eye = np.broadcast_to(np.eye(3), (n, 2, 3, 3)).copy()
    if n1 > 0:
        if not fit["close"][rank == 1].all():
            return eye, "rank1-not-close"
        r1 = np.stack(fit["R_rank1"], axis=1)   # [n, 2, 3, 3]
        if n1 == n:
            return r1, "rank1-all"
        if n1 == 1:
            j = int(np.nonzero(rank == 1)[0][0])
            return np.broadcast_to(r1[j], (n, 2, 3, 3)).copy(), "rank1-broadcast"
        return eye, "rank1-mismatch"
    rk = np.stack([fit["R_kabsch"], fit["R_kabsch"]], axis=1)
    if n23 == n:
        return rk, "kabsch"
    if n23 == 1:
        j = int(np.nonzero(rank >= 2)[0][0])
        return np.broadcast_to(rk[j], (n, 2, 3, 3)).copy(), "kabsch-broadcast"
    return eye, "mismatch"


def quat_mat2quat(R: np.ndarray) -> np.ndarray:
    """mat2quat (:25-64), branches as written, (w, x, y, z). Evaluated in the
    input's precision: near 180 degrees the float32 trace rounds to -1 and the
    reference then takes another branch."""
    R = np.asarray(R)
    if R.dtype != np.float32:
        R = R.astype(np.float64)
    q = np.zeros((R.shape[0], 4), R.dtype)
    t = np.maximum(R[:, 0, 0] + R[:, 1, 1] + R[:, 2, 2], R.dtype.type(-1.0))
    m0 = t > -1
    s = np.sqrt(t[m0] + 1)
    q[m0, 0] = 0.5 * s
    f = 0.5 / s
    q[m0, 1] = (R[m0, 2, 1] - R[m0, 1, 2]) * f
    q[m0, 2] = (R[m0, 0, 2] - R[m0, 2, 0]) * f
    q[m0, 3] = (R[m0, 1, 0] - R[m0, 0, 1]) * f
    m1 = ~m0 & (R[:, 0, 0] >= R[:, 1, 1]) & (R[:, 0, 0] >= R[:, 2, 2])
    f = 0.5 / np.sqrt(1 + R[m1, 0, 0] - R[m1, 1, 1] - R[m1, 2, 2])
    q[m1] = np.stack([(R[m1, 2, 1] - R[m1, 1, 2]) * f, 0.5 * f, (R[m1, 1, 0] + R[m1, 0, 1]) * f,
                      (R[m1, 2, 0] + R[m1, 0, 2]) * f], -1)
    m2 = ~m0 & (R[:, 1, 1] >= R[:, 2, 2]) & (R[:, 1, 1] > R[:, 0, 0])
    f = 0.5 / np.sqrt(1 + R[m2, 1, 1] - R[m2, 0, 0] - R[m2, 2, 2])
    q[m2] = np.stack([(R[m2, 0, 2] - R[m2, 2, 0]) * f, (R[m2, 2, 1] + R[m2, 1, 2]) * f, 0.5 * f,
                      (R[m2, 0, 1] + R[m2, 1, 0]) * f], -1)
    m3 = ~m0 & (R[:, 2, 2] > R[:, 0, 0]) & (R[:, 2, 2] > R[:, 1, 1])
    f = 0.5 / np.sqrt(1 + R[m3, 2, 2] - R[m3, 0, 0] - R[m3, 1, 1])
    q[m3] = np.stack([(R[m3, 1, 0] - R[m3, 0, 1]) * f, (R[m3, 0, 2] + R[m3, 2, 0]) * f,
                      (R[m3, 1, 2] + R[m3, 2, 1]) * f, 0.5 * f], -1)
    return q


def quat_kornia(R: np.ndarray, eps: float = 1e-8) -> np.ndarray:
    """kornia 0.8.1 rotation_matrix_to_quaternion, (w, x, y, z), in the
    input's precision (float32 or float64)."""
    R = np.asarray(R)
    if R.dtype != np.float32:
        R = R.astype(np.float64)
    one = R.dtype.type(1.0)
    eps = R.dtype.type(eps)
    m = R.reshape(-1, 9).T
    m00, m01, m02, m10, m11, m12, m20, m21, m22 = m
    trace = m00 + m11 + m22

    def sdiv(a, b):
        return a / np.maximum(b, R.dtype.type(TINY_F32))

    two, quarter, zero = 2 * one, one / 4, 0 * one
    sq0 = np.sqrt(np.maximum(trace + one + eps, zero)) * two
    q0 = np.stack([quarter * sq0, sdiv(m21 - m12, sq0), sdiv(m02 - m20, sq0), sdiv(m10 - m01, sq0)], -1)
    sq1 = np.sqrt(np.maximum(one + m00 - m11 - m22 + eps, zero)) * two
    q1 = np.stack([sdiv(m21 - m12, sq1), quarter * sq1, sdiv(m01 + m10, sq1), sdiv(m02 + m20, sq1)], -1)
    sq2 = np.sqrt(np.maximum(one + m11 - m00 - m22 + eps, zero)) * two
    q2 = np.stack([sdiv(m02 - m20, sq2), sdiv(m01 + m10, sq2), quarter * sq2, sdiv(m12 + m21, sq2)], -1)
    sq3 = np.sqrt(np.maximum(one + m22 - m00 - m11 + eps, zero)) * two
    q3 = np.stack([sdiv(m10 - m01, sq3), sdiv(m02 + m20, sq3), sdiv(m12 + m21, sq3), quarter * sq3], -1)
    w2 = np.where((m11 > m22)[:, None], q2, q3)
    w1 = np.where(((m00 > m11) & (m00 > m22))[:, None], q1, w2)
    return np.where((trace > 0)[:, None], q0, w1)


def normalize(q: np.ndarray) -> np.ndarray:
    return q / np.maximum(np.linalg.norm(q, axis=-1, keepdims=True), 1e-12)


def quat_multiply(q1: np.ndarray, q2: np.ndarray) -> np.ndarray:
    """quaternion_multiply (:449-457), (w, x, y, z)."""
    a0, a1, a2, a3 = np.moveaxis(q1, -1, 0)
    b0, b1, b2, b3 = np.moveaxis(q2, -1, 0)
    return np.stack([a0 * b0 - a1 * b1 - a2 * b2 - a3 * b3,
                     a0 * b1 + a1 * b0 + a2 * b3 - a3 * b2,
                     a0 * b2 - a1 * b3 + a2 * b0 + a3 * b1,
                     a0 * b3 + a1 * b2 - a2 * b1 + a3 * b0], -1)


def blend_sparse(bones, motions, R, xyz, idx, weights, quat=None, convention="kornia"):
    """Gaussian stage of interpolate_motions_speedup for bone rotations R [n_bones, 3, 3]."""
    b = np.asarray(bones, np.float64)
    m = np.asarray(motions, np.float64)
    x = np.asarray(xyz, np.float64)
    w = np.asarray(weights, np.float64)
    loc = x[:, None] - b[idx]
    rl = np.einsum("nkij,nkj->nki", R[idx], loc)
    out = ((rl + m[idx] + b[idx]) * w[:, :, None]).sum(1)
    rot = None
    if quat is not None:
        qb = normalize((quat_kornia if convention == "kornia" else quat_mat2quat)(R))
        qs = normalize((qb[idx] * w[:, :, None]).sum(1))
        rot = quat_multiply(qs, np.asarray(quat, np.float64))
    return out, rot


def dense_weights(bones, xyz) -> np.ndarray:
    """Default weights of interpolate_motions: 1 / max(d, 1e-4) to every bone, normalised (:168-178)."""
    d = np.linalg.norm(np.asarray(xyz, np.float64)[:, None] - np.asarray(bones, np.float64)[None], axis=2)
    v = 1.0 / np.maximum(d, 1e-4)
    return v / v.sum(1, keepdims=True)


def blend_dense(bones, motions, R, xyz, weights: Optional[np.ndarray] = None, quat=None):
    """Gaussian stage of interpolate_motions (mat2quat quaternions)."""
    b = np.asarray(bones, np.float64)
    m = np.asarray(motions, np.float64)
    x = np.asarray(xyz, np.float64)
    w = dense_weights(b, x) if weights is None else np.asarray(weights, np.float64)
    loc = x[:, None] - b[None]
    rl = np.einsum("nbj,bij->nbi", loc, R)
    out = ((rl + m[None] + b[None]) * w[:, :, None]).sum(1)
    rot = None
    if quat is not None:
        qb = normalize(quat_mat2quat(R))
        qs = normalize(w @ qb)
        rot = quat_multiply(qs, np.asarray(quat, np.float64))
    return out, rot, w
