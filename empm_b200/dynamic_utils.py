"""Gaussian motion interpolation on the device.

The functions of the reference's third_party/gaussian_splatting/dynamic_utils.py
with the same names, arguments and results, computed by the kernels of
``csrc/lbs.cu``. The reference calls them once per rendered frame to move the
scene's Gaussians with the simulated particles (trainer_warp_mpm.py:1626-1659,
scripts/interactive_viser.py:258-275, scripts/gs/gs_render_dynamics.py:239-262);
``MotionInterpolator`` is that per-frame loop with its buffers kept.

Differences from the reference, by design:
  * every tensor argument must be on a CUDA device (the reference computes
    knn_weights_sparse on the CPU and the rest where its inputs live);
  * the quaternion of a bone rotation uses kornia 0.8.1's conversion in
    interpolate_motions_speedup (what the reference imports; ``quat_convention``
    selects the reference's mat2quat fallback instead) and mat2quat in
    interpolate_motions, as the reference does;
  * neighbour lists come from an exact search with ties in index order
    (torch.topk leaves tie order unspecified); get_topk_indices leaves each
    point's own index out instead of dropping the first of K + 1, which differs
    only where points coincide;
  * a rank-1 bone's axis sign follows this library's SVD (the reference's
    follows its LAPACK/cuSOLVER build).
"""
from __future__ import annotations

from typing import Optional, Tuple

import torch
from torch import Tensor

from . import _native as N

QUAT_KORNIA, QUAT_MAT2QUAT = 0, 1
TABLE_FLOATS = 16
N_COUNTS = 8
_STATUS, _BLEND_STATUS = 6, 7
_CONVENTIONS = {"kornia": QUAT_KORNIA, "mat2quat": QUAT_MAT2QUAT}


def _stream(t: Tensor) -> int:
    return torch.cuda.current_stream(t.device).cuda_stream


def _cuda(t: Tensor, name: str) -> Tensor:
    if not isinstance(t, Tensor) or not t.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor: the interpolation runs on the GPU")
    return t


def _f32(t: Tensor, name: str, cols: Optional[int] = None) -> Tensor:
    t = _cuda(t, name).detach().to(torch.float32).contiguous()
    if cols is not None and (t.dim() != 2 or t.shape[1] != cols):
        raise ValueError(f"{name} must be [n, {cols}], got {tuple(t.shape)}")
    return t


def _idx(t: Tensor, name: str, device) -> Tuple[Tensor, int]:
    t = torch.as_tensor(t).to(device)
    if t.dim() != 2:
        raise ValueError(f"{name} must be [n, k], got {tuple(t.shape)}")
    if t.dtype == torch.int32:
        return t.contiguous(), 4
    return t.to(torch.int64).contiguous(), 8


def _raise_on_status(counts: Tensor) -> None:
    c = counts.cpu()
    if int(c[_STATUS]) | int(c[_BLEND_STATUS]):
        raise IndexError("bone index out of range in relations or neighbour indices")


# ---------------------------------------------------------------------------
# quaternions
# ---------------------------------------------------------------------------
def quat2mat(q: Tensor) -> Tensor:
    """Rotation matrices of (w, x, y, z) quaternions, normalised first (:5-22)."""
    q = q / torch.sqrt((q * q).sum(1))[:, None]
    r, x, y, z = q.unbind(1)
    return torch.stack([1 - 2 * (y * y + z * z), 2 * (x * y - r * z), 2 * (x * z + r * y),
                        2 * (x * y + r * z), 1 - 2 * (x * x + z * z), 2 * (y * z - r * x),
                        2 * (x * z - r * y), 2 * (y * z + r * x), 1 - 2 * (x * x + y * y)], 1).reshape(-1, 3, 3)


def _rotation_to_quat(rot: Tensor, convention: int) -> Tensor:
    R = _f32(rot, "rot").reshape(-1, 9)
    q = torch.empty(R.shape[0], 4, dtype=torch.float32, device=R.device)
    N.check(N.lib().empm_rotation_to_quat(R.data_ptr(), R.shape[0], convention, q.data_ptr(), _stream(R)))
    return q


def mat2quat(rot: Tensor) -> Tensor:
    """(w, x, y, z) of [n, 3, 3] rotations, the reference's mat2quat (:25-64)."""
    return _rotation_to_quat(rot, QUAT_MAT2QUAT)


def rotation_matrix_to_quaternion(rotation_matrix: Tensor) -> Tensor:
    """kornia 0.8.1's conversion of [n, 3, 3] rotations to (w, x, y, z)."""
    return _rotation_to_quat(rotation_matrix, QUAT_KORNIA)


# ---------------------------------------------------------------------------
# neighbours and weights
# ---------------------------------------------------------------------------
def _knn(queries: Tensor, points: Tensor, k: int, exclude_self: bool) -> Tuple[Tensor, Tensor]:
    q = _f32(queries, "queries", 3)
    p = _f32(points, "points", 3)
    idx = torch.empty(q.shape[0], k, dtype=torch.int64, device=q.device)
    dist = torch.empty(q.shape[0], k, dtype=torch.float32, device=q.device)
    N.check(N.lib().empm_knn(q.data_ptr(), q.shape[0], p.data_ptr(), p.shape[0], int(k), int(exclude_self),
                             idx.data_ptr(), 8, dist.data_ptr(), _stream(q)))
    return idx, dist


def get_topk_indices(points: Tensor, K: int = 5) -> Tensor:
    """[N, K] int64 indices of every point's K nearest other points (:248-265)."""
    return _knn(points, points, K, True)[0]


def create_relation_matrix(points: Tensor, K: int = 5) -> Tensor:
    """[N, N] int32 CPU matrix with ones at each row's K nearest other points (:219-245)."""
    idx = get_topk_indices(points, K).cpu()
    n = points.shape[0]
    rel = torch.zeros((n, n), dtype=torch.int)
    rel[torch.arange(n).unsqueeze(1).expand(-1, K), idx] = 1
    return rel


def calc_weights_vals_from_indices(bones: Tensor, pts: Tensor, indices: Tensor) -> Tensor:
    """Inverse-distance weights 1 / (d + 1e-6) of the given bones, normalised per row (:282-292)."""
    b = _f32(bones, "bones", 3)
    p = _f32(pts, "pts", 3)
    idx, nbytes = _idx(indices, "indices", p.device)
    k = idx.shape[1]
    w = torch.empty(p.shape[0], k, dtype=torch.float32, device=p.device)
    status = torch.zeros(1, dtype=torch.int32, device=p.device)
    N.check(N.lib().empm_idw_weights(b.data_ptr(), b.shape[0], p.data_ptr(), p.shape[0], idx.data_ptr(), nbytes, k,
                                     w.data_ptr(), status.data_ptr(), _stream(p)))
    if int(status.item()):
        raise IndexError("bone index out of range in indices")
    return w


def knn_weights_sparse(bones: Tensor, pts: Tensor, K: int = 5) -> Tuple[Tensor, Tensor]:
    """(weights [n, K], indices [n, K] int64) of every point's K nearest bones (:295-302)."""
    idx, _ = _knn(pts, bones, K, False)
    return calc_weights_vals_from_indices(bones, pts, idx), idx


def knn_weights(bones: Tensor, pts: Tensor, K: int = 5) -> Tensor:
    """Dense [n_pts, n_bones] weights, nonzero at each point's K nearest bones (:268-279)."""
    w, idx = knn_weights_sparse(bones, pts, K)
    out = torch.zeros(pts.shape[0], bones.shape[0], dtype=torch.float32, device=w.device)
    return out.scatter_(1, idx, w)


# ---------------------------------------------------------------------------
# interpolation
# ---------------------------------------------------------------------------
class BoneTable:
    """Device buffers of the bone stage, reusable across frames."""

    def __init__(self, device):
        self.device = torch.device(device)
        self.table = torch.empty(0, device=self.device)
        self.work = torch.empty(0, device=self.device)
        self.counts = torch.zeros(N_COUNTS, dtype=torch.int32, device=self.device)

    def fit(self, bones: Tensor, motions: Tensor, relations: Tensor, convention: int) -> Tensor:
        b = _f32(bones, "bones", 3)
        m = _f32(motions, "motions", 3)
        if m.shape != b.shape:
            raise ValueError(f"motions {tuple(m.shape)} must match bones {tuple(b.shape)}")
        rel, nbytes = _idx(relations, "relations", b.device)
        if rel.shape[0] != b.shape[0]:
            raise ValueError(f"relations must have one row per bone ({b.shape[0]}), got {rel.shape[0]}")
        n = b.shape[0]
        if self.table.numel() < n * TABLE_FLOATS:
            self.table = torch.empty(n * TABLE_FLOATS, dtype=torch.float32, device=b.device)
            self.work = torch.empty(n * 10, dtype=torch.float32, device=b.device)
        N.check(N.lib().empm_lbs_bones(b.data_ptr(), m.data_ptr(), n, rel.data_ptr(), nbytes, rel.shape[1],
                                       convention, self.table.data_ptr(), self.work.data_ptr(),
                                       self.counts.data_ptr(), _stream(b)))
        return self.table

    def rotations(self, n_bones: int) -> Tensor:
        """[n_bones, 3, 3] final bone rotations of the last fit (rebuilt from
        the table's unit quaternion (x, y, z, w) at floats 6-9 of each row)."""
        x, y, z, w = self.table[: n_bones * TABLE_FLOATS].view(n_bones, TABLE_FLOATS)[:, 6:10].unbind(1)
        return quat2mat(torch.stack([w, x, y, z], 1))

    def quaternions(self, n_bones: int) -> Tensor:
        """[n_bones, 4] (w, x, y, z) blended quaternions of the last fit (floats 10-13)."""
        return self.table[: n_bones * TABLE_FLOATS].view(n_bones, TABLE_FLOATS)[:, 10:14].clone()

    def rank_counts(self) -> Tuple[int, int, int]:
        """Bones of rank 0, 1 and 2-3 in the last fit."""
        c = self.counts.cpu()
        return int(c[0]), int(c[1]), int(c[2])


def _blend(bt: BoneTable, n_bones: int, xyz: Tensor, quat: Optional[Tensor], idx: Tensor, nbytes: int,
           w: Optional[Tensor], w_out: Optional[Tensor] = None) -> Tuple[Tensor, Optional[Tensor]]:
    """w None: inverse-distance weights to the table's bones, computed in the
    blend (and written to w_out when given)."""
    x = _f32(xyz, "xyz", 3)
    q = None if quat is None else _f32(quat, "quat", 4)
    if q is not None and q.shape[0] != x.shape[0]:
        raise ValueError("quat must have one row per Gaussian")
    if idx.shape[0] != x.shape[0] or (w is not None and w.shape != idx.shape):
        raise ValueError(f"weights / indices {tuple(idx.shape)} must be [n_gaussians, k]")
    xo = torch.empty_like(x)
    qo = None if q is None else torch.empty_like(q)
    status = bt.counts[_BLEND_STATUS:]
    N.check(N.lib().empm_lbs_blend(bt.table.data_ptr(), n_bones, x.data_ptr(), 0 if q is None else q.data_ptr(),
                                   x.shape[0], idx.data_ptr(), nbytes, idx.shape[1],
                                   0 if w is None else w.data_ptr(), 0 if w_out is None else w_out.data_ptr(),
                                   xo.data_ptr(), 0 if qo is None else qo.data_ptr(), status.data_ptr(), _stream(x)))
    return xo, qo


def interpolate_motions_speedup(bones, motions, relations, xyz, rot=None, quat=None, weights=None,
                                weights_indices=None, device='cuda', step='n/a', quat_convention: str = "kornia",
                                check: bool = True):
    """Move Gaussians with their K weighted bones (:305-491).

    Returns (xyz_transformed [n, 3], rot, (weights, weights_indices)); rot is
    the new (w, x, y, z) quaternion of every Gaussian when quat is given, else
    the rot argument unchanged. check: read the status word back (one
    synchronisation) and raise IndexError on an out-of-range index."""
    if weights is None or weights_indices is None:
        raise TypeError("interpolate_motions_speedup needs weights and weights_indices")
    bt = BoneTable(_cuda(xyz, "xyz").device)
    n_bones = bones.shape[0]
    bt.fit(bones, motions, relations, _CONVENTIONS[quat_convention])
    idx, nbytes = _idx(weights_indices, "weights_indices", bt.device)
    w = _f32(weights, "weights")
    xo, qo = _blend(bt, n_bones, xyz, quat, idx, nbytes, w)
    if check:
        _raise_on_status(bt.counts)
    return xo, (qo if quat is not None else rot), (weights, weights_indices)


def interpolate_motions(bones, motions, relations, xyz, rot=None, quat=None, weights=None, device='cuda',
                        step='n/a', check: bool = True):
    """Move Gaussians with dense [n, n_bones] weights (:67-216); weights None:
    1 / max(d, 1e-4) to every bone, normalised. Returns (xyz, rot, weights)."""
    bt = BoneTable(_cuda(xyz, "xyz").device)
    n_bones = bones.shape[0]
    bt.fit(bones, motions, relations, QUAT_MAT2QUAT)
    x = _f32(xyz, "xyz", 3)
    q = None if quat is None else _f32(quat, "quat", 4)
    if weights is None:
        w_in = None
        w_out = torch.empty(x.shape[0], n_bones, dtype=torch.float32, device=x.device)
    else:
        w_in = _f32(weights, "weights")
        if w_in.shape != (x.shape[0], n_bones):
            raise ValueError(f"weights must be [{x.shape[0]}, {n_bones}], got {tuple(w_in.shape)}")
        w_out = None
    xo = torch.empty_like(x)
    qo = None if q is None else torch.empty_like(q)
    N.check(N.lib().empm_lbs_blend_dense(bt.table.data_ptr(), n_bones, x.data_ptr(), 0 if q is None else q.data_ptr(),
                                         x.shape[0], 0 if w_in is None else w_in.data_ptr(),
                                         0 if w_out is None else w_out.data_ptr(), xo.data_ptr(),
                                         0 if qo is None else qo.data_ptr(), _stream(x)))
    if check:
        _raise_on_status(bt.counts)
    return xo, (qo if quat is not None else rot), (weights if weights is not None else w_out)


class MotionInterpolator:
    """The trainer's per-frame Gaussian update (trainer_warp_mpm.py:1626-1659)
    with its buffers kept: on the first frame the bones' K nearest bones
    (relations) and every Gaussian's K nearest bones are found; every frame
    then fits the bone rotations and moves positions and quaternions in one
    pass that also recomputes the inverse-distance weights from the previous
    particle positions (kept in ``weights`` when keep_weights is set). The
    neighbour indices are held as int32."""

    def __init__(self, k_relations: int = 16, k_weights: int = 16, quat_convention: str = "kornia",
                 check: bool = False, keep_weights: bool = False):
        self.k_relations = k_relations
        self.k_weights = k_weights
        self.convention = _CONVENTIONS[quat_convention]
        self.check = check
        self.keep_weights = keep_weights
        self.relations: Optional[Tensor] = None
        self.weights_indices: Optional[Tensor] = None
        self.weights: Optional[Tensor] = None
        self.bt: Optional[BoneTable] = None
        self.status = None

    def reset(self) -> None:
        self.relations = self.weights_indices = self.weights = None

    def __call__(self, prev_pos: Tensor, cur_pos: Tensor, xyz: Tensor, quat: Optional[Tensor]):
        """(xyz, quat) of the Gaussians after the particles moved prev_pos -> cur_pos."""
        dev = _cuda(prev_pos, "prev_pos").device
        if self.bt is None or self.bt.device != dev:
            self.bt = BoneTable(dev)
        prev = _f32(prev_pos, "prev_pos", 3)
        if self.relations is None:
            self.relations = get_topk_indices(prev, self.k_relations).to(torch.int32)
        if self.weights_indices is None:
            self.weights_indices = _knn(xyz, prev, self.k_weights, False)[0].to(torch.int32)
        x = _f32(xyz, "xyz", 3)
        n_b = prev.shape[0]
        if self.keep_weights and (self.weights is None or self.weights.shape != self.weights_indices.shape):
            self.weights = torch.empty(self.weights_indices.shape, dtype=torch.float32, device=dev)
        motions = _f32(cur_pos, "cur_pos", 3) - prev
        self.bt.fit(prev, motions, self.relations, self.convention)
        xo, qo = _blend(self.bt, n_b, x, quat, self.weights_indices, 4, None,
                        self.weights if self.keep_weights else None)
        if self.check:
            _raise_on_status(self.bt.counts)
        return xo, qo
