"""CPU checks of the Gaussian motion interpolation: the oracle against the
golden vectors made by the reference's own dynamic_utils functions, the C ABI's
argument checks (no device work), and the Python wrapper's input checks."""
import ctypes
import os

import numpy as np
import pytest
import torch

from empm_b200 import _native as N
from oracle import lbs_oracle as L

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "lbs.npz")


def case(name):
    g = np.load(GOLDEN)
    return {k.split("/", 1)[1]: g[k] for k in g.files if k.startswith(name + "/")}


def test_oracle_neighbours_and_weights_match_reference():
    c = case("generic")
    idx, _ = L.knn(c["bones"], c["bones"], 16, exclude_self=True)
    np.testing.assert_array_equal(idx, c["relations"])
    idx2, _ = L.knn(c["gauss"], c["bones"], 16)
    np.testing.assert_array_equal(idx2, c["knn_idx"])
    w = L.idw_weights(c["bones"], c["gauss"], c["knn_idx"])
    np.testing.assert_allclose(w, c["weights"], atol=2e-7)
    np.testing.assert_allclose(w, c["knn_weights"], atol=2e-7)


@pytest.mark.parametrize("convention", ["mat2quat", "kornia"])
def test_oracle_sparse_interpolation_matches_reference(convention):
    c = case("generic")
    R, how = L.bone_rotations(c["bones"], c["motions"], c["relations"])
    assert how == "kabsch"
    xyz, rot = L.blend_sparse(c["bones"], c["motions"], R[:, 0], c["gauss"], c["knn_idx"], c["weights"], c["quat"],
                              convention=convention)
    np.testing.assert_allclose(xyz, c["xyz"], atol=5e-7)
    # the golden took the reference's mat2quat fallback; kornia's conversion
    # agrees with it for rotations below 120 degrees
    np.testing.assert_allclose(rot, c["rot"], atol=5e-7)


def test_oracle_dense_interpolation_matches_reference():
    c = case("generic")
    R, _ = L.bone_rotations(c["bones"], c["motions"], c["relations"])
    W = np.zeros((len(c["gauss"]), len(c["bones"])))
    np.put_along_axis(W, c["knn_idx"], c["knn_weights"], 1)
    xyz, rot, _ = L.blend_dense(c["bones"], c["motions"], R[:, 0], c["gauss"], W, c["quat"])
    np.testing.assert_allclose(xyz, c["xyz_dense"], atol=5e-7)
    np.testing.assert_allclose(rot, c["rot_dense"], atol=5e-7)
    d = case("dense_default")
    R, _ = L.bone_rotations(d["bones"], d["motions"], d["relations"])
    xyz, rot, w = L.blend_dense(d["bones"], d["motions"], R[:, 0], d["gauss"], None, d["quat"])
    np.testing.assert_allclose(xyz, d["xyz"], atol=5e-7)
    np.testing.assert_allclose(rot, d["rot"], atol=5e-7)
    # torch.cdist's matrix-product distances carry float32 cancellation
    np.testing.assert_allclose(w, d["weights"], atol=1e-4)


@pytest.mark.parametrize("name,how", [("rank1_all", "rank1-all"), ("rank1_one", "rank1-broadcast"),
                                      ("rank1_two", "rank1-mismatch"), ("rank0_some", "mismatch")])
def test_oracle_rank_deficient_bones_match_reference(name, how):
    c = case(name)
    R, got = L.bone_rotations(c["bones"], c["motions"], c["relations"])
    assert got == how
    errs = []
    for s in range(2):   # axis sign of rank-1 bones: either SVD convention
        xyz, rot = L.blend_sparse(c["bones"], c["motions"], R[:, s], c["gauss"], c["knn_idx"], c["weights"],
                                  c["quat"], convention="mat2quat")
        errs.append(max(np.abs(xyz - c["xyz"]).max(), np.abs(rot - c["rot"]).max()))
    assert min(errs) < 5e-7, errs


def test_oracle_quaternion_helpers_match_reference():
    c = case("quat")
    np.testing.assert_array_equal(L.quat_mat2quat(c["R"]).astype(np.float32), c["mat2quat"])
    R64 = c["R"].astype(np.float64)
    tr = np.trace(R64, axis1=1, axis2=2)
    qk = L.normalize(L.quat_kornia(R64))
    qm = L.normalize(L.quat_mat2quat(R64))
    np.testing.assert_allclose(qk[tr > 0], qm[tr > 0], atol=1e-7)
    # both are the rotation's quaternion up to sign wherever they are unit
    q = L.normalize(L.quat_kornia(R64))
    w, x, y, z = q.T
    Rq = np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
                   2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                   2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], 1).reshape(-1, 3, 3)
    np.testing.assert_allclose(Rq, R64, atol=2e-6)


def test_abi_rejects_bad_arguments_without_gpu():
    lib = N.lib()
    f = (ctypes.c_float * 12)()
    i = (ctypes.c_longlong * 4)()
    assert lib.empm_knn(f, 4, f, 4, 0, 0, i, 8, None, None) == -1          # k < 1
    assert lib.empm_knn(f, 4, f, 4, 33, 0, i, 8, None, None) == -1         # k above the maximum
    assert lib.empm_knn(f, 4, f, 4, 4, 1, i, 8, None, None) == -1          # k > candidates without self
    assert lib.empm_knn(f, 4, f, 3, 2, 1, i, 8, None, None) == -1          # exclude_self, different sets
    assert lib.empm_knn(f, 4, f, 4, 2, 0, i, 2, None, None) == -1          # index width
    assert lib.empm_knn(f, 0, f, 4, 2, 0, i, 8, None, None) == 0           # nothing to do
    assert lib.empm_idw_weights(f, 4, f, 4, i, 8, 0, f, None, None) == -1
    assert lib.empm_idw_weights(f, 4, f, 0, i, 8, 2, f, None, None) == 0
    assert lib.empm_lbs_bones(f, f, 4, i, 8, 2, 7, f, f, None, None) == -1  # unknown convention
    assert lib.empm_lbs_bones(f, f, 4, i, 8, 2, 0, f, f, None, None) == -1  # no counts
    assert lib.empm_lbs_blend(f, 4, f, None, 4, i, 8, 0, f, None, f, None, None, None) == -1
    assert lib.empm_lbs_blend(f, 4, f, None, 0, i, 8, 2, f, None, f, None, None, None) == 0
    st = (ctypes.c_int * 1)()
    assert lib.empm_lbs_blend(f, 0, f, None, 4, i, 8, 2, f, None, f, None, st, None) == -1   # no bones
    assert lib.empm_lbs_blend_dense(f, 0, f, None, 4, None, None, f, None, None) == -1
    assert lib.empm_rotation_to_quat(f, 4, 5, f, None) == -1


def test_wrapper_requires_cuda_tensors():
    from empm_b200 import dynamic_utils as du
    x = torch.zeros(8, 3)
    with pytest.raises(RuntimeError, match="CUDA"):
        du.get_topk_indices(x, K=2)
    with pytest.raises(RuntimeError, match="CUDA"):
        du.mat2quat(torch.eye(3)[None])
    with pytest.raises(TypeError):
        du.interpolate_motions_speedup(x, x, None, x)
