"""GPU parity of the Gaussian motion interpolation kernels (csrc/lbs.cu)
against the golden vectors of the reference's dynamic_utils functions and the
NumPy oracle."""
import os

import numpy as np
import pytest
import torch

from oracle import lbs_oracle as L

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "lbs.npz")
DEV = "cuda:0"


def case(name):
    g = np.load(GOLDEN)
    return {k.split("/", 1)[1]: torch.as_tensor(g[k]).to(DEV) for k in g.files if k.startswith(name + "/")}


def np_case(name):
    g = np.load(GOLDEN)
    return {k.split("/", 1)[1]: g[k] for k in g.files if k.startswith(name + "/")}


@pytest.fixture(scope="module")
def du():
    from empm_b200 import dynamic_utils
    return dynamic_utils


def test_neighbours_and_weights_match_reference(du):
    c = case("generic")
    rel = du.get_topk_indices(c["bones"], K=16)
    assert rel.dtype == torch.int64
    assert torch.equal(rel, c["relations"].long())
    w, idx = du.knn_weights_sparse(c["bones"], c["gauss"], K=16)
    assert torch.equal(idx, c["knn_idx"].long())
    torch.testing.assert_close(w, c["knn_weights"], atol=2e-7, rtol=0)
    w2 = du.calc_weights_vals_from_indices(c["bones"], c["gauss"], c["knn_idx"])
    torch.testing.assert_close(w2, c["weights"], atol=2e-7, rtol=0)
    dense = du.knn_weights(c["bones"], c["gauss"], K=16)
    assert dense.shape == (c["gauss"].shape[0], c["bones"].shape[0])
    torch.testing.assert_close(dense.gather(1, idx), w, atol=0, rtol=0)
    assert int((dense != 0).sum()) == idx.numel()
    rm = du.create_relation_matrix(c["bones"][:100], K=5)
    assert rm.dtype == torch.int32 and rm.device.type == "cpu" and int(rm.sum()) == 500


@pytest.mark.parametrize("convention", ["kornia", "mat2quat"])
@pytest.mark.parametrize("idx_dtype", [torch.int64, torch.int32])
def test_sparse_interpolation_matches_reference(du, convention, idx_dtype):
    c = case("generic")
    xyz, rot, (w, wi) = du.interpolate_motions_speedup(
        bones=c["bones"], motions=c["motions"], relations=c["relations"].to(idx_dtype), xyz=c["gauss"],
        quat=c["quat"], weights=c["weights"], weights_indices=c["knn_idx"].to(idx_dtype), quat_convention=convention)
    torch.testing.assert_close(xyz, c["xyz"], atol=1e-6, rtol=0)
    torch.testing.assert_close(rot, c["rot"], atol=1e-6, rtol=0)
    assert w is c["weights"]
    # without quaternions the rot argument comes back unchanged
    sentinel = object()
    xyz2, rot2, _ = du.interpolate_motions_speedup(c["bones"], c["motions"], c["relations"], c["gauss"], rot=sentinel,
                                                   weights=c["weights"], weights_indices=c["knn_idx"])
    assert rot2 is sentinel
    torch.testing.assert_close(xyz2, xyz, atol=0, rtol=0)


def test_bone_rotations_match_oracle(du):
    c = case("generic")
    n = np_case("generic")
    bt = du.BoneTable(DEV)
    bt.fit(c["bones"], c["motions"], c["relations"], du.QUAT_KORNIA)
    assert bt.rank_counts() == (0, 0, c["bones"].shape[0])
    R_ref, _ = L.bone_rotations(n["bones"], n["motions"], n["relations"])
    R = bt.rotations(c["bones"].shape[0]).cpu().numpy()
    np.testing.assert_allclose(R, R_ref[:, 0], atol=2e-6)
    q = bt.quaternions(c["bones"].shape[0]).cpu().numpy()
    np.testing.assert_allclose(q, L.normalize(L.quat_kornia(R_ref[:, 0])), atol=2e-6)


def test_dense_interpolation_matches_reference(du):
    c = case("generic")
    W = torch.zeros(c["gauss"].shape[0], c["bones"].shape[0], device=DEV)
    W.scatter_(1, c["knn_idx"].long(), c["knn_weights"])
    xyz, rot, w = du.interpolate_motions(c["bones"], c["motions"], c["relations"], c["gauss"], quat=c["quat"],
                                         weights=W)
    torch.testing.assert_close(xyz, c["xyz_dense"], atol=1e-6, rtol=0)
    torch.testing.assert_close(rot, c["rot_dense"], atol=1e-6, rtol=0)
    assert w is W
    d = case("dense_default")
    xyz, rot, w = du.interpolate_motions(d["bones"], d["motions"], d["relations"], d["gauss"], quat=d["quat"])
    torch.testing.assert_close(xyz, d["xyz"], atol=1e-6, rtol=0)
    torch.testing.assert_close(rot, d["rot"], atol=1e-6, rtol=0)
    # the reference's distances come from torch.cdist's matrix-product form
    torch.testing.assert_close(w, d["weights"], atol=1e-4, rtol=0)


@pytest.mark.parametrize("name,counts", [("rank1_all", (0, 24, 0)), ("rank1_one", (0, 1, 49)),
                                         ("rank1_two", (0, 2, 48)), ("rank0_some", (5, 0, 39))])
def test_rank_deficient_bones_match_reference(du, name, counts):
    c = case(name)
    n = np_case(name)
    xyz, rot, _ = du.interpolate_motions_speedup(c["bones"], c["motions"], c["relations"], c["gauss"], quat=c["quat"],
                                                 weights=c["weights"], weights_indices=c["knn_idx"],
                                                 quat_convention="mat2quat")
    bt = du.BoneTable(DEV)
    bt.fit(c["bones"], c["motions"], c["relations"], du.QUAT_MAT2QUAT)
    assert bt.rank_counts() == counts
    # the axis sign of a rank-1 bone is the SVD's choice: accept the golden or
    # the oracle's result with the other sign
    R, _ = L.bone_rotations(n["bones"], n["motions"], n["relations"])
    alts = [(n["xyz"], n["rot"])]
    for s in range(2):
        alts.append(L.blend_sparse(n["bones"], n["motions"], R[:, s], n["gauss"], n["knn_idx"], n["weights"],
                                   n["quat"], convention="mat2quat"))
    got_x, got_q = xyz.cpu().numpy(), rot.cpu().numpy()
    err = min(max(np.abs(got_x - ax).max(), np.abs(got_q - aq).max()) for ax, aq in alts)
    assert err < 1e-6, err


def test_quaternion_helpers_match_reference(du):
    c = case("quat")
    torch.testing.assert_close(du.mat2quat(c["R"]), c["mat2quat"], atol=1e-6, rtol=0)
    n = np_case("quat")
    torch.testing.assert_close(du.rotation_matrix_to_quaternion(c["R"]).cpu(),
                               torch.as_tensor(L.quat_kornia(n["R"])), atol=1e-6, rtol=0)
    torch.testing.assert_close(du.quat2mat(c["quat_in"]), c["quat2mat"], atol=1e-6, rtol=0)


@pytest.mark.parametrize("k", [1, 5, 8, 16, 23, 32])
def test_knn_matches_oracle(du, k):
    rng = np.random.default_rng(k)
    pts = rng.uniform(0, 1, (3000, 3)).astype(np.float32)
    q = rng.uniform(0, 1, (2000, 3)).astype(np.float32)
    idx, dist = du._knn(torch.as_tensor(q, device=DEV), torch.as_tensor(pts, device=DEV), k, False)
    ridx, rdist = L.knn(q, pts, k)
    np.testing.assert_allclose(dist.cpu().numpy(), rdist, atol=1e-6)
    # indices equal wherever the distances are not tied within rounding
    agree = (idx.cpu().numpy() == ridx).mean()
    assert agree > 0.999, agree
    self_idx = du.get_topk_indices(torch.as_tensor(pts, device=DEV), K=k).cpu().numpy()
    sidx, _ = L.knn(pts, pts, k, exclude_self=True)
    assert (self_idx == sidx).mean() > 0.999
    assert not (self_idx == np.arange(len(pts))[:, None]).any()


def test_out_of_range_index_raises_and_leaves_the_device_usable(du):
    c = case("generic")
    bad = c["knn_idx"].clone().long()
    bad[5, 3] = c["bones"].shape[0] + 7
    with pytest.raises(IndexError):
        du.interpolate_motions_speedup(c["bones"], c["motions"], c["relations"], c["gauss"], quat=c["quat"],
                                       weights=c["weights"], weights_indices=bad)
    rel = c["relations"].clone().long()
    rel[0, 0] = -1
    with pytest.raises(IndexError):
        du.interpolate_motions_speedup(c["bones"], c["motions"], rel, c["gauss"], quat=c["quat"],
                                       weights=c["weights"], weights_indices=c["knn_idx"])
    with pytest.raises(IndexError):
        du.calc_weights_vals_from_indices(c["bones"], c["gauss"], bad)
    xyz, _, _ = du.interpolate_motions_speedup(c["bones"], c["motions"], c["relations"], c["gauss"],
                                               weights=c["weights"], weights_indices=c["knn_idx"])
    torch.testing.assert_close(xyz, c["xyz"], atol=1e-6, rtol=0)


def test_motion_interpolator_follows_the_trainer_loop(du):
    """Three frames through MotionInterpolator equal the trainer's calls."""
    rng = np.random.default_rng(7)
    n_p, n_g = 2000, 20000
    pos = [torch.as_tensor(rng.uniform(0.3, 0.7, (n_p, 3)), dtype=torch.float32, device=DEV)]
    for _ in range(3):
        pos.append(pos[-1] + torch.as_tensor(rng.normal(0, 2e-3, (n_p, 3)), dtype=torch.float32, device=DEV))
    xyz = torch.as_tensor(rng.uniform(0.3, 0.7, (n_g, 3)), dtype=torch.float32, device=DEV)
    q = torch.as_tensor(rng.normal(size=(n_g, 4)), dtype=torch.float32, device=DEV)
    q = q / q.norm(dim=1, keepdim=True)
    mi = du.MotionInterpolator(check=True)
    x1, q1 = xyz, q
    x2, q2 = xyz, q
    relations = weights_indices = None
    for f in range(1, 4):
        x1, q1 = mi(pos[f - 1], pos[f], x1, q1)
        if relations is None:
            relations = du.get_topk_indices(pos[f - 1], K=16)
        if weights_indices is None:
            _, weights_indices = du.knn_weights_sparse(pos[f - 1], x2, K=16)
        w = du.calc_weights_vals_from_indices(pos[f - 1], x2, weights_indices)
        x2, q2, _ = du.interpolate_motions_speedup(pos[f - 1], pos[f] - pos[f - 1], relations, x2, quat=q2,
                                                   weights=w, weights_indices=weights_indices)
    # the interpolator computes the weights inside the blend: same formula,
    # rounding may differ in the last bit
    torch.testing.assert_close(x1, x2, atol=1e-6, rtol=0)
    torch.testing.assert_close(q1, q2, atol=1e-6, rtol=0)
    assert torch.isfinite(x1).all() and (x1 - xyz).abs().max() > 1e-4


def test_motion_interpolator_reports_out_of_range_indices(du):
    rng = np.random.default_rng(9)
    prev = torch.as_tensor(rng.uniform(0.3, 0.7, (3000, 3)), dtype=torch.float32, device=DEV)
    cur = prev + 1e-3
    xyz = torch.as_tensor(rng.uniform(0.3, 0.7, (1000, 3)), dtype=torch.float32, device=DEV)
    q = torch.nn.functional.normalize(torch.as_tensor(rng.normal(size=(1000, 4)), dtype=torch.float32,
                                                      device=DEV), dim=1)
    mi = du.MotionInterpolator(check=True)
    x1, _ = mi(prev, cur, xyz, q)
    torch.testing.assert_close(x1, xyz + 1e-3, atol=2e-6, rtol=0)   # a pure translation
    mi.weights_indices[999, 15] = 3000
    with pytest.raises(IndexError):
        mi(prev, cur, xyz, q)
    mi.weights_indices[999, 15] = 0
    x2, _ = mi(prev, cur, xyz, q)
    torch.testing.assert_close(x2[:999], x1[:999], atol=0, rtol=0)
