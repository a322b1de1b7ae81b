"""The static-pose restart (restart_and_compute_F_C) on the GPU, against the
reference's own kernels run under the FP64 Warp stand-in
(tests/golden/kernel_restart.npz): F_trial within 2e-5 relative (FP32
scatter/gather of displacements), positions equal to the targets. Also the
autograd Function's static_pos path, which uses it."""
import os

import numpy as np
import pytest
import torch

from empm_b200 import MPMDifferentiableSimulation, MPMModelStruct, MPMStateStruct, MPMWARPDiff

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
HERE = os.path.dirname(__file__)


def _t(a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device=DEV)


def test_restart_matches_reference_kernels():
    d = np.load(os.path.join(HERE, "golden", "kernel_restart.npz"))
    G, x, mass, target = int(d["restart/G"]), d["restart/x"], d["restart/mass"], d["restart/target"]
    n = x.shape[0]
    st = MPMStateStruct()
    st.init(n, device=DEV)
    st.from_torch(_t(x), _t(np.full(n, 1e-6)), None, None, n_grid=G, device=DEV)
    st.particle_mass = _t(mass)
    md = MPMModelStruct()
    md.init(n, device=DEV)
    md.init_other_params(n_grid=G)
    sv = MPMWARPDiff()
    sv.initialize(n, n_grid=G, device=DEV)
    sv.restart_and_compute_F_C(md, st, _t(target), device=DEV)
    torch.cuda.synchronize()
    F = st.particle_F_trial.double().cpu().numpy()
    ref = d["restart/F_out"]
    err = np.abs(F - ref).max()
    print(f"restart F_trial max err {err:.2e}")
    assert err <= 2e-5 * np.abs(ref).max()
    assert np.array_equal(st.particle_x.cpu().numpy(), target.astype(np.float32))
    assert float(st.particle_C.abs().max()) == 0.0


def test_restart_covariance_update_matches_reference_kernels():
    """update_cov_with_F: particle_cov += G cov + cov G^T with the restart's
    displacement gradient G, as the reference's set_F_C_g2p does."""
    d = np.load(os.path.join(HERE, "golden", "kernel_restart.npz"))
    G, x, mass, target = int(d["restart_cov/G"]), d["restart_cov/x"], d["restart_cov/mass"], d["restart_cov/target"]
    n = x.shape[0]
    st = MPMStateStruct()
    st.init(n, device=DEV)
    st.from_torch(_t(x), _t(np.full(n, 1e-6)), _t(d["restart_cov/cov"]), None, n_grid=G, device=DEV)
    st.particle_mass = _t(mass)
    md = MPMModelStruct()
    md.init(n, device=DEV)
    md.init_other_params(n_grid=G)
    md.update_cov_with_F = True
    sv = MPMWARPDiff()
    sv.initialize(n, n_grid=G, device=DEV)
    sv.restart_and_compute_F_C(md, st, _t(target), device=DEV)
    torch.cuda.synchronize()
    cov = st.particle_cov.double().cpu().numpy()
    ref = d["restart_cov/cov_out"]
    err = np.abs(cov - ref).max()
    print(f"restart covariance max err {err:.2e}")
    assert err <= 2e-5 * np.abs(ref).max()
    # off by default, as in the reference
    st2 = MPMStateStruct()
    st2.init(n, device=DEV)
    st2.from_torch(_t(x), _t(np.full(n, 1e-6)), _t(d["restart_cov/cov"]), None, n_grid=G, device=DEV)
    st2.particle_mass = _t(mass)
    md.update_cov_with_F = False
    sv.restart_and_compute_F_C(md, st2, _t(target), device=DEV)
    torch.cuda.synchronize()
    assert np.array_equal(st2.particle_cov.cpu().numpy(), d["restart_cov/cov"].astype(np.float32))


def test_simulation_function_with_static_pose():
    rng = np.random.default_rng(9)
    n, G = 2000, 32
    static = rng.uniform(0.35, 0.65, (n, 3)).astype(np.float32)
    posed = (static + 0.01 * rng.standard_normal((n, 3))).astype(np.float32)
    st = MPMStateStruct()
    st.init(n, device=DEV)
    st.from_torch(_t(static), _t(np.full(n, 0.027 / n)), None, None, n_grid=G, device=DEV)
    md = MPMModelStruct()
    md.init(n, device=DEV)
    md.init_other_params(n_grid=G)
    sv = MPMWARPDiff()
    sv.initialize(n, n_grid=G, device=DEV)
    sv.add_bounding_box()
    rho = _t(np.full(n, 1e3))
    out = MPMDifferentiableSimulation.apply(sv, st, md, 1, 2e-4, 10, _t(posed), _t(np.zeros((n, 3))),
                                            torch.tensor(2e4, device=DEV), torch.tensor(0.3, device=DEV), rho,
                                            torch.ones(n, dtype=torch.int32, device=DEV), _t(static), DEV, False, 0)
    torch.cuda.synchronize()
    assert out.shape == (n, 3) and torch.isfinite(out).all()
    # the restart moved the particles to the posed positions before the substeps
    assert float((out - _t(posed)).abs().max()) < 0.01
