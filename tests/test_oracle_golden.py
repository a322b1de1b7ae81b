"""Pin the CPU oracle (oracle/mpm_oracle.c, FP64) against golden vectors
produced by the reference's own kernel source (tests/golden/make_golden.py).

Both sides compute in FP64 with the same statement order, so agreement is
expected at round-off level; the only algorithmic difference is the SVD
(LAPACK in the fixtures, one-sided Jacobi in the oracle), which leaves the
spectral stress functions unchanged.
"""
import json

import numpy as np
import pytest

from oracle import oracle as O
from tests import scenarios as S

RTOL = 1e-9


def _close(a, b, rtol=RTOL, atol_scale=1e-12):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-30)
    np.testing.assert_allclose(a, b, rtol=rtol, atol=atol_scale * scale)


def _model(L, G, material=0, grid_lim=1.0, gravity=(0.0, 0.0, 0.0), rpic=0.0, damping=1.1, softening=0.1,
           plastic_viscosity=0.0, alpha=0.0):
    m = L.OrModel()
    m.G = G
    m.grid_lim = grid_lim
    m.dx = grid_lim / G
    m.inv_dx = float(G / grid_lim)
    m.material = material
    m.gravity = (L.real * 3)(*gravity)
    m.rpic_damping = rpic
    m.grid_v_damping_scale = damping
    m.softening = softening
    m.plastic_viscosity = plastic_viscosity
    m.alpha = alpha
    return m


P = O._ptr


@pytest.mark.parametrize("material", range(7))
def test_stress_kernel(golden, material):
    g = golden("kernel_stress")
    k = f"m{material}/"
    L = O.lib("fp64")
    n = g[k + "F_trial"].shape[0]
    m = _model(L, 8, material=material, softening=float(g[k + "softening"]),
               plastic_viscosity=float(g[k + "plastic_viscosity"]), alpha=float(g[k + "alpha"]))
    Ft = np.ascontiguousarray(g[k + "F_trial"].reshape(n, 9))
    mu = g[k + "mu_in"].copy(); lam = g[k + "lam_in"].copy(); ys = g[k + "ys_in"].copy()
    E = g[k + "E"].copy(); nu = g[k + "nu"].copy()
    mu2 = np.zeros(n); lam2 = np.zeros(n)
    L.lib.or_mu_lam(n, P(E), P(nu), P(mu2), P(lam2))
    _close(mu2, mu)
    _close(lam2, lam)
    F = np.zeros((n, 9)); st = np.zeros((n, 9))
    L.lib.or_stress(m, n, None, P(Ft), P(mu), P(lam), P(ys), float(g[k + "dt"]), P(F), P(st))
    _close(F, g[k + "F"].reshape(n, 9), rtol=1e-8)
    _close(st, g[k + "stress"].reshape(n, 9), rtol=1e-7, atol_scale=1e-9)
    _close(ys, g[k + "ys_out"])
    _close(mu, g[k + "mu_out"])
    _close(lam, g[k + "lam_out"])


@pytest.mark.parametrize("tag", ["apic", "rpic", "pic"])
def test_p2g_kernel(golden, tag):
    g = golden("kernel_p2g")
    k = tag + "/"
    L = O.lib("fp64")
    G = int(g[k + "G"])
    n = g[k + "x"].shape[0]
    m = _model(L, G, rpic=float(g[k + "rpic"]))
    gm = np.zeros(G ** 3); gv = np.zeros(3 * G ** 3)
    arr = {a: np.ascontiguousarray(g[k + a].reshape(n, -1)).reshape(-1) for a in ("x", "v", "C", "stress", "vol", "mass")}
    L.lib.or_p2g(m, n, None, P(arr["x"]), P(arr["v"]), P(arr["C"]), P(arr["stress"]), P(arr["vol"]), P(arr["mass"]),
                 float(g[k + "dt"]), P(gm), P(gv))
    _close(gm, g[k + "grid_m"].reshape(-1))
    _close(gv, g[k + "grid_v_in"].reshape(-1))
    # partition of unity: sum of node masses equals sum of particle masses
    np.testing.assert_allclose(gm.sum(), arr["mass"].sum(), rtol=1e-12)


@pytest.mark.parametrize("tag", ["plain", "damped_colliders"])
def test_grid_kernel(golden, tag):
    g = golden("kernel_grid")
    k = tag + "/"
    L = O.lib("fp64")
    G = int(g[k + "G"])
    m = _model(L, G, gravity=tuple(g[k + "gravity"]), damping=float(g[k + "damping"]))
    specs = json.loads(str(g[k + "colliders"]))
    mask = g[k + "mask"]
    sim_specs = S.oracle_colliders(specs, mask=mask)
    sim = O.OracleSim(np.zeros((1, 3)), np.zeros((1, 3)), np.ones(1), np.ones(1), 1.0, 0.3, n_grid=G)
    sim.colliders = sim_specs
    coll, nc, _, _ = sim._tables(float(g[k + "dt"]))
    gm = np.ascontiguousarray(g[k + "grid_m"].reshape(-1))
    gv = np.ascontiguousarray(g[k + "grid_v_in"].reshape(-1))
    out = np.zeros(3 * G ** 3)
    L.lib.or_grid_update(m, P(gm), P(gv), P(out), coll, nc, float(g[k + "dt"]))
    _close(out, g[k + "grid_v_out"].reshape(-1))


def test_g2p_kernel(golden):
    g = golden("kernel_g2p")
    k = "g2p/"
    L = O.lib("fp64")
    G = int(g[k + "G"])
    n = g[k + "x"].shape[0]
    m = _model(L, G)
    x = np.ascontiguousarray(g[k + "x"].reshape(-1)); F = np.ascontiguousarray(g[k + "F"].reshape(-1))
    gv = np.ascontiguousarray(g[k + "grid_v_out"].reshape(-1))
    x1 = np.zeros(3 * n); v1 = np.zeros(3 * n); C1 = np.zeros(9 * n); F1 = np.zeros(9 * n)
    L.lib.or_g2p(m, n, None, P(x), P(F), P(gv), float(g[k + "dt"]), P(x1), P(v1), P(C1), P(F1))
    _close(x1, g[k + "x_out"].reshape(-1))
    _close(v1, g[k + "v_out"].reshape(-1))
    _close(C1, g[k + "C_out"].reshape(-1))
    _close(F1, g[k + "F_out"].reshape(-1))
    assert x1[0] == pytest.approx(2.0 / G)  # clamped into the [2dx, lim - 2dx] band


ROLLOUTS = ["jelly", "plasticine", "metal", "sand", "foam", "snow", "neohookean", "damped"]


@pytest.mark.parametrize("key", ROLLOUTS)
def test_rollout(golden, key):
    d = golden("rollouts")
    sim, s = S.oracle_from_rollout(d, key)
    traj = [sim.x.copy()]
    for f in range(s["n_frames"]):
        for _ in range(s["n_substeps"]):
            sim.substep(s["sim_dt"])
        traj.append(sim.x.copy())
    _close(np.stack(traj), d[f"{key}/traj"], rtol=1e-8, atol_scale=1e-10)
    _close(sim.v, d[f"{key}/v"].reshape(-1, 3), rtol=1e-6, atol_scale=1e-8)
    _close(sim.C, d[f"{key}/C"].reshape(-1, 9), rtol=1e-6, atol_scale=1e-8)
    _close(sim.F_trial, d[f"{key}/F_trial"].reshape(-1, 9), rtol=1e-8, atol_scale=1e-10)
    _close(sim.ys, d[f"{key}/ys_out"])
    _close(sim.mu, d[f"{key}/mu_out"])


def test_oracle_svd_properties():
    rng = np.random.default_rng(7)
    for i in range(200):
        A = rng.standard_normal((3, 3)) * (10.0 ** rng.uniform(-3, 3))
        if i % 7 == 0:
            A[:, 2] = A[:, 0] + 1e-9 * A[:, 1]   # nearly rank deficient
        U, s, V = O.svd3(A)
        np.testing.assert_allclose(U @ np.diag(s) @ V.T, A, atol=1e-12 * np.abs(A).max())
        assert np.linalg.det(U) == pytest.approx(1.0, abs=1e-12)
        assert np.linalg.det(V) == pytest.approx(1.0, abs=1e-12)
        assert s[0] >= s[1] >= abs(s[2]) - 1e-12 * s[0]
        assert np.sign(s[2]) == np.sign(np.linalg.det(A)) or abs(s[2]) < 1e-8 * s[0]


def test_restart_matches_reference_kernels():
    """restart_and_compute_F_C, against the reference's own kernels run under
    the FP64 Warp stand-in (tests/golden/kernel_restart.npz)."""
    import os
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "kernel_restart.npz"))
    F, x = O.restart(int(d["restart/G"]), d["restart/x"], d["restart/mass"], d["restart/target"])
    assert np.abs(F - d["restart/F_out"]).max() <= 1e-10
    assert np.array_equal(x, d["restart/x_out"])
    # with update_cov_with_F: the PhysGaussian covariance update
    n = d["restart_cov/x"].shape[0]
    F, x, cov = O.restart(int(d["restart_cov/G"]), d["restart_cov/x"], d["restart_cov/mass"], d["restart_cov/target"],
                          cov=d["restart_cov/cov"])
    assert np.abs(F - d["restart_cov/F_out"]).max() <= 1e-10
    assert np.abs(cov.reshape(-1) - d["restart_cov/cov_out"]).max() <= 1e-12
    assert np.abs(d["restart_cov/cov_out"] - d["restart_cov/cov"]).max() > 1e-4   # the update did something
