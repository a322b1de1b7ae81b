"""The in-place substep MPMWARPDiff.p2g2p (mpm_solver_diff.py:293-429) on the
GPU against golden vectors of the reference's own kernels
(tests/golden/inplace.npz, made by tests/golden/make_golden.py): g2p with
atomic_add on x and the covariance update under update_cov_with_F
(mpm_utils.py:441-499), clip_particle_x (:582-599), unsimulated particles left
unchanged. Tolerances as in the other parity tests: positions 1e-4 of the
domain, other fields relative to their largest magnitude (2e-5 for F, 1e-4
for v, C and the covariances)."""
import json

import numpy as np
import pytest
import torch

from empm_b200 import WarpMPMWrapper
from tests.gpu_helpers import max_abs

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _rel(a, b):
    b = np.asarray(b, np.float64)
    return max_abs(a, b) / max(float(np.abs(b).max()), 1e-30)


@pytest.mark.parametrize("case", ["cov", "nocov"])
def test_inplace_substeps_vs_reference_golden(golden, case):
    g = golden("inplace")
    k = f"{case}/"
    s = json.loads(str(g[k + "scenario"]))
    n, G, dt, T = s["n"], s["G"], s["dt"], s["T"]
    t = lambda a, dtype=torch.float32: torch.as_tensor(np.asarray(a), dtype=dtype, device=DEV)  # noqa: E731
    mpm = WarpMPMWrapper(grid_size=G, grid_lim=1.0, frame_dt=dt, sim_dt=dt, device=DEV)
    mpm.gravity = list(s["gravity"])
    mpm.material_params = {"material": "plasticine", "yield_stress": 5000., "softening": 0.1}
    mpm.add_particles(t(g[k + "x0"]), t(g[k + "v0"]), float(s["vol"]), t(g[k + "E"]), t(g[k + "nu"]), s["rho"])
    mpm.surface_colliders.append([(0.0, 3.0 / G, 0.0), (0.0, 1.0, 0.0), "sticky", 0.0])
    c = s["cuboid"]
    mpm.moving_boundaries.append([c["point"], c["size"], c["velocity"], 0.0])
    mpm.initialize()
    mpm.mpm_solver.add_bounding_box()
    st, md, sv = mpm.mpm_state, mpm.mpm_model, mpm.mpm_solver
    md.yield_stress.copy_(t(g[k + "ys_in"]))
    imp = s["impulse"]
    sv.add_impulse_on_particles(st, force=imp["force"], dt=dt, point=imp["point"], size=imp["size"],
                                num_dt=imp["num_dt"], device=DEV)
    st.set_selection(t(g[k + "sel"], torch.int32))
    st.particle_cov.copy_(t(g[k + "cov0"]))
    md.update_cov_with_F = bool(s["update_cov"])
    x_before = st.particle_x.clone()
    for step in range(T):
        sv.p2g2p(md, st, step, dt, device=DEV)
    torch.cuda.synchronize()
    sel = np.asarray(g[k + "sel"]).astype(bool)
    errs = {
        "x": max_abs(st.particle_x, g[k + "x"].reshape(n, 3)),
        "v": _rel(st.particle_v, g[k + "v"].reshape(n, 3)),
        "C": _rel(st.particle_C.reshape(n, 3, 3), g[k + "C"].reshape(n, 3, 3)),
        "F_trial": _rel(st.particle_F_trial.reshape(n, 3, 3), g[k + "F_trial"].reshape(n, 3, 3)),
        "F": _rel(st.particle_F.reshape(n, 3, 3), g[k + "F"].reshape(n, 3, 3)),
        "cov": _rel(st.particle_cov, g[k + "cov"]),
        "yield": _rel(md.yield_stress, g[k + "ys_out"]),
    }
    print(case, {a: f"{b:.2e}" for a, b in errs.items()})
    assert errs["x"] <= 1e-4
    assert errs["F_trial"] <= 2e-5 and errs["F"] <= 2e-5
    assert errs["v"] <= 1e-4 and errs["C"] <= 1e-4 and errs["cov"] <= 1e-4 and errs["yield"] <= 1e-5
    # unsimulated particles keep their state, unlike the differentiable substep
    assert max_abs(st.particle_x[torch.from_numpy(sel).to(DEV)], x_before[torch.from_numpy(sel).to(DEV)]) == 0.0
    moved = float(np.abs(g[k + "x"].reshape(n, 3) - g[k + "x0"]).max())
    assert moved > 1e-3
    assert sv.read_status() & 1 == 0
