"""The autotuner on the GPU: it restores the workload's state exactly, picks
one of its candidates, and the picked options give the same rollout as the
defaults within 1e-5 (the tolerance between launch options, which differ only
in FP32 reduction order)."""
import numpy as np
import pytest
import torch

from empm_b200 import autotune as A
from empm_b200.batch import BatchedMPM, single_instance
from tests.gpu_helpers import max_abs
from tests.test_gpu_batch import _specs

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def test_tune_batch_restores_state_and_agrees_with_defaults(tmp_path):
    specs = _specs(dynamic=True)
    batch = BatchedMPM(specs, device=DEV)
    x0 = batch.positions().clone()
    F0 = batch.F_trial().clone()
    cands = A.CANDIDATES[:4] + A.CANDIDATES[-2:]
    res = A.tune_batch(batch, 2e-4, substeps=8, candidates=cands, path=str(tmp_path / "t.json"), force=True)
    torch.cuda.synchronize()
    print(res["options"], {k: round(v, 4) for k, v in res["ms"].items()})
    assert res["options"] in cands and not res["cached"]
    assert torch.equal(batch.positions(), x0) and torch.equal(batch.F_trial(), F0) and batch.time == 0.0
    assert [c["point"] for c in specs[2].colliders if c["kind"] == "cuboid"] == [[0.45, 0.74, 0.45]]
    batch.rollout(2e-4, 24, block=12)
    ref = BatchedMPM(specs, device=DEV)
    ref.rollout(2e-4, 24, block=12)
    torch.cuda.synchronize()
    assert max_abs(batch.positions(), ref.positions()) <= 1e-5
    again = A.tune_batch(BatchedMPM(specs, device=DEV), 2e-4, path=str(tmp_path / "t.json"))
    assert again["cached"] and again["options"] == res["options"]


def test_tune_solver_restores_state():
    spec = _specs()[0]
    solver, md, st = single_instance(spec, device=DEV)
    x0 = st.particle_x.clone()
    res = A.tune_solver(solver, md, st, 2e-4, substeps=8, candidates=A.CANDIDATES[:3], force=True)
    torch.cuda.synchronize()
    assert res["options"] in A.CANDIDATES[:3]
    assert torch.equal(st.particle_x, x0) and solver.time == 0.0
    assert solver.sort_every == res["options"]["sort_every"]
