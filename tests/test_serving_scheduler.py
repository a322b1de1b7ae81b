"""Host-side policy of the request loop (no GPU): admission against the
capacities and the byte model, block lengths, re-layouts, cancellation,
deadlines and rejection of malformed or oversized requests."""
import numpy as np
import pytest

from empm_b200.batch import InstanceSpec
from empm_b200.serving import Capacity, Request, Scheduler, Ticket, checkpoint_bytes, grid_blocks


def _req(n=1000, G=32, T=100, grad=False, deadline=None, seed=0):
    rng = np.random.default_rng(seed)
    spec = InstanceSpec(x=rng.uniform(0.3, 0.7, (n, 3)).astype(np.float32),
                        vol=np.full(n, 1e-6, np.float32), rho=np.full(n, 1e3, np.float32),
                        E=np.full(n, 2e4, np.float32), nu=np.full(n, 0.3, np.float32), n_grid=G,
                        material="plasticine", yield_stress=np.full(n, 1e3, np.float32))
    tgt = spec.x.copy() if grad else None
    return Request(spec=spec, n_substeps=T, dt=1e-4, grad=grad, target=tgt, deadline_s=deadline)


def _cap(particles=10_000, blocks=10_000, instances=4, ckpt=10**9):
    return Capacity(particles=particles, blocks=blocks, instances=instances, ckpt_bytes=ckpt,
                    adjoint_particles=5_000, adjoint_blocks=grid_blocks(64))


def _submit(s, req, now=0.0):
    t = Ticket(req, now)
    return t, s.submit(t)


def test_admission_in_order_until_a_capacity_is_full():
    s = Scheduler(_cap(particles=2500, instances=8), block=50)
    ts = [_submit(s, _req(n=1000, seed=i))[0] for i in range(4)]
    p = s.plan(0.0)
    assert [t.id for t in p.admitted] == [ts[0].id, ts[1].id]      # a third would exceed 2500 particles
    assert p.relayout and p.block == 50
    assert len(s.pending) == 2
    # no change: no re-layout
    s.advance(p)
    p2 = s.plan(0.1)
    assert not p2.admitted and not p2.relayout
    assert p2.active == p.active


def test_no_overtaking_and_instance_slots():
    s = Scheduler(_cap(particles=100_000, instances=2), block=50)
    a, _ = _submit(s, _req(n=500))
    b, _ = _submit(s, _req(n=500))
    c, _ = _submit(s, _req(n=10))
    p = s.plan(0.0)
    assert [t.id for t in p.admitted] == [a.id, b.id]
    assert list(s.pending) == [c]


def test_blocks_run_full_length_and_finished_requests_are_held():
    s = Scheduler(_cap(), block=50)
    a, _ = _submit(s, _req(T=30))
    b, _ = _submit(s, _req(T=200, grad=True))
    lens = []
    for step in range(20):
        p = s.plan(float(step))
        if not p.active:
            break
        lens.append((p.block, [t.id for t in p.active]))
        s.advance(p)
    # a finishes inside the first block (held for its last 20 substeps) and
    # leaves at its end; b runs four full blocks, one checkpoint per boundary
    assert lens[0] == (50, [a.id, b.id])
    assert [L for L, _ in lens] == [50, 50, 50, 50]
    assert all(ids == [b.id] for _, ids in lens[1:])
    assert a.progress == 30 and b.progress == 200
    assert b in s.backward      # finished forward -> adjoint queue


def test_short_block_only_when_every_request_finishes_in_it():
    s = Scheduler(_cap(), block=50)
    a, _ = _submit(s, _req(T=70))
    b, _ = _submit(s, _req(T=80))
    p = s.plan(0.0)
    assert p.block == 50
    s.advance(p)
    p = s.plan(1.0)
    assert p.block == 30          # max remaining: 20 and 30
    s.advance(p)
    assert (a.progress, b.progress) == (70, 80)


def test_finished_and_cancelled_requests_leave_with_relayout():
    s = Scheduler(_cap(), block=50)
    a, _ = _submit(s, _req(T=50))
    b, _ = _submit(s, _req(T=500))
    p = s.plan(0.0)
    s.advance(p)
    b.cancel()
    p = s.plan(1.0)
    assert b in p.cancelled and b.phase == "cancelled"
    assert not p.active and p.relayout       # a finished, b cancelled
    assert s.idle()


def test_deadline_expiry():
    s = Scheduler(_cap(instances=1), block=50)
    a, _ = _submit(s, _req(T=1000))
    b, _ = _submit(s, _req(T=10, deadline=0.5))
    p = s.plan(0.0)
    assert p.admitted == [a]
    p = s.plan(1.0)       # b waited past its deadline
    assert b in p.cancelled and b.phase == "timeout"


def test_checkpoint_budget_blocks_admission_and_is_released():
    req = _req(n=1000, T=100, grad=True)
    need = checkpoint_bytes(req, 50)
    assert need == (100 // 50 + 3) * 1000 * (104 + 12)
    s = Scheduler(_cap(ckpt=int(need * 1.5)), block=50)
    a, _ = _submit(s, req)
    b, _ = _submit(s, _req(n=1000, T=100, grad=True, seed=1))
    p = s.plan(0.0)
    assert p.admitted == [a] and s.ckpt_in_use == need
    while a.progress < 100:
        s.advance(p)
        p = s.plan(0.0)
    assert a in s.backward
    assert b not in p.admitted        # a still holds its checkpoints during its adjoint
    s.release_backward(a)
    p = s.plan(0.0)
    assert p.admitted == [b]


def test_oversized_requests_are_rejected_at_submission():
    s = Scheduler(_cap(particles=500), block=50)
    _, why = _submit(s, _req(n=1000))
    assert "arena" in why
    s = Scheduler(_cap(blocks=10), block=50)
    _, why = _submit(s, _req(G=64))
    assert "grid" in why
    s = Scheduler(_cap(ckpt=1000), block=50)
    _, why = _submit(s, _req(grad=True))
    assert "checkpoint" in why
    s = Scheduler(_cap(), block=50)
    _, why = _submit(s, _req(n=6000, grad=True))
    assert "adjoint" in why


def test_malformed_requests_raise():
    r = _req()
    r.spec.x = r.spec.x[:, :2]
    with pytest.raises(ValueError):
        r.validate()
    r = _req()
    r.spec.x[0] = 1.5                      # outside the domain
    with pytest.raises(ValueError):
        r.validate()
    r = _req()
    r.n_substeps = 0
    with pytest.raises(ValueError):
        r.validate()
    r = _req(grad=True)
    r.target = None
    with pytest.raises(ValueError):
        r.validate()
    _req().validate()


def test_capacity_budget_charges_the_adjoint_store():
    """The adjoint engine's share of the budget includes its per-substep store
    (touched grid blocks, 2 KiB + 4 B each, and elastic F, 36 B per particle,
    for every substep of a segment); the rest is split between arena, grids
    and checkpoints."""
    from empm_b200.serving import capacity_for_budget

    budget = 60 << 30
    a = capacity_for_budget(budget, every=50, adjoint_particles=1_000_000, adjoint_grid=160)
    b = capacity_for_budget(budget, every=25, adjoint_particles=1_000_000, adjoint_grid=160)
    blocks = grid_blocks(160)
    store_50 = 50 * (blocks * (128 * 16 + 4) + 1_000_000 * 36)
    store_25 = 25 * (blocks * (128 * 16 + 4) + 1_000_000 * 36)
    # halving the segment length frees the store difference (and the segment states) for the other shares
    assert b.ckpt_bytes > a.ckpt_bytes
    freed = (b.ckpt_bytes - a.ckpt_bytes) / 0.35
    assert freed >= store_50 - store_25
    assert a.adjoint_blocks == blocks and a.adjoint_particles == 1_000_000
    with pytest.raises(ValueError):
        capacity_for_budget(store_50 // 2, every=50, adjoint_particles=1_000_000, adjoint_grid=160)
