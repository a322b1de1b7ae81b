"""Host-side logic of the checkpointed rollout (no GPU): where segments start
and end, and where record adjoints are injected."""
from empm_b200.adjoint import CheckpointedRollout


def _bounds(n_steps, every, record_every=None):
    return CheckpointedRollout(None, None, None, 1e-4, n_steps, checkpoint_every=every,
                               record_every=record_every)._bounds()


def test_segments_every_k_substeps():
    assert _bounds(10, 4) == [0, 4, 8, 10]
    assert _bounds(8, 4) == [0, 4, 8]
    assert _bounds(3, 20) == [0, 3]
    assert _bounds(1, 1) == [0, 1]


def test_segments_end_at_records():
    # records after substeps 0, 3, 6, 9 -> segment ends at states 1, 4, 7 (10 is the end)
    b = _bounds(10, 20, record_every=3)
    assert b == [0, 1, 4, 7, 10]
    b = _bounds(10, 4, record_every=5)
    assert b == [0, 1, 4, 6, 8, 10]


def test_record_steps_follow_trail_recording():
    t = CheckpointedRollout(None, None, None, 1e-4, 10, checkpoint_every=4, record_every=3)
    assert t.record_steps == [0, 3, 6, 9]


# ---------------------------------------------------------------------------
# stored segments: the budget, the context's pool and the grid-store size
# (a fake library and context stand in for the device)
# ---------------------------------------------------------------------------
import ctypes  # noqa: E402

import pytest  # noqa: E402

from empm_b200 import _native as N  # noqa: E402
from empm_b200.mpm_solver_diff import _Context  # noqa: E402


class _FakeLib:
    """empm_segment_* with a byte count of steps * (1000 + 10 * block_cap)."""

    def __init__(self, fail_after=None):
        self.created, self.destroyed = [], []
        self.fail_after = fail_after
        self._next = 1

    def empm_segment_bytes(self, ctx, n_steps, block_cap, out):
        out._obj.value = n_steps * (1000 + 10 * block_cap)
        return N.EMPM_OK

    def empm_segment_create(self, ctx, n_steps, block_cap, out):
        if self.fail_after is not None and len(self.created) >= self.fail_after:
            return N.EMPM_ERR_OOM
        out._obj.value = self._next
        self.created.append((self._next, n_steps, block_cap))
        self._next += 1
        return N.EMPM_OK

    def empm_segment_destroy(self, seg):
        self.destroyed.append(seg.value if hasattr(seg, "value") else seg)
        return N.EMPM_OK


def _fake_ctx(lib):
    ctx = _Context.__new__(_Context)   # no device context: only the pool logic is used
    ctx.L = lib
    ctx.ptr = None
    ctx.segment_pool = {}
    ctx.touched_blocks = None
    return ctx


def _tape(n_steps, every, store=None, budget=None):
    t = CheckpointedRollout(None, None, None, 1e-4, n_steps, checkpoint_every=every, store=store,
                            store_budget=budget)
    t.bounds = t._bounds()
    return t


def _no_device(monkeypatch):
    import contextlib

    import torch

    monkeypatch.setattr(torch.cuda, "device", lambda d: contextlib.nullcontext())


@pytest.fixture
def fake_lib(monkeypatch):
    lib = _FakeLib()
    monkeypatch.setattr(N, "lib", lambda: lib)
    _no_device(monkeypatch)
    return lib


def test_store_decision_and_budget(fake_lib):
    ctx = _fake_ctx(fake_lib)
    # 10 substeps in segments of 4, 4, 2 at 100 blocks: (8 + 2) * 2000 bytes
    assert not _tape(10, 4, store=False)._allocate_segments(ctx, "cpu", 100)
    assert not _tape(10, 4, budget=19_999)._allocate_segments(ctx, "cpu", 100)
    with pytest.raises(MemoryError):
        _tape(10, 4, store=True, budget=19_999)._allocate_segments(ctx, "cpu", 100)
    assert fake_lib.created == []
    t = _tape(10, 4, budget=20_000)
    assert t._allocate_segments(ctx, "cpu", 100)
    assert [(sg.step, sg.n_steps, sg.block_cap) for sg in t.segments] == [(0, 4, 100), (4, 4, 100), (8, 2, 100)]


def test_pool_reuse_counts_as_available(fake_lib):
    ctx = _fake_ctx(fake_lib)
    t = _tape(10, 4, budget=20_000)
    assert t._allocate_segments(ctx, "cpu", 100)
    t.release()
    assert ctx.pooled(4, 100) == 2 and ctx.pooled(2, 100) == 1
    # the same rollout again: everything comes from the pool, nothing is created
    n_created = len(fake_lib.created)
    t2 = _tape(10, 4, budget=20_000)
    assert t2._allocate_segments(ctx, "cpu", 100)
    assert len(fake_lib.created) == n_created and ctx.pooled(4) == 0
    # a larger block capacity cannot use the pooled segments
    t2.release()
    t3 = _tape(10, 4, budget=10 ** 9)
    assert t3._allocate_segments(ctx, "cpu", 200)
    assert len(fake_lib.created) == n_created + 3 and ctx.pooled(4, 100) == 2


def test_out_of_memory_falls_back_or_raises(monkeypatch):
    lib = _FakeLib(fail_after=1)
    monkeypatch.setattr(N, "lib", lambda: lib)
    _no_device(monkeypatch)
    monkeypatch.setattr(N, "last_error", lambda ptr=None: "segment store does not fit")
    ctx = _fake_ctx(lib)
    t = _tape(10, 4, budget=10 ** 9)
    assert not t._allocate_segments(ctx, "cpu", 100)      # automatic: checkpoints instead
    assert t.segments == [] and ctx.pooled(4, 100) == 1   # the one made is pooled, not leaked
    with pytest.raises(MemoryError):
        _tape(10, 4, store=True, budget=10 ** 9)._allocate_segments(ctx, "cpu", 100)


def test_block_capacity_estimate_and_oversized_segments(fake_lib):
    ctx = _fake_ctx(fake_lib)
    t = _tape(8, 4, budget=10 ** 9)
    assert t._block_cap(ctx, 200_000) == 781            # first guess: N / 256
    assert t._block_cap(ctx, 1000) == 512
    assert t._allocate_segments(ctx, "cpu", t._block_cap(ctx, 200_000))
    ctx.touched_blocks = 100                            # a pass measured 100 blocks
    assert t._block_cap(ctx, 200_000) == 141
    t.release()                                          # 781 > 2 * 125 + 64: freed, not pooled
    assert ctx.pooled(4) == 0 and len(fake_lib.destroyed) == 2
    t = _tape(8, 4, budget=10 ** 9)
    assert t._allocate_segments(ctx, "cpu", t._block_cap(ctx, 200_000))
    t.release()                                          # right-sized: pooled
    assert ctx.pooled(4, 141) == 2


def test_overflow_check_updates_the_estimate(fake_lib):
    """_blocks_overflowed reads each segment's touched-block maximum once,
    keeps the largest as the context's estimate and reports a segment whose
    slots were too few."""
    maxima = {}

    def blocks(seg, max_touched, block_cap, stream):
        touched, cap = maxima[seg.value]
        max_touched._obj.value = touched
        block_cap._obj.value = cap
        return N.EMPM_OK

    fake_lib.empm_segment_blocks = blocks
    ctx = _fake_ctx(fake_lib)
    t = _tape(10, 4, budget=10 ** 9)
    assert t._allocate_segments(ctx, "cpu", 100)
    ids = [sg.ptr.value for sg in t.segments]
    maxima.update({ids[0]: (60, 100), ids[1]: (90, 100), ids[2]: (40, 100)})
    assert not t._blocks_overflowed(ctx, None)
    assert ctx.touched_blocks == 90
    maxima[ids[1]] = (130, 100)
    assert t._blocks_overflowed(ctx, None)
    assert ctx.touched_blocks == 130
    assert t._block_cap(ctx, 10 ** 6) == int(130 * 1.25) + 16
    maxima[ids[1]] = (20, 100)                 # a smaller pass keeps the larger estimate
    assert not t._blocks_overflowed(ctx, None)
    assert ctx.touched_blocks == 130


def test_backward_without_forward_data_raises():
    t = CheckpointedRollout(None, None, None, 1e-4, 10, checkpoint_every=4)
    with pytest.raises(RuntimeError, match="nothing to differentiate"):
        t.backward()
