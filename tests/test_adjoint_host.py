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
