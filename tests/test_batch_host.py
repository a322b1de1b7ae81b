"""Host-side logic of the batched engine (no GPU): the flags of each graph
block of a rollout."""
from empm_b200 import _native as N
from empm_b200.batch import block_flags


def _plan(n_steps, block, use_graph=True, resume=True):
    out, done = [], 0
    while done < n_steps:
        k = min(block, n_steps - done)
        out.append(block_flags(done, k, n_steps, use_graph, resume))
        done += k
    return out


def test_blocks_resume_and_keep_except_at_the_ends():
    G, R, K = N.ROLLOUT_GRAPH, N.ROLLOUT_RESUME, N.ROLLOUT_KEEP
    assert _plan(300, 50) == [G | K] + [G | R | K] * 4 + [G | R]
    assert _plan(120, 50) == [G | K, G | R | K, G | R]
    assert _plan(50, 50) == [G]                       # one block: sort in, write back
    assert _plan(30, 50) == [G]


def test_without_resume_every_block_sorts_and_writes_back():
    assert _plan(300, 50, resume=False) == [N.ROLLOUT_GRAPH] * 6
    assert _plan(120, 50, use_graph=False, resume=False) == [0, 0, 0]
    assert _plan(120, 50, use_graph=False) == [N.ROLLOUT_KEEP, N.ROLLOUT_RESUME | N.ROLLOUT_KEEP, N.ROLLOUT_RESUME]
