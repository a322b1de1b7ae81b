"""Host-side schedule logic (no GPU): the layered release's outermost active
box per substep, and the bench's launch counts for fused and separate runs."""
import numpy as np

import bench
from empm_b200.mpm_solver_diff import MPMWARPDiff


class _Layers:
    def __init__(self, start, end, n=50):
        self.start_time = start
        self.layer_end_times = [end / n * (i + 1) for i in range(n)]


def test_outermost_release_layer_follows_each_boxs_window():
    """release_particles_sequentially (mpm_solver_diff.py:1146-1171) registers
    50 nested boxes; box i holds its particles while start <= t < end/50*(i+1).
    The one modifier that replaces them applies where a particle lies in the
    outermost box still active: the smallest active index."""
    p = _Layers(0.0, 0.006)
    f32 = np.float32
    assert MPMWARPDiff._outermost_layer(f32(0.0), p) == 0
    assert MPMWARPDiff._outermost_layer(f32(0.006 / 50 * 0.5), p) == 0
    assert MPMWARPDiff._outermost_layer(f32(0.006 / 50 * 1.5), p) == 1
    assert MPMWARPDiff._outermost_layer(f32(0.006 / 50 * 49.5), p) == 49
    assert MPMWARPDiff._outermost_layer(f32(0.0061), p) == -1          # every box released
    q = _Layers(0.002, 0.006)
    assert MPMWARPDiff._outermost_layer(f32(0.001), q) == -1           # before the start


def test_layered_threshold_matches_the_union_of_the_boxes():
    """A particle inside boxes 0..k (k + 1 boxes, nested) is held by box i
    exactly when i <= k; the union over the active boxes i >= i_min holds it
    exactly when its count k + 1 >= i_min + 1, the threshold the kernel uses."""
    rng = np.random.default_rng(0)
    counts = rng.integers(0, 51, 1000)          # boxes holding each particle
    for i_min in (0, 1, 7, 49):
        union = np.array([any(i <= c - 1 for i in range(i_min, 50)) for c in counts])
        assert np.array_equal(union, counts >= i_min + 1)


def test_bench_launch_counts_fused_and_separate():
    # one 300-substep rollout in 50-substep blocks, sort every 32, resumed blocks
    sep = bench.rollout_launches(300, 50, 32, True, fused=False)
    fus = bench.rollout_launches(300, 50, 32, True, fused=True)
    assert sep == 4 * 300 + 4 * 10 + 1         # P2G, block list, grid update, G2P per substep; 10 sorts; write-back
    # a run of k substeps launches k + 1 particle kernels instead of 2 k
    runs = [32, 18, 14, 32, 4, 28, 22, 10, 32, 8, 24, 26, 6, 32, 12]
    assert sum(runs) == 300
    assert sep - fus == sum(2 * k - (k + 1 if k >= 2 else 2 * k) for k in runs)
    assert bench.rollout_launches(300, 50, 0, True) == 4 * 300   # direct path
