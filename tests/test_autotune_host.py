"""Autotuner host logic (no GPU): candidate set, workload signature, cache."""
import os

from empm_b200 import autotune as A


def test_candidates_cover_every_launch_option():
    keys = {tuple(sorted(c.items())) for c in A.CANDIDATES}
    assert len(keys) == len(A.CANDIDATES) == 36
    assert {c["sort_every"] for c in A.CANDIDATES} == {8, 16, 32}
    assert {(c["p2g_mode"], c["tile_cap"], c["seg_cap"]) for c in A.CANDIDATES} == {
        (2, 1024, 4), (2, 1024, 8), (1, 512, 4), (1, 1024, 4), (1, 2048, 4)}
    assert {c["g2p_tile"] for c in A.CANDIDATES} == {0, 1}
    # the separate-kernel variant is a candidate wherever fusing applies
    unfused = [c for c in A.CANDIDATES if c["fuse"] == 0]
    assert len(unfused) == 6 and all(c["p2g_mode"] == 2 and c["g2p_tile"] == 0 for c in unfused)
    assert A.DEFAULTS in A.CANDIDATES


def test_apply_fills_options_missing_from_old_cache_entries():
    class T:
        pass

    t = T()
    A._apply(t, dict(sort_every=16, p2g_mode=2, tile_cap=1024, seg_cap=8, g2p_tile=0))
    assert (t.sort_every, t.seg_cap, t.fuse, t.g2p_tile) == (16, 8, True, False)


def test_signature_buckets_particle_counts():
    a = A.signature([96, 48], 100_000, ["plasticine"])
    assert a == A.signature([48, 96], 110_000, ["plasticine", "plasticine"])
    assert a != A.signature([48, 96], 300_000, ["plasticine"])
    assert a != A.signature([48, 64], 100_000, ["plasticine"])


def test_cache_round_trip(tmp_path):
    path = os.path.join(tmp_path, "tune.json")
    entry = {"key": "k1", "options": dict(A.CANDIDATES[3]), "ms": {"x": 1.0}}
    A._store(path, "k1", entry)
    A._MEMORY.pop("k1", None)
    assert A.lookup("k1", path) == entry
    assert A.lookup("missing", path) is None


def test_collider_snapshot_restores_host_state():
    class P:
        def __init__(self):
            self.point = (0.1, 0.2, 0.3)

    class S:
        collider_params = [P()]

    sv = S()
    snap = A._snapshot_colliders([sv])
    sv.collider_params[0].point = (9.0, 9.0, 9.0)
    A._restore_colliders(snap)
    assert sv.collider_params[0].point == (0.1, 0.2, 0.3)
