"""The multi-rank plumbing of bench.py on CPU: two gloo ranks set up from the
launcher's environment, meet at the barrier, and agree on the maximum of
their timings (the bench reports the slowest rank). The same helpers run
over NCCL when bench.py is launched on GPUs."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench

    w, r, local = bench.dist_setup(None, backend="gloo")
    try:
        bench.rank_barrier(w)
        slowest = bench.rank_max(1.5 * (r + 1), w, "cpu")
        with open(os.path.join(out_dir, f"rank{r}.txt"), "w") as f:
            f.write(f"{w} {r} {local} {slowest}")
        bench.rank_barrier(w)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    for r in range(world):
        w, rank, local, slowest = open(tmp_path / f"rank{r}.txt").read().split()
        assert (int(w), int(rank), int(local)) == (world, r, r)
        assert float(slowest) == pytest.approx(3.0)


def test_one_rank_needs_no_process_group(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench

    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert bench.dist_setup(None) == (1, 0, 0)
    bench.rank_barrier(1)
    assert bench.rank_max(2.5, 1, "cpu") == 2.5


def test_reference_arm_runs_on_rank_zero_only():
    """Under a multi-rank launch the reference arm (the host-core CPU
    implementation) runs on rank 0 alone: another rank exits 0 without work
    or output."""
    import subprocess

    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], env=env, capture_output=True, text=True, timeout=120, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_mix_weighted_plain_rate():
    """The serving leg's plain rate weights the sample's per-kind rates by the
    stream's own work in each kind."""
    sys.path.insert(0, ROOT)
    import bench

    by_kind = {False: {"ps": 100, "ms": 10.0}, True: {"ps": 100, "ms": 100.0}}
    # 900 units of rollouts at 10 per ms, 100 of gradients at 1 per ms: 90 + 100 ms for 1000 units
    rate = bench.mix_weighted_rate(by_kind, {False: 900, True: 100}, "ms")
    assert abs(rate - 1000 / 0.190) < 1e-6
    # a kind the stream has but the sample lacks: no estimate
    assert bench.mix_weighted_rate({False: {"ps": 100, "ms": 10.0}}, {False: 900, True: 100}, "ms") is None
    # a kind the sample has but the stream lacks is ignored
    assert abs(bench.mix_weighted_rate(by_kind, {False: 900, True: 0}, "ms") - 900 / 0.090) < 1e-6
