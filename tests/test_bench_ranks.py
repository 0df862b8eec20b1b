"""The multi-rank host logic of bench.py on CPU: two gloo ranks on 127.0.0.1.

bench.py runs one process per GPU (replicas: frames are independent, no
collective on the data path). The only cross-rank steps are the barriers around
the timed region and the maximum of the per-rank times; the reported value is
all ranks' frames over the slowest rank's time. The reference arm runs on rank
0 alone and the other ranks exit without work.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out_dir):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # Rank r "took" (10 + r) ms for the headline pass and (20 - r) ms with stage events.
        dist.barrier()
        got = bench.max_over_ranks([10.0 + rank, 20.0 - rank], ws)
        dist.barrier()
        value = bench.whole_job_us_per_frame(got[0], 50, ws)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"max": got, "value": value}, f)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_value_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    ws, port = 2, _free_port()
    mp.start_processes(_rank_main, args=(ws, port, str(tmp_path)), nprocs=ws, join=True, start_method="spawn")
    results = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(ws)]
    for r in results:
        # Every rank sees the maximum of each entry, not its own time.
        assert r["max"] == [11.0, 20.0]
        # 2 ranks x 50 frames in the slowest rank's 11 ms.
        assert r["value"] == pytest.approx(11.0 * 1e3 / 100)


def test_max_over_ranks_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks([3, 4.5], 1) == [3.0, 4.5]
    assert bench.whole_job_us_per_frame(2.0, 10, 1) == pytest.approx(200.0)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
