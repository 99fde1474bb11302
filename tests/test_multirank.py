"""Multi-rank host logic of bench.py on CPU (gloo, world size 2).

The path shards by pairs with no exchange step: every rank builds its own
batch (seeded by its rank), aligns it alone, and only the timing is reduced
(max over ranks).  These tests run that logic on two gloo ranks: the
batches differ between ranks, each rank's results come from its own batch,
the reduction returns the slowest rank's time, and the reference arm runs on
rank 0 only.
"""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    import bench
    import oracle

    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        wl = bench.make_workload("dna_batched", 300, seed_offset=rank)
        sim = oracle.select_matrix(wl.similarity, wl.match, wl.mismatch, wl.ambiguity)
        score, _, _ = oracle.sw_batch(wl.codes, wl.a_off, wl.a_len, wl.b_off, wl.b_len, sim,
                                      wl.gap_init, wl.gap_extend, forward_only=True)
        fake_ms = 10.0 + 5.0 * rank
        slowest = bench.max_over_ranks(dist, fake_ms, "cpu")
        cells = torch.tensor([float(wl.cells)], dtype=torch.float64)
        dist.all_reduce(cells)
        np.savez(os.path.join(out_dir, "rank%d.npz" % rank), score=score, a_len=wl.a_len,
                 slowest=slowest, total_cells=float(cells.item()), cells=float(wl.cells))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce(tmp_path):
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    r0 = np.load(tmp_path / "rank0.npz")
    r1 = np.load(tmp_path / "rank1.npz")
    # each rank aligned its own batch
    assert not np.array_equal(r0["a_len"], r1["a_len"])
    assert r0["score"].shape == r1["score"].shape == (300,)
    # timing is the slowest rank's, on every rank
    assert float(r0["slowest"]) == float(r1["slowest"]) == 15.0
    # whole-job work is the sum of the ranks' work
    assert float(r0["total_cells"]) == float(r0["cells"]) + float(r1["cells"])


def test_reference_arm_under_torchrun_prints_once():
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    if not oracle.have_ssw():
        pytest.skip("reference SSW library not built")
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(REPO, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1",
           "--pairs", "2000"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=300, env=env, cwd=REPO)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0


def test_gpus_flag_launches_ranks_without_torchrun():
    # `bench.py --gpus 2` started as one process re-launches itself through
    # torch.distributed.run (WORLD_SIZE unset): two ranks start, rank 0 alone
    # prints the line and reports the real world size.  The reference arm
    # needs no GPU, so the launch runs here on CPU.
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    if not oracle.have_ssw():
        pytest.skip("reference SSW library not built")
    cmd = [sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "1", "--pairs", "2000"]
    env = {k: v for k, v in os.environ.items()
           if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    env["OMP_NUM_THREADS"] = "2"
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=300, env=env, cwd=REPO)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["config"]["pairs_per_gpu"] == 2000


def test_launcher_builds_a_torchrun_command(monkeypatch):
    # The re-launch keeps every argument and rendezvouses on 127.0.0.1.
    sys.path.insert(0, REPO)
    import bench
    seen = {}

    class Done:
        returncode = 0

    def fake_run(cmd, timeout):
        seen["cmd"] = cmd
        return Done()

    monkeypatch.setattr(bench.subprocess, "run", fake_run)
    args = bench.parse(["--gpus", "4", "--steps", "7"])
    assert bench.launch_ranks(args, ["--gpus", "4", "--steps", "7"]) == 0
    cmd = seen["cmd"]
    i = cmd.index("--nproc-per-node")
    assert cmd[i + 1] == "4"
    assert cmd[cmd.index("--master-addr") + 1] == "127.0.0.1"
    assert cmd[-3:] == ["--gpus", "4", "--steps", "7"][-3:] and "torch.distributed.run" in cmd
