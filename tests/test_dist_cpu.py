"""The multi-rank host path on CPU (gloo, two ranks): the bench's process
group plumbing (max over ranks, barrier, teardown) and the reference arm
launched the way the multi-GPU bench is launched (torchrun, one process per
rank, rank 0 alone prints the JSON line).  Ranks run the replicas of the
step independently; the only collective is the timing's max."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist()
    try:
        got = d.max(float(10 + rank))
        d.barrier()
    finally:
        d.close()
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as fh:
        json.dump({"world": d.world, "rank": d.rank, "max": got, "backend": d.backend}, fh)


def test_dist_max_over_two_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0, 0]
    res = [json.load(open(tmp_path / f"r{r}.json")) for r in range(2)]
    assert [x["rank"] for x in res] == [0, 1]
    assert all(x["world"] == 2 and x["backend"] == "gloo" and x["max"] == 11.0 for x in res)


@pytest.mark.timeout(300)
def test_reference_arm_under_torchrun():
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus",
           "2", "--config", "cavity", "--steps", "2", "--warmup", "1"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=280, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    out = json.loads(lines[0])
    assert out["impl"] == "reference" and out["n_gpus"] == 2 and out["steps"] == 2 and out["value"] > 0
    assert out["e2e"]["h2d_bytes_per_step"] == 0 and out["cpu_baseline"]["kind"] == "port"
