"""The N > 1 plumbing on the CPU: two gloo ranks exercise the replica helpers
the benchmark uses on NCCL (max of the timed interval over ranks, per-rank
seeds, the ensemble split), and a two-rank torchrun of the reference arm
checks that exactly one rank reports."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, out_dir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(ws), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    from paratc_b200 import replicas
    dist = replicas.init("gloo", timeout_s=60)
    res = {
        "env": list(replicas.dist_env()),
        "max": replicas.max_over_ranks(10.0 * (rank + 1), dist),
        "sum": replicas.sum_over_ranks(rank + 1, dist),
        "seed": replicas.replica_seed(1234, rank),
        "share": replicas.ensemble_share(32, ws, rank),
    }
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, "rank%d.json" % rank), "w") as f:
        json.dump(res, f)


def test_replica_helpers_two_gloo_ranks(tmp_path):
    ws = 2
    mp.start_processes(_worker, args=(ws, _free_port(), str(tmp_path)), nprocs=ws, join=True, start_method="spawn")
    res = [json.load(open(tmp_path / ("rank%d.json" % r))) for r in range(ws)]
    for r in range(ws):
        assert res[r]["env"] == [ws, r, r]
        assert res[r]["max"] == 20.0          # the job's time is the slowest rank's
        assert res[r]["sum"] == 3.0
    assert res[0]["seed"] != res[1]["seed"]  # independent replicas
    share = res[0]["share"] + res[1]["share"]
    assert sorted(share) == list(range(32)) and len(set(res[0]["share"]) & set(res[1]["share"])) == 0


def test_reference_arm_reports_once_under_torchrun():
    env = dict(os.environ)
    env.pop("CUDA_VISIBLE_DEVICES", None)
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "grid-point substeps/s"
    assert d["e2e"]["h2d_bytes_per_step"] == 0
