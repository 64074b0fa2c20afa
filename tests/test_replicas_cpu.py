"""The multi-GPU path of bench.py on CPU: the timestep does not shard, so N
GPUs run N replicas, and the ranks only line up the timed region and take
the slowest rank's time.  Here two gloo ranks exercise that plumbing
(lare3d_b200/replicas.py), the reference arm runs under torchrun with two
ranks, and a rank whose peer never joins fails within its timeout."""
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    from lare3d_b200 import replicas
    w, r, _ = replicas.env()
    replicas.init(w, "gloo", timeout_s=60)
    replicas.barrier(w)
    # each rank "timed" a different duration; the job takes the slowest
    m = replicas.max_over_ranks(0.5 + rank, w, "cpu")
    rate = replicas.whole_job_rate(w, 1000.0, m)
    replicas.barrier(w)
    replicas.finish(w)
    with open(os.path.join(out_dir, f"rank{r}.json"), "w") as f:
        json.dump({"rank": r, "ws": w, "max": m, "rate": rate}, f)


def test_two_gloo_ranks_take_the_slowest_time(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    got = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    for g in got:
        assert g["ws"] == 2
        assert g["max"] == 1.5                      # max of 0.5 and 1.5, seen by both ranks
        assert g["rate"] == pytest.approx(2 * 1000.0 / 1.5)


def _lonely_rank(port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK="0", WORLD_SIZE="2", LOCAL_RANK="0")
    sys.path.insert(0, ROOT)
    from lare3d_b200 import replicas
    try:
        replicas.init(2, "gloo", timeout_s=5)
        q.put("joined")
    except Exception as e:  # the peer never arrives: the rendezvous times out
        q.put(type(e).__name__)


def test_rank_whose_peer_never_joins_fails_within_its_timeout():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_lonely_rank, args=(_free_port(), q))
    p.start()
    p.join(120)
    assert not p.is_alive()
    res = q.get(timeout=5)
    assert res != "joined"


def test_reference_arm_under_torchrun_prints_one_line():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "3", "--edge", "12"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1                             # rank 0 alone prints
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
