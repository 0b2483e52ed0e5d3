"""Multi-process replica path of bench.py on CPU (gloo, world size 2): the job time is the
slowest rank's, the throughput sums the ranks' work, and the CPU reference arm runs on rank 0 only."""
import json
import os
import socket
import subprocess
import sys

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_two_gloo_replicas(tmp_path):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "tests", "replica_worker.py"), str(tmp_path)]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=240)
    assert r.returncode == 0, r.stderr[-3000:]
    res = [json.load(open(os.path.join(tmp_path, f"rank{k}.json"))) for k in range(2)]
    for d in res:
        assert d["ws"] == 2
        assert d["ms"] == 20.0                       # max over ranks of 10 and 20 ms
        assert abs(d["value"] - 2 * 1000 * 5 / 0.020) < 1e-6
    assert res[1]["gated"] is True
