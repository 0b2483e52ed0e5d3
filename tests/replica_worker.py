"""Worker for tests/test_replicas.py, launched by torchrun with the gloo backend: exercises the
bench's replica plumbing (barrier, max over ranks, whole-job throughput, rank gating of the CPU
reference arm) without a GPU."""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def main():
    out_dir = sys.argv[1]
    dist, rank, ws, local = bench._dist("gloo")
    bench._barrier(dist, "cpu")
    ms_local = 10.0 * (rank + 1)  # the ranks' own timings differ
    ms, value = bench.replica_throughput(dist, ws, 1000, 5, ms_local, "cpu")
    # the CPU reference arm runs on rank 0 only; other ranks return at once without work
    gated = None
    if rank != 0:
        class A:
            workload, steps, warmup, gpus = "32k", 1, 1, ws
        gated = bench.run_reference(A()) is None
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"rank": rank, "ws": ws, "ms": ms, "value": value, "gated": gated}, f)
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
