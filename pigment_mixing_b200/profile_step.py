"""Profiling driver: per-kernel CUDA-event times of the step on a named workload, followed by a
few plain (non-graph) steps that an external profiler can capture.

    python -m pigment_mixing_b200.profile_step [--workload 2m|8m|32k|32m] [--warm 10] [--profile 3] [--plain 3]
"""
import argparse
import json

from . import Simulation, scenes

WORKLOADS = {"2m": scenes.config2, "8m": scenes.config3, "32k": scenes.config1, "32m": scenes.config5}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="2m", choices=sorted(WORKLOADS))
    ap.add_argument("--warm", type=int, default=10, help="steps through advance() first")
    ap.add_argument("--profile", type=int, default=3, help="event-timed steps")
    ap.add_argument("--plain", type=int, default=3, help="plain step() calls at the end")
    ap.add_argument("--set", action="append", default=[], metavar="NAME=VALUE",
                    help="override a scene parameter, e.g. --set perzyna_exp=1")
    a = ap.parse_args()
    sc = WORKLOADS[a.workload]()
    for kv in a.set:
        k, v = kv.split("=", 1)
        sc["params"][k] = float(v)
    sim = Simulation(0)
    scenes.apply(sc, sim)
    sim.prepareSimulation()
    sim.advance(a.warm)
    out = {"workload": a.workload, "particles": len(sc["x"])}
    if a.profile > 0:
        out["kernel_ms"] = sim.profileSteps(a.profile)
    for _ in range(a.plain):
        sim.step()
    out.update(plastic_count=sim.plastic_count, grid_nodes=sim.grid_nodes, error_flags=sim.errorFlags())
    print(json.dumps(out))


if __name__ == "__main__":
    main()
