#!/usr/bin/env python
"""Throughput of the paint-mixing MPM step (particle-steps/s) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload 2m|8m|32k]

Workload (default "2m"): two 64x64x32-cell paint blocks at dx = 1/256 (2,097,152 particles,
8 jittered particles per cell, seeded), von Mises / Herschel-Bulkley viscoplastic paint
(yield 100 Pa, 10 Pa s^0.6), box knife on a seeded 3-segment path at 0.5 units/s, floor plate,
MUSL, FP32 transfers with FP64 SVD/return map.  A "step" is one MPM time step of that scene.

``value`` is device-timed (CUDA events on the library's stream, state resident in HBM);
``e2e`` is the same metric through the C ABI from pinned host buffers: scene upload, prepare,
K steps with the particle readback at every finished frame (the render loop's idiom), and the
final readback, timed on the host clock.  Multi-GPU runs are independent replicas (one scene per
GPU, no collective on the data path): value sums over ranks, time is the max over ranks.
``--impl reference`` times the CPU restatement of the reference step (the oracle, float,
-O3 -ffast-math -fopenmp, all host threads) on the same scene.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s"
# Algorithmic bytes per unit of work (per particle, per active grid node) of each kernel: the
# compulsory SoA particle traffic and grid traffic of the reference step structure.
ALGO_BYTES = {
    "k_p2g": (128.0, 48.0),          # read x,v,B,latent,diffusion,tau ; accumulate m,mv,f,latent,shear
    "k_g2p_musl": (144.0, 108.0),    # read x,v,latent + write v,B,latent,diff,pic ; read grid + MUSL grid
    # the deformation update runs as two kernels; their 72 B of F_trial round trip are not in
    # the reference's step structure, so they are not algorithmic bytes
    "k_defgrad_head": (36.0, 12.0),  # read x,pic + write x ; read MUSL velocity
    "k_defgrad_tail": (100.0, 0.0),  # read F,plastic + write F,plastic
    "k_grid_update": (0.0, 40.0),    # read 16 B, write v and flip 24 B per node
    "k_clear_bricks": (0.0, 80.0),   # zero the accumulated and MUSL records of touched bricks
}
STEP_BYTES = (408.0, 256.0)          # whole step: 408 B per particle + 256 B per active node


def _workload(name: str):
    from pigment_mixing_b200 import scenes
    if name == "2m":
        return scenes.config2(seed=0)
    if name == "8m":
        return scenes.config3(seed=0)
    if name == "32k":
        return scenes.config1(seed=0)
    if name == "32m":
        return scenes.config5(seed=0)
    if name == "262k":  # the same scene at dx = 1/128: the small case for profiler captures
        return scenes.two_block_scene(1.0 / 128, (32, 32, 16), seed=0, steps=1000)
    raise SystemExit(f"unknown workload {name}")


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
        except Exception:
            pass
        finally:
            if self.path and os.path.exists(self.path):
                os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def _dist(backend: str = "nccl"):
    """(process group or None, rank, world size, local rank) from the torchrun environment.
    Replicas: the group carries only the barrier and the max-over-ranks of the timings."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return None, 0, 1, 0
    import torch.distributed as dist
    from datetime import timedelta
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist.init_process_group(backend, timeout=timedelta(seconds=600))
    return dist, rank, ws, local


def _coll_device(dist, device):
    """Where collective tensors live: the GPU for NCCL, the host for gloo."""
    return device if dist is not None and dist.get_backend() == "nccl" else "cpu"


def _max_over_ranks(dist, x: float, device) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=_coll_device(dist, device))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(dist, device):
    if dist is not None:
        import torch
        t = torch.zeros(1, device=_coll_device(dist, device))
        dist.all_reduce(t)
        if t.is_cuda:
            torch.cuda.synchronize(device)


def replica_throughput(dist, ws: int, units_per_rank: int, steps: int, ms_local: float, device) -> tuple:
    """Whole-job throughput of N independent replicas: every rank processed units_per_rank x steps
    units; the job took the slowest rank's time.  Returns (max ms over ranks, units per second)."""
    ms = _max_over_ranks(dist, ms_local, device)
    return ms, ws * units_per_rank * steps / (ms / 1e3)


def cpu_baseline(scene, budget_s: float = 25.0, max_steps: int = 20):
    """The oracle (float, -O3 -ffast-math -fopenmp, all host threads) on the same scene."""
    from oracle.oracle import OracleSim
    from pigment_mixing_b200 import scenes
    cores = os.cpu_count() or 1
    o = OracleSim(32, fast=True)
    o.set(n_threads=cores)
    scenes.apply(scene, o)
    o.prepare()
    t0 = time.perf_counter()
    o.advance(1)  # first step allocates
    first = time.perf_counter() - t0
    n = int(max(1, min(max_steps, budget_s / max(first, 1e-3))))
    t0 = time.perf_counter()
    o.advance(n)
    el = time.perf_counter() - t0
    npart = len(scene["x"])
    return {"value": npart * n / el, "unit": METRIC, "cores": cores, "kind": "port",
            "sample": f"{n} full steps of the {npart}-particle scene after 1 warm-up step "
                      f"(CPU restatement of the reference step, float, OpenMP)", "seconds": el}


def _err_stats(a, b):
    d = np.linalg.norm(np.asarray(a, np.float64).reshape(len(a), -1) - np.asarray(b, np.float64).reshape(len(b), -1),
                       axis=1)
    return {"max": float(d.max()), "p99": float(np.percentile(d, 99))}


def accuracy_vs_oracle(scene, steps=50, surrogate_params=None, device=0):
    """Error of the GPU path against the FP64 oracle (the checker) on the same seeded scene after
    ``steps`` steps: per-particle |dx| / domain size, |dv|, |d latent| (max and p99), total mass
    and momentum, mass-weighted mean latent."""
    from oracle.oracle import OracleSim
    from pigment_mixing_b200 import RETURN_MAP_SURROGATE, Simulation, scenes
    o = OracleSim(64)
    o.set(n_threads=os.cpu_count() or 1)
    scenes.apply(scene, o)
    o.prepare()
    o.advance(steps)
    po = o.particles_f64()
    out = {"scene": f"{scene['name']}: {len(scene['x'])} particles", "steps": steps, "domain_size": 1.0}
    forms = [("plain", None)] + ([("surrogate", surrogate_params)] if surrogate_params is not None else [])
    mp = scene["params"]["particle_mass"]
    for name, params in forms:
        g = Simulation(device)
        scenes.apply(scene, g)
        if params is not None:
            g.setSurrogate(params)
            g.setReturnMap(RETURN_MAP_SURROGATE)
        g.prepareSimulation()
        g.advance(steps)
        pg = g.getParticles(fields=("x", "v", "latent"))
        st = g.stats()
        g.close()
        mom_o = mp * po["v"].sum(0)
        out[name] = {"position": _err_stats(pg.x, po["x"]), "velocity": _err_stats(pg.v, po["v"]),
                     "latent": _err_stats(pg.latent, po["latent"]),
                     "mass_rel": abs(st["mass"] - mp * len(scene["x"])) / (mp * len(scene["x"])),
                     "momentum_abs": float(np.abs(st["momentum"] - mom_o).max()),
                     "momentum_scale": float(np.abs(mom_o).max()),
                     "mean_latent_abs": float(np.abs(st["mean_latent"] - po["latent"].mean(0)).max())}
    return out


def drift(scene, steps, device=0):
    """Mass and mass-weighted mean latent of the GPU path at step 0 and after ``steps`` steps."""
    from pigment_mixing_b200 import Simulation, scenes
    g = Simulation(device)
    scenes.apply(scene, g)
    g.prepareSimulation()
    s0 = g.stats()
    import torch
    stream = torch.cuda.ExternalStream(g.stream(), device=device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    seg = max(1, steps // 10)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range((steps + seg - 1) // seg + 1)]
    torch.cuda.synchronize(device)
    ev[0].record(stream)
    done = 0
    seg_state = []
    for j in range(1, len(ev)):
        k = min(seg, steps - done)
        g.advance(k)
        done += k
        ev[j].record(stream)
        rm = g.returnMapStats()  # the last step of the segment (waits for it)
        seg_state.append({"plastic": int(g.plastic_count), "newton_solves": rm["solves"],
                          "newton_updates": rm["newton_iters"], "grid_nodes": int(g.grid_nodes)})
    torch.cuda.synchronize(device)
    ms = ev[0].elapsed_time(ev[-1])
    seg_ms = [ev[j - 1].elapsed_time(ev[j]) / seg for j in range(1, len(ev))]
    late = {k: round(v * 1e3, 1) for k, v in g.profileSteps(5).items()}  # us per kernel, after the run
    s1 = g.stats()
    flags = g.errorFlags()
    nodes = int(g.grid_nodes)
    regrow = {"count": int(g.regrowths), "host_ms": float(g.regrow_ms),
              "capacity_nodes_end": int(g.grid_capacity_nodes)}
    g.close()
    return {"steps": steps, "ms_per_step_avg": ms / steps, "ms_per_step_by_segment": seg_ms,
            "state_by_segment": seg_state, "kernel_us_after_run": late,
            "particle_steps_per_s": len(scene["x"]) * steps / (ms / 1e3),
            "mass_rel": abs(s1["mass"] - s0["mass"]) / s0["mass"],
            "mean_latent_abs": float(np.abs(s1["mean_latent"] - s0["mean_latent"]).max()),
            "momentum_step_end": [float(v) for v in s1["momentum"]], "n_active_end": int(s1["n_active"]),
            "grid_nodes_end": nodes, "grid_regrowth": regrow, "error_flags": int(flags)}


def run_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return  # replicas: rank 0 alone times the CPU path
    scene = _workload(args.workload)
    b = cpu_baseline(scene, budget_s=max(10.0, min(120.0, 3.0 * args.steps)), max_steps=max(1, args.steps))
    line = {"impl": "reference", "metric": METRIC, "value": b["value"], "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": len(scene["x"]) / b["value"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": _config(scene, args),
            "cpu_baseline": {k: b[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": b["value"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


_BLOCKS = {"2m": "two 64x64x32-cell blocks", "32k": "two 16x16x8-cell blocks",
           "8m": "four 64^3-cell blocks of four pigments", "32m": "six 87^3-cell blocks (3 x 2) of six pigments"}
_PATH = {"2m": "a 3-segment path", "32k": "a 3-segment path", "8m": "a 3-segment path",
         "32m": "four back-and-forth strokes"}


def _config(scene, args):
    n = len(scene["x"])
    return {"workload": f"{scene['name']}: {n} particles, dx={scene['params']['dx']:.6g}, "
                        f"{_BLOCKS[args.workload]}, VMVisc (Herschel-Bulkley) paint, box knife 0.4x0.2x0.01 on "
                        f"{_PATH[args.workload]} at 0.5 u/s, MUSL, APIC",
            "particles": n, "return_map": args.return_map,
            "precision": "FP32 transfers, grid and VMVisc return map; FP64 SVD of the elastic F",
            "l2": f"inputs larger than L2 (particle state {n * 168 / 1e9:.2f} GB per buffer, L2 126 MB)",
            "parallelism": f"replicas x{args.gpus}"}


def run_ours(args):
    import torch
    from pigment_mixing_b200 import Simulation, scenes
    dist, rank, ws, local = _dist()
    device = local
    torch.cuda.set_device(device)
    scene = _workload(args.workload)
    npart = len(scene["x"])
    sim = Simulation(device)
    scenes.apply(scene, sim)
    sim.prepareSimulation()
    sim.advance(args.warmup)
    stream = torch.cuda.ExternalStream(sim.stream(), device=device)
    # -------- timed region: K steps, state resident in HBM --------
    with ClockSampler(device) as clk:
        _barrier(dist, device)
        torch.cuda.synchronize(device)
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        sim.advance(args.steps)
        ev1.record(stream)
        torch.cuda.synchronize(device)
        ms = ev0.elapsed_time(ev1)
        _barrier(dist, device)
    clocks = clk.summary()
    flags = sim.errorFlags()
    ref = sim.getParticles(fields=("x", "latent"))
    x_ref, lat_ref = ref.x, ref.latent
    newton_plain = _newton_per_solve(sim, 4)
    ms_max, value = replica_throughput(dist, ws, npart, args.steps, ms, device)
    # -------- per-kernel times (CUDA events on the same stream, separate steps) --------
    g = sim.grid()
    active_nodes = int((g["mass"] > 0).sum())
    kps = int(sim.kernels_per_step)
    sim.close()
    # per-kernel times over the same steps as the timed region: a fresh simulation of the scene
    # after the same warm-up, every kernel of its K steps timed with CUDA events on its stream
    prof = Simulation(device)
    scenes.apply(scene, prof)
    prof.prepareSimulation()
    prof.advance(args.warmup)
    kms = prof.profileSteps(args.steps)
    prof.close()
    dom = max((k for k in kms if k in ALGO_BYTES), key=lambda k: kms[k])
    peak, peak_kind = _peaks()
    pb, nb = ALGO_BYTES[dom]
    algo = pb * npart + nb * active_nodes
    achieved = algo / (kms[dom] / 1e3) / 1e9
    traffic = _ncu_traffic(dom) if args.workload == "2m" else None
    step_ms = ms_max / args.steps
    step_bytes = STEP_BYTES[0] * npart + STEP_BYTES[1] * active_nodes
    roof = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic, "algorithmic_bytes": algo,
            "peak_source": ("measured copy bandwidth (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                            else "fallback copy bandwidth 6650 GB/s (MEASURED_PEAKS.json absent)")}
    step_roof = {"bytes": step_bytes, "achieved": step_bytes / (step_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                 "frac": step_bytes / (step_ms / 1e3) / 1e9 / peak, "active_nodes": active_nodes}
    roof["timed_over"] = f"the {args.steps} steps after {args.warmup} warm-up steps (a second run of the timed steps)"
    sur = None
    if not args.no_surrogate:
        sur = _surrogate_leg(scene, args, device, dist, ws, value, x_ref, lat_ref, newton_plain)
    splat = None
    if not args.no_splat:
        splat = _splat_leg(scene, args, device, dist, rank == 0 and ws == 1 and not args.no_cpu)
    batch = None
    if not args.no_batch:
        batch = _batch_leg(args, device, dist, ws)
        if sur is not None:
            batch["surrogate"] = _batch_leg(args, device, dist, ws, sur["_params"])
    # -------- end to end through the C ABI from pinned host buffers --------
    _e2e(scene, args, device, dist, ws)  # untimed pass: first-use costs of the API path (allocator, streams)
    # three timed passes, the median reported: one pass is about a tenth of a second of host and
    # device work, so the host's own noise (page faults, other tenants) moves single passes
    runs = sorted((_e2e(scene, args, device, dist, ws) for _ in range(3)), key=lambda r: r["value"])
    e2e = dict(runs[1])
    e2e["passes"] = [r["value"] for r in runs]
    e2e["passes_host_ms"] = [r.pop("host_ms") for r in runs]
    e2e.pop("host_ms", None)
    e2e["includes"] += "; median of three timed passes"
    if rank == 0:
        e2e["breakdown"] = _e2e_breakdown(scene, args, device)
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": _config(scene, args),
            "roofline": roof, "step_roofline": step_roof, "e2e": e2e, "clocks": clocks,
            "gpu_launches": args.steps * kps,
            "kernel_ms": kms, "error_flags": flags}
    sur_params = None
    if sur is not None:
        sur_params = sur.pop("_params")
        line["surrogate"] = sur
    if rank == 0 and ws == 1 and args.workload == "2m" and not args.no_big:
        line["point_8m"] = _big_point(args, device, sur_params)
    if batch is not None:
        line["batch"] = batch
    if splat is not None:
        line["splat"] = splat
    if args.drift_steps > 0:
        line["drift"] = drift(scene, args.drift_steps, device)
        d = line["drift"]
        line["full_run"] = {"steps": d["steps"], "value": d["particle_steps_per_s"], "unit": METRIC,
                            "ms_per_step": d["ms_per_step_avg"],
                            "note": "the workload's full step count from a fresh start (drift leg); the plastic "
                                    "particle count and Newton updates per solve grow as the knife works the paint"}
    if rank == 0 and ws == 1 and not args.no_cpu:
        line["cpu_baseline"] = {k: v for k, v in cpu_baseline(scene).items() if k != "seconds"}
        # the FP64 oracle as checker: 50-step error on the 32,768-particle scene of the same recipe
        line["accuracy"] = accuracy_vs_oracle(_workload("32k"), 50, _small_surrogate(device), device)
        if args.workload == "2m" and not args.no_accuracy_2m:
            # the headline scene itself: 50 steps of the FP64 oracle (all host threads) as the checker
            line["accuracy_2m"] = accuracy_vs_oracle(scene, 50, sur_params, device)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def _ncu_traffic(kernel):
    """dram__bytes_read.sum + dram__bytes_write.sum per launch of ``kernel`` from the committed ncu
    summary of the 2M scene (line ``traffic_bytes_per_launch: name=bytes ...``)."""
    path = os.path.join(ROOT, "profiles", "dram_traffic_transfer_kernels_2m.md")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_launch:"):
                    for kv in line.split(":", 1)[1].split():
                        k, v = kv.split("=")
                        if k == kernel:
                            return float(v)
    except OSError:
        pass
    return None


def _newton_per_solve(sim, steps):
    it = sv = acc = 0
    for _ in range(steps):
        sim.advance(1)
        st = sim.returnMapStats()
        it += st["newton_iters"]
        sv += st["solves"]
        acc += st["accepted"]
    return {"updates_per_solve": it / max(sv, 1), "solves": sv, "accepted_fraction": acc / max(sv, 1)}


def _surrogate_leg(scene, args, device, dist, ws, plain_value, x_ref, lat_ref, newton_plain):
    """Surrogate + FP32 form: samples logged by the plain solver on this workload, GPU training,
    then the same warm-up + timed steps with the learned return map."""
    import torch
    from pigment_mixing_b200 import RETURN_MAP_SURROGATE, Simulation, scenes, surrogate
    npart = len(scene["x"])
    log = Simulation(device)
    scenes.apply(scene, log)
    every = max(1, int(round(npart * args.log_steps / 4e6)))  # about 4M samples spread over the logged steps
    log.set(sample_log_every=every)
    log.enableSampleLog(6 << 20)
    log.prepareSimulation()
    log.advance(args.log_steps)
    xs, ys = log.samples()
    log.close()
    t0 = time.perf_counter()
    params, hist = surrogate.train(xs, ys, epochs=args.train_epochs, batch=8192, lr=3e-3, seed=0)
    train_s = time.perf_counter() - t0
    s = Simulation(device)
    scenes.apply(scene, s)
    s.setSurrogate(params)
    s.setReturnMap(RETURN_MAP_SURROGATE)
    s.prepareSimulation()
    s.advance(args.warmup)
    stream = torch.cuda.ExternalStream(s.stream(), device=device)
    _barrier(dist, device)
    torch.cuda.synchronize(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s.advance(args.steps)
    e1.record(stream)
    torch.cuda.synchronize(device)
    ms = _max_over_ranks(dist, e0.elapsed_time(e1), device)
    value = ws * npart * args.steps / (ms / 1e3)
    p = s.getParticles(fields=("x", "latent"))
    dx = float(np.abs(p.x.astype(np.float64) - x_ref).max())
    dl = float(np.abs(p.latent.astype(np.float64) - lat_ref).max())
    newton_sur = _newton_per_solve(s, 4)
    kms = s.profileSteps(3)
    s.close()
    st = _rm_stats_after(scene, params, device)
    return {"_params": params, "value": value, "unit": METRIC, "ms_per_step": ms / args.steps,
            "speedup_vs_plain": value / plain_value, "acceptance": st,
            "train": {"samples": int(len(xs)), "logged_steps": args.log_steps, "log_every": every, "epochs": args.train_epochs,
                      "seconds": train_s, "loss_first_epoch": float(hist[0]), "loss_last_epoch": float(hist[-1])},
            "newton": {"plain": newton_plain, "surrogate": newton_sur},
            "max_position_diff_vs_plain": dx, "max_latent_diff_vs_plain": dl,
            "kernel_ms": {k: kms[k] for k in ("k_defgrad_head", "k_defgrad_tail", "k_mlp_infer", "k_sur_finish")
                          if k in kms}}


def _rm_stats_after(scene, params, device, steps=10):
    """Return-map statistics of the surrogate form after a few steps of the scene: particles sent to
    the network, estimates that passed the consistency check, and the fallback rate."""
    from pigment_mixing_b200 import RETURN_MAP_SURROGATE, Simulation, scenes
    s = Simulation(device)
    scenes.apply(scene, s)
    s.setSurrogate(params)
    s.setReturnMap(RETURN_MAP_SURROGATE)
    s.prepareSimulation()
    s.advance(steps)
    st = s.returnMapStats()
    s.close()
    return {"after_steps": steps, "queued": st["queued"], "accepted": st["accepted"],
            "fallback_rate": 1.0 - st["accepted"] / max(1, st["queued"]),
            "newton_updates": st["newton_iters"], "solves": st["solves"]}


def _small_surrogate(device):
    """Surrogate trained on the 32,768-particle scene's own logged samples (60 plain steps)."""
    from pigment_mixing_b200 import Simulation, scenes, surrogate
    log = Simulation(device)
    scenes.apply(_workload("32k"), log)
    log.enableSampleLog(1 << 22)
    log.prepareSimulation()
    log.advance(60)
    xs, ys = log.samples()
    log.close()
    params, _ = surrogate.train(xs, ys, epochs=20, batch=4096, lr=3e-3, seed=0)
    return params


def _batch_leg(args, device, dist, ws, params=None):
    """The batched workload: args.batch_scenes independent palette scenes (particle counts
    log-uniform 20k-400k, grids 64^3-160^3, random pigment pair, yield and knife path) stepped
    together through pm_batch (autotuned launch shapes, one CUDA graph per round), against the
    same scenes advanced one after another through the single-scene API.  With params, every
    scene runs the learned return map (the surrogate form)."""
    import torch
    from pigment_mixing_b200 import RETURN_MAP_SURROGATE, Batch, Simulation, scenes
    scs = scenes.batch_scenes(args.batch_scenes, seed=0)
    npart = sum(len(sc["x"]) for sc in scs)

    def make():
        out = []
        for sc in scs:
            g = Simulation(device)
            scenes.apply(sc, g)
            if params is not None:
                g.setSurrogate(params)
                g.setReturnMap(RETURN_MAP_SURROGATE)
            g.prepareSimulation()
            out.append(g)
        return out

    sims = make()
    b = Batch(sims)
    t0 = time.perf_counter()
    tuning, tuned_ms = b.autotune(trial_rounds=6)
    tune_s = time.perf_counter() - t0
    b.step(args.warmup)
    pre_steps = min(g.steps_done for g in sims)  # the sequential run is timed at the same steps
    stream = torch.cuda.ExternalStream(b.stream(), device=device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    _barrier(dist, device)
    torch.cuda.synchronize(device)
    e0.record(stream)
    b.step(args.batch_steps)
    e1.record(stream)
    torch.cuda.synchronize(device)
    ms = _max_over_ranks(dist, e0.elapsed_time(e1), device)
    value = ws * npart * args.batch_steps / (ms / 1e3)
    prof = b.profile(3)
    steps = sorted({g.steps_done for g in sims})
    flags = int(np.bitwise_or.reduce([g.errorFlags() for g in sims]))
    b.close()
    for g in sims:
        g.close()
    # the same scenes, one after another through pm_advance (each synchronises at its end), timed
    # over the same steps of the scenes as the batch (scenes get heavier as the knife works them)
    seq = make()
    for g in seq:
        g.advance(pre_steps)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    for g in seq:
        g.advance(args.batch_steps)
    torch.cuda.synchronize(device)
    seq_s = time.perf_counter() - t0
    for g in seq:
        g.close()
    seq_value = ws * npart * args.batch_steps / seq_s
    counts = [len(sc["x"]) for sc in scs]
    grids = [int(round(1.0 / sc["params"]["dx"])) for sc in scs]
    kernel_sum = sum(prof.values())
    return {"value": value, "unit": METRIC, "form": "surrogate" if params is not None else "plain",
            "scenes": len(scs), "particles": npart,
            "particles_min_max": [min(counts), max(counts)], "grid_min_max": [min(grids), max(grids)],
            "rounds": args.batch_steps, "ms_per_round": ms / args.batch_steps,
            "kernel_ms_sum_per_round": kernel_sum,
            "launch_gaps_ms_per_round": ms / args.batch_steps - kernel_sum,
            "tuning": tuning,
            "autotune_ms_per_round": tuned_ms, "autotune_seconds": tune_s,
            "sequential_value": seq_value, "speedup_vs_sequential": value / seq_value,
            "timed_steps": [pre_steps, pre_steps + args.batch_steps],
            "steps_after": steps, "error_flags": flags, "kernel_ms": prof,
            "workload": "palette scenes: 2 blocks each, random pigment pair of 6 RGB seeds, yield U(50,200) Pa, "
                        "random 3-segment knife path, VMVisc, MUSL, APIC"}


def _splat_leg(scene, args, device, dist, with_cpu: bool):
    """Headless pigment volume splat (the renderer's two-pass bilateral splat) of the workload
    after its warm-up steps: device time of pm_splat_pigments into a device buffer; beside it the
    numpy restatement (the checker) on a sample of the particles."""
    import torch
    from pigment_mixing_b200 import Simulation, scenes
    g = Simulation(device)
    scenes.apply(scene, g)
    g.prepareSimulation()
    g.advance(args.warmup)
    vox0, origin, vs = g.splatPigments(0.5, 0.2)
    out = torch.empty(vox0.shape, dtype=torch.float32, device=f"cuda:{device}")
    stream = torch.cuda.ExternalStream(g.stream(), device=device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g.splatPigments(0.5, 0.2, out=out)  # warm-up
    torch.cuda.synchronize(device)
    reps = 5
    e0.record(stream)
    for _ in range(reps):
        g.splatPigments(0.5, 0.2, out=out)
    e1.record(stream)
    torch.cuda.synchronize(device)
    ms = _max_over_ranks(dist, e0.elapsed_time(e1) / reps, device)
    n = len(scene["x"])
    res = {"particles": n, "voxels": int(np.prod(vox0.shape[:3])), "voxel_size": vs, "ms": ms,
           "particles_per_s": n / (ms / 1e3), "sigma_spatial": 0.5, "sigma_color": 0.2,
           "includes": "both passes and normalisations into a device buffer (scratch grids kept between calls); "
                       "no host copy"}
    # the renderer's per-frame preprocessing before the splat: binary density grid, anisotropy
    # matrices and densities, then the splat with those matrices (all device outputs)
    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize(device)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.synchronize(device)
        return _max_over_ranks(dist, a.elapsed_time(b) / reps, device)
    bdg = g.densityGrid(device=True)
    an = g.anisotropy(device=True)
    res["density_grid"] = {"ms": timed(lambda: g.densityGrid(device=True)),
                           "voxels": int(np.prod(bdg["dims"])), "occupied": bdg["occupancy"][1],
                           "includes": "binning, filter, occupancy and its 2^3 / 4^3 ORs into device buffers"}
    ams = timed(lambda: g.anisotropy(device=True))
    res["anisotropy"] = {"ms": ams, "particles_per_s": n / (ams / 1e3), "n_aggregate": an["n_aggregate"],
                         "includes": "binning, per-particle matrices, inverses, determinants and densities "
                                     "into device buffers"}
    res["splat_anisotropic_ms"] = timed(lambda: g.splatPigments(0.5, 0.2, G=an["G"], out=out))
    if with_cpu:
        from oracle import splat_ref
        st = g.getParticles(fields=("x", "latent"))
        lo, hi = g.getGridBoundaries()
        k = min(n, 50000)
        t0 = time.perf_counter()
        splat_ref.splat(st.x[:k], st.latent[:k], lo, hi, scene["params"]["dx"], 0.5, 0.2)
        el = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": k / el, "unit": "particles/s", "cores": 1, "kind": "port",
                               "sample": f"first {k} particles, numpy restatement of both passes"}
        from oracle import density_ref
        # a compact piece of the body: the particles within 4 dx of the centre of mass
        dxs = scene["params"]["dx"]
        sel = np.all(np.abs(st.x - st.x.mean(0)) < 4 * dxs, axis=1)
        t0 = time.perf_counter()
        density_ref.anisotropy(st.x[sel], lo, hi, dxs)
        el = time.perf_counter() - t0
        res["anisotropy"]["cpu_baseline"] = {"value": int(sel.sum()) / el, "unit": "particles/s", "cores": 1,
                                             "kind": "port", "sample": f"{int(sel.sum())} particles within 4 dx of "
                                             "the centre of mass, numpy restatement"}
    g.close()
    return res


def _e2e(scene, args, device, dist, ws):
    import torch
    from pigment_mixing_b200 import Simulation, scenes
    n = len(scene["x"])
    hx = torch.from_numpy(np.ascontiguousarray(scene["x"], np.float32)).pin_memory()
    hl = torch.from_numpy(np.ascontiguousarray(scene["latent"], np.float32)).pin_memory()
    ox = torch.empty((n, 3), dtype=torch.float32).pin_memory()
    ol = torch.empty((n, 7), dtype=torch.float32).pin_memory()
    od = torch.empty((n,), dtype=torch.float32).pin_memory()
    _barrier(dist, device)
    t0 = time.perf_counter()
    marks = [t0]  # host clock after each call (no added synchronisation)
    sim = Simulation(device)
    sim.setParticles(hx.numpy(), hl.numpy())
    marks.append(time.perf_counter())
    sim.set(**scene["params"])
    for k, v in scene["vectors"].items():
        setattr(sim, k, v)
    for kind, kw in scene["objects"]:
        if kind == "plate":
            sim.addPlate(kw["pos"], kw["plate_type"], kw["bc"], kw["friction"])
        elif kind == "box_knife":
            sim.addBoxKnife(kw["bc"], kw["friction"], kw["half"], kw["waypoints"], kw["speed"])
    sim.prepareSimulation()
    marks.append(time.perf_counter())
    frames = 0
    done = 0
    chunk = 16
    while done < args.steps:
        k = min(chunk, args.steps - done)
        if sim.advance(k) > 0:
            # the frame's readback overlaps the next steps; the renderer would wait before drawing
            sim.readIntoAsync(x=ox.numpy(), latent=ol.numpy(), diffusion=od.numpy())
            frames += 1
        done += k
        marks.append(time.perf_counter())
    sim.readIntoAsync(x=ox.numpy(), latent=ol.numpy(), diffusion=od.numpy())
    sim.waitReadback()
    marks.append(time.perf_counter())
    el = time.perf_counter() - t0
    alloc_ms, graph_ms = float(sim.alloc_ms), float(sim.graph_ms)
    sim.close()
    ms = [round(1e3 * (marks[i + 1] - marks[i]), 2) for i in range(len(marks) - 1)]
    el_max = _max_over_ranks(dist, el, device)
    h2d = (hx.numel() + hl.numel()) * 4
    d2h = (frames + 1) * (ox.numel() + ol.numel() + od.numel()) * 4
    return {"value": ws * n * args.steps / el_max, "unit": METRIC, "h2d_bytes_per_step": h2d / args.steps,
            "d2h_bytes_per_step": d2h / args.steps, "frames_read_back": frames + 1,
            "includes": "creation, upload, prepare, K steps, per-frame x/latent/diffusion readback (overlapped "
                        "with the following steps), final readback; after one untimed pass",
            "host_ms": {"create_upload": ms[0], "setup_prepare": ms[1], "advance_chunks": ms[2:-1],
                        "final_readback": ms[-1], "of_which_alloc": round(alloc_ms, 2),
                        "of_which_graph_build": round(graph_ms, 2)}}


def _e2e_breakdown(scene, args, device):
    """One more end-to-end pass, synchronised at every phase boundary, itemising its host time:
    creation, particle upload (of which buffer allocation), parameters and objects, prepare (of
    which grid allocation), the K steps (of which step-graph capture and instantiation, and the
    device time of the steps themselves), the final readback.  Synchronising removes the overlap
    of the timed passes, so the items add up to a little more than a timed pass."""
    import torch
    from pigment_mixing_b200 import Simulation
    n = len(scene["x"])
    hx = torch.from_numpy(np.ascontiguousarray(scene["x"], np.float32)).pin_memory()
    hl = torch.from_numpy(np.ascontiguousarray(scene["latent"], np.float32)).pin_memory()
    ox = torch.empty((n, 3), dtype=torch.float32).pin_memory()
    ol = torch.empty((n, 7), dtype=torch.float32).pin_memory()
    od = torch.empty((n,), dtype=torch.float32).pin_memory()
    t = [time.perf_counter()]

    def mark():
        torch.cuda.synchronize(device)
        t.append(time.perf_counter())
    sim = Simulation(device)
    mark()
    sim.setParticles(hx.numpy(), hl.numpy())
    mark()
    alloc_upload = float(sim.alloc_ms)
    sim.set(**scene["params"])
    for k, v in scene["vectors"].items():
        setattr(sim, k, v)
    for kind, kw in scene["objects"]:
        if kind == "plate":
            sim.addPlate(kw["pos"], kw["plate_type"], kw["bc"], kw["friction"])
        elif kind == "box_knife":
            sim.addBoxKnife(kw["bc"], kw["friction"], kw["half"], kw["waypoints"], kw["speed"])
    mark()
    sim.prepareSimulation()
    mark()
    alloc_prepare = float(sim.alloc_ms) - alloc_upload
    stream = torch.cuda.ExternalStream(sim.stream(), device=device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.advance(args.steps)
    e1.record(stream)
    mark()
    sim.readIntoAsync(x=ox.numpy(), latent=ol.numpy(), diffusion=od.numpy())
    sim.waitReadback()
    mark()
    graph = float(sim.graph_ms)
    sim.close()
    ms = [1e3 * (t[i + 1] - t[i]) for i in range(len(t) - 1)]
    return {"create_ms": ms[0], "upload_ms": ms[1], "upload_alloc_ms": alloc_upload, "setup_ms": ms[2],
            "prepare_ms": ms[3], "prepare_alloc_ms": alloc_prepare, "steps_ms": ms[4],
            "steps_graph_build_ms": graph, "steps_device_ms": e0.elapsed_time(e1), "readback_ms": ms[5],
            "readback_bytes": (ox.numel() + ol.numel() + od.numel()) * 4, "total_ms": sum(ms)}


def _train_on(scene, args, device):
    """A surrogate trained on the scene's own samples: args.log_steps plain steps logging about one
    in `every` Newton solves, then the library's GPU training."""
    from pigment_mixing_b200 import Simulation, scenes, surrogate
    npart = len(scene["x"])
    log = Simulation(device)
    scenes.apply(scene, log)
    every = max(1, int(round(npart * args.log_steps / 4e6)))
    log.set(sample_log_every=every)
    log.enableSampleLog(6 << 20)
    log.prepareSimulation()
    log.advance(args.log_steps)
    xs, ys = log.samples()
    log.close()
    params, hist = surrogate.train(xs, ys, epochs=args.train_epochs, batch=8192, lr=3e-3, seed=0)
    return params, {"samples": int(len(xs)), "log_every": every, "loss_last_epoch": float(hist[-1])}


def _big_point(args, device, params):
    """The 8,388,608-particle scene (four 64^3-cell blocks of four pigments at dx = 1/384): plain and
    surrogate forms, device-timed like the headline, with the surrogate's acceptance and its
    difference from the plain path after the same steps.  The surrogate is trained on this scene's
    own logged samples (as the 2M leg's is on its scene's)."""
    import torch
    from pigment_mixing_b200 import RETURN_MAP_SURROGATE, Simulation, scenes
    sc = _workload("8m")
    n = len(sc["x"])
    out = {"workload": sc["name"], "particles": n, "steps": args.steps}
    if params is not None:
        params, out["surrogate_training"] = _train_on(sc, args, device)
    ref = None
    for form in ("plain", "surrogate"):
        if form == "surrogate" and params is None:
            break
        s = Simulation(device)
        scenes.apply(sc, s)
        if form == "surrogate":
            s.setSurrogate(params)
            s.setReturnMap(RETURN_MAP_SURROGATE)
        s.prepareSimulation()
        s.advance(args.warmup)
        stream = torch.cuda.ExternalStream(s.stream(), device=device)
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.advance(args.steps)
        e1.record(stream)
        torch.cuda.synchronize(device)
        ms = e0.elapsed_time(e1)
        st = s.returnMapStats()
        p = s.getParticles(fields=("x", "latent"))
        d = {"value": n * args.steps / (ms / 1e3), "unit": METRIC, "ms_per_step": ms / args.steps,
             "newton_solves_last_step": st["solves"], "newton_updates_last_step": st["newton_iters"]}
        if form == "surrogate":
            d["surrogate_queued_last_step"] = st["queued"]
            d["surrogate_accepted_last_step"] = st["accepted"]
            d["fallback_rate"] = 1.0 - st["accepted"] / max(1, st["queued"])
            d["max_position_diff_vs_plain"] = float(np.abs(p.x.astype(np.float64) - ref[0]).max())
            d["max_latent_diff_vs_plain"] = float(np.abs(p.latent.astype(np.float64) - ref[1]).max())
            d["speedup_vs_plain"] = d["value"] / out["plain"]["value"]
        else:
            ref = (p.x.astype(np.float64), p.latent.astype(np.float64))
        out[form] = d
        s.close()
    return out


def _active_nodes(sim) -> int:
    """Grid nodes holding mass after the last step (reads the node masses only)."""
    import ctypes as C
    from pigment_mixing_b200._lib import call
    origin = np.zeros(3)
    dims = np.zeros(3, np.uint32)
    up = dims.ctypes.data_as(C.POINTER(C.c_uint32))
    dp = origin.ctypes.data_as(C.POINTER(C.c_double))
    call("pm_get_grid", sim._h, dp, up, None, None, None, None, None, None)
    mass = np.zeros(int(np.prod(dims.astype(np.int64))), np.float32)
    call("pm_get_grid", sim._h, dp, up, mass.ctypes.data_as(C.POINTER(C.c_float)), None, None, None, None, None)
    return int((mass > 0).sum())


def long_run(args):
    """The workload's full step count in both return-map forms (the large scene's report): particle-
    steps/s over the whole run, per-kernel HBM throughput at the end of the run (algorithmic bytes of
    each transfer kernel over its CUDA-event time), and how far the surrogate form's final latents
    are from the plain path's: per latent channel, the total variation distance between the two
    histograms (64 bins over the channel's joint range), the largest per-particle difference and the
    difference of the mean latent."""
    import torch
    from pigment_mixing_b200 import RETURN_MAP_SURROGATE, Simulation, scenes
    device = 0
    torch.cuda.set_device(device)
    sc = _workload(args.workload)
    n = len(sc["x"])
    steps = args.long_steps or int(sc["steps"])
    params, training = _train_on(sc, args, device)
    peak, peak_kind = _peaks()
    out = {"metric": "long_run", "workload": sc["name"], "particles": n, "steps": steps, "unit": METRIC,
           "surrogate_training": training, "peak_gbs": peak, "peak_source": peak_kind}
    latents = {}
    for form in ("plain", "surrogate"):
        s = Simulation(device)
        scenes.apply(sc, s)
        if form == "surrogate":
            s.setSurrogate(params)
            s.setReturnMap(RETURN_MAP_SURROGATE)
        s.prepareSimulation()
        stream = torch.cuda.ExternalStream(s.stream(), device=device)
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.advance(steps)
        e1.record(stream)
        torch.cuda.synchronize(device)
        ms = e0.elapsed_time(e1)
        latents[form] = s.getParticles(fields=("latent",)).latent
        nodes = _active_nodes(s)
        kms = s.profileSteps(3)
        gbs = {k: (ALGO_BYTES[k][0] * n + ALGO_BYTES[k][1] * nodes) / (kms[k] / 1e3) / 1e9 for k in ALGO_BYTES if k in kms}
        rm = s.returnMapStats()
        d = {"value": n * steps / (ms / 1e3), "ms_per_step": ms / steps, "active_nodes_end": nodes,
             "kernel_ms_end": {k: round(v, 4) for k, v in kms.items()},
             "kernel_gbs_end": {k: round(v, 1) for k, v in gbs.items()},
             "kernel_frac_end": {k: round(v / peak, 4) for k, v in gbs.items()}, "error_flags": s.errorFlags()}
        if form == "surrogate":
            d["fallback_rate_last_step"] = 1.0 - rm["accepted"] / max(1, rm["queued"])
            d["speedup_vs_plain"] = d["value"] / out["plain"]["value"]
        out[form] = d
        s.close()
    a, b = latents["plain"].astype(np.float64), latents["surrogate"].astype(np.float64)
    tv = []
    for c in range(7):
        lo, hi = min(a[:, c].min(), b[:, c].min()), max(a[:, c].max(), b[:, c].max())
        ha, _ = np.histogram(a[:, c], bins=64, range=(lo, hi + 1e-12))
        hb, _ = np.histogram(b[:, c], bins=64, range=(lo, hi + 1e-12))
        tv.append(0.5 * float(np.abs(ha / len(a) - hb / len(b)).sum()))
    out["latent_vs_plain"] = {"histogram_tv_distance_by_channel": tv, "histogram_tv_distance_max": max(tv),
                              "max_abs": float(np.abs(a - b).max()),
                              "mean_latent_abs": float(np.abs(a.mean(0) - b.mean(0)).max())}
    print(json.dumps(out), flush=True)


def profile_run(args):
    """A fixed step sequence for profiler captures: `--warm` steps through advance() (graphs),
    `--profile` steps timed kernel by kernel with CUDA events (printed as JSON), then `--plain`
    ordinary step() calls, which an external profiler captures launch by launch."""
    from pigment_mixing_b200 import Simulation, scenes
    sc = _workload(args.workload)
    for kv in args.set:
        k, v = kv.split("=", 1)
        sc["params"][k] = float(v)
    sim = Simulation(0)
    scenes.apply(sc, sim)
    sim.prepareSimulation()
    sim.advance(args.warm)
    out = {"workload": args.workload, "particles": len(sc["x"])}
    if args.profile > 0:
        out["kernel_ms"] = sim.profileSteps(args.profile)
    for _ in range(args.plain):
        sim.step()
    out.update(plastic_count=sim.plastic_count, grid_nodes=sim.grid_nodes, error_flags=sim.errorFlags())
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="2m", choices=["2m", "8m", "32k", "32m", "262k"])
    ap.add_argument("--profile-run", action="store_true",
                    help="no bench line: run the profiler-capture sequence (--warm, --profile, --plain)")
    ap.add_argument("--long-run", action="store_true",
                    help="no bench line: the workload's full step count in both forms (run rate, per-kernel "
                         "HBM GB/s, surrogate latent histogram distance), e.g. --workload 32m --long-run")
    ap.add_argument("--long-steps", type=int, default=0, help="long run: steps (0 = the workload's own count)")
    ap.add_argument("--warm", type=int, default=10, help="profile run: steps through advance() first")
    ap.add_argument("--profile", type=int, default=3, help="profile run: event-timed steps")
    ap.add_argument("--plain", type=int, default=3, help="profile run: plain step() calls at the end")
    ap.add_argument("--set", action="append", default=[], metavar="NAME=VALUE",
                    help="profile run: override a scene parameter, e.g. --set perzyna_exp=1")
    ap.add_argument("--return-map", default="plain", choices=["plain"],
                    help="return map of the headline value (the surrogate form is reported beside it)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-surrogate", action="store_true", help="skip the learned return-map leg")
    ap.add_argument("--log-steps", type=int, default=20, help="plain steps logged for surrogate training")
    ap.add_argument("--train-epochs", type=int, default=30)
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-scenes leg")
    ap.add_argument("--no-splat", action="store_true", help="skip the pigment-splat leg")
    ap.add_argument("--batch-scenes", type=int, default=64)
    ap.add_argument("--batch-steps", type=int, default=50, help="timed rounds of the batched leg")
    ap.add_argument("--no-big", action="store_true", help="skip the 8M-particle point")
    ap.add_argument("--no-accuracy-2m", action="store_true", help="skip the FP64-oracle check of the 2M scene")
    ap.add_argument("--drift-steps", type=int, default=1000,
                    help="steps of the mass / mean-latent drift run on the workload (0 = skip)")
    args = ap.parse_args()
    if args.profile_run:
        return profile_run(args)
    if args.long_run:
        return long_run(args)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
