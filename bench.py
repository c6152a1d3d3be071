"""Throughput benchmark of the force path: body-steps/s of a N = 2^20 Plummer sphere
(quadrupole linear BVH, leaf 16, theta 0.5, softening 0.005, dt 5e-4), one instance per GPU.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = Solver::step (accelerations by Morton sort + LBVH build + bottom-up moments +
warp traversal, then kick-drift) on the whole body set. Prints ONE JSON line on rank 0.

  value   device-resident steps, CUDA events on the solver's stream; L2 (126 MB) flushed by a
          256 MB write before every timed step (outside the events)
  e2e     the same steps through the C ABI with host buffers: copy bodies in (nb_set_bodies),
          step, copy bodies out (nb_get_bodies), wall clock per step
  roofline dominant kernel = the traversal (FP32 pipe + MUFU bound, no tensor-core work):
          achieved = counted interactions x flop weights / traversal event time; a second entry
          gives the sort's algorithmic HBM bytes against the measured copy bandwidth
  cpu_baseline  the oracle (CPU restatement of the reference's TBB path, timing build -O3
          -march=native) for one whole measured step of the same workload: sort, build,
          summaries, traversal of all N bodies, kick-drift; OpenMP over all host cores

With --impl reference the same metric is measured for the reference's algorithm on the host
cores (the oracle port: the reference itself cannot be built on this image): whole steps,
as many of the requested ones as fit in 150 s (at least one), the count stated in the line.
Under torchrun (N > 1) every rank runs its own instance (weak scaling, no data-path collective);
timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "n-body_b200"))

N_BODIES = 1 << 20
SOFTENING = 0.005
THETA = 0.5
LEAF = 16
ORDER = 2
DT = 5e-4
SEED = 43
METRIC = "body-steps/s at N=1M Plummer theta=0.5, force RMS<=1e-3"
# Flop weights per interaction, counted from n-body_b200/csrc/traverse.cu (FMA = 2 flops):
# pair term 20 (usual direct-sum convention; 12 FP32 instructions + 1 rsqrt), quadrupole node 56.
PAIR_FLOPS = 20
QUAD_NODE_FLOPS = 56
MONO_NODE_FLOPS = 20
FP32_FLOP_PER_CLK_PER_SM = 256  # 128 FP32 lanes x FMA
MUFU_PER_CLK_PER_SM = 16        # rsqrt results per clock per SM (4 per sub-partition)
NUM_SMS = 148
# Minimum HBM bytes per body and step of the memory-bound phases (float4 state, 64-bit keys):
# bbox 16, Morton 28, sort 8 passes x 24 = 192, gather 32, Karras build 40, moments 24, kick-drift 80.
BODY_STEP_BYTES = 16 + 28 + 192 + 32 + 40 + 24 + 80


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default: the configuration's own count: 100 for plummer-1m, 50 for "
                         "batched, 2 for dual-4m; 3 CPU samples for --impl reference)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=N_BODIES)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=["plummer-1m", "batched", "serving", "dual-4m"], default="plummer-1m",
                    help="plummer-1m: one N=2^20 instance (the headline); batched: 256 uneven instances; "
                         "serving: Poisson request stream into the continuous-batching server")
    ap.add_argument("--duration", type=float, default=60.0, help="serving: seconds of arrivals per run")
    ap.add_argument("--rate", type=float, default=40.0, help="serving: arrivals per second (open loop)")
    ap.add_argument("--instances", type=int, default=256)
    ap.add_argument("--fp64-summaries", type=int, default=None,
                    help="internal nodes with at least this many bodies combine their moments in FP64 "
                         "(default: 65536 for dual-4m, as its configuration asks; off elsewhere)")
    ap.add_argument("--emulate-ranks", type=int, default=0,
                    help="plummer-1m, dual-4m: also run each of W target shards' force pass alone on this GPU")
    ap.add_argument("--shard-targets", action="store_true",
                    help="N>1: one instance sharded over the ranks' targets with an NCCL all-gather of "
                         "positions and velocities per step (strong scaling) instead of one instance per rank")
    args = ap.parse_args()
    if args.steps is None:
        if args.impl == "reference":
            args.steps = 3
        else:
            args.steps = {"plummer-1m": 100, "batched": 50, "dual-4m": 2}.get(args.workload, 20)
    return args


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = os.path.join("/tmp", f"nb_clocks_{os.getpid()}_{device}.csv")

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = np.array([float(r[1]) for r in rows if r[1].replace(".", "").isdigit()])
        smax = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        loaded = sm[sm >= 0.5 * sm.max()] if len(sm) else sm
        return {"sm_mhz": float(np.median(loaded)) if len(loaded) else None, "sm_max_mhz": smax,
                "reasons": reasons, "samples": int(len(sm))}


def flush_l2(buf):
    buf.zero_()


def accuracy(nb, solver, pm, eps, torch, device):
    """Relative RMS force error vs an FP64 direct sum on a seeded 8192-target subsample, plus the
    reference's own graders: RMSGrader = sqrt(max relerr^2) * 100 (RMSGrader.h:17-37) and
    ConstitutionalGrader = max 100 |dF| / min(|F|, F_rms) (ConstitutionalGrader.h:40-64)."""
    n = len(pm)
    rng = np.random.default_rng(12345)
    idx = np.sort(rng.choice(n, min(8192, n), replace=False))
    acc = solver.update_accelerations()
    dpm = torch.from_numpy(pm).to(device)
    dt = torch.from_numpy(pm[idx].copy()).to(device)
    out = torch.zeros((len(idx), 3), dtype=torch.float64, device=device)
    solver.direct_device(n, dpm.data_ptr(), len(idx), dt.data_ptr(), out.data_ptr(), 64)
    solver.synchronize()
    ref = out.cpu().numpy()
    got = acc[idx, :3].astype(np.float64)
    diff = np.linalg.norm(got - ref, axis=1)
    mag = np.linalg.norm(ref, axis=1)
    rel = diff / mag
    m = pm[idx, 3].astype(np.float64)
    f_rms = np.sqrt(np.mean((mag * m) ** 2))
    # the same pass with the top levels' moments combined in FP64 (the precision option), then back
    solver.set_fp64_summaries(65536)
    got64 = solver.update_accelerations()[idx, :3].astype(np.float64)
    solver.set_fp64_summaries(0)
    rel64 = np.linalg.norm(got64 - ref, axis=1) / mag
    return {
        "force_rms_rel": float(np.sqrt(np.mean(rel ** 2))),
        "force_rms_rel_fp64_top_summaries": float(np.sqrt(np.mean(rel64 ** 2))),
        "force_max_rel": float(rel.max()),
        "rms_grader_pct": float(np.sqrt((rel ** 2).max()) * 100.0),
        "constitutional_pct": float(np.max(100.0 * diff * m / np.minimum(mag * m, f_rms))),
        "sample_targets": int(len(idx)),
        "reference": "FP64 direct sum on GPU",
    }


REF_BUDGET_S = 150.0   # the reference arm stops timing whole steps once this much has elapsed (>= 1 step)
CPU_WARMUP_N = 1 << 16


def _oracle_timing():
    """The oracle's timing build (-O3 -march=native, compiled for this host on first use)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O

    return O, O.timing_lib()


def cpu_whole_steps(pm, vel, eps, max_steps, budget_s):
    """Whole Solver::step()s of the oracle (the reference's algorithm, OpenMP over the host cores
    where the reference runs tbb::parallel_for_each): Morton codes, sort, tree build, summaries,
    the traversal of every body, then the kick-drift. Stops after max_steps, or once budget_s has
    elapsed (at least one step). Returns (seconds per step list, threads)."""
    O, L = _oracle_timing()
    p, v = pm, vel
    times = []
    t_all = time.perf_counter()
    for _ in range(max_steps):
        t0 = time.perf_counter()
        a, _ = O.bh_accelerations(p, eps=eps, theta=THETA, leaf=LEAF, order=ORDER, L=L)
        p, v = O.kick_drift(p, v, a, DT, L=L)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_all > budget_s:
            break
    return times, O.max_threads(L)


def cpu_warmup(eps):
    """One untimed whole step at 2^16 bodies (builds the timing library, pages in, starts threads)."""
    from nbody_b200 import scenarios

    wp, wv = scenarios.plummer(CPU_WARMUP_N, seed=SEED)
    cpu_whole_steps(wp, wv, eps, 1, 0.0)


def cpu_baseline(pm, vel, eps):
    """The oracle timed for one whole step of the workload (measured, not extrapolated)."""
    cpu_warmup(eps)
    times, threads = cpu_whole_steps(pm, vel, eps, 1, 0.0)
    n = len(pm)
    return {
        "value": n / times[0],
        "unit": "body-steps/s",
        "cores": threads,
        "kind": "port",
        "sample": f"1 whole step measured at N = {n} (Morton sort, tree build, summaries, traversal of all "
                  f"{n} bodies, kick-drift): {times[0]:.1f} s; oracle timing build -O3 -march=native, "
                  f"OpenMP over {threads} host threads",
    }


def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(REPO, "n-body_b200"))
    from nbody_b200 import scenarios

    pm, vel = scenarios.plummer(args.n, seed=SEED)
    eps = scenarios.softening_to_epsilon(SOFTENING)
    for _ in range(min(args.warmup, 1)):
        cpu_warmup(eps)
    times, threads = cpu_whole_steps(pm, vel, eps, args.steps, REF_BUDGET_S)
    step_s = float(np.mean(times))
    value = args.n / step_s
    base = {
        "value": value, "unit": "body-steps/s", "cores": threads, "kind": "port",
        "sample": f"{len(times)} whole steps measured at N = {args.n} (of {args.steps} requested; timing stops "
                  f"after {REF_BUDGET_S:.0f} s): Morton sort, tree build, summaries, traversal of all bodies, "
                  f"kick-drift; oracle timing build -O3 -march=native, OpenMP over {threads} host threads",
    }
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "body-steps/s", "n_gpus": args.gpus,
        "steps": len(times), "steps_requested": args.steps, "warmup": min(args.warmup, 1),
        "warmup_note": f"one untimed whole step at N = {CPU_WARMUP_N}",
        "ms_per_step": 1000.0 * step_s, "step_ms": [1000.0 * t for t in times],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args), "cpu_baseline": base,
        "e2e": {"value": value, "unit": "body-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_config(args):
    return {"workload": f"plummer-{args.n}-quadrupole-linear-bvh", "n_bodies": args.n, "theta": THETA,
            "leaf_size": LEAF, "order": ORDER, "softening": SOFTENING, "epsilon_added_to_r2": SOFTENING ** 2,
            "dt": DT, "seed": SEED, "l2": "flushed (256 MB write) before every timed step",
            "parallelism": "one instance per GPU"}


def run_ours(args):
    import torch

    world, rank, local = dist_env()
    device = local
    torch.cuda.set_device(device)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import nbody_b200 as nb
    from nbody_b200 import scenarios

    pm, vel = scenarios.plummer(args.n, seed=SEED + rank)
    eps = scenarios.softening_to_epsilon(SOFTENING)
    # A dedicated (non-default) stream shared by the solver, the L2 flush and the timing events.
    stream = torch.cuda.Stream(device)
    with torch.cuda.stream(stream):
        if args.shard_targets and world > 1:
            pm, vel = scenarios.plummer(args.n, seed=SEED)  # one instance, the same on every rank
            line = _run_sharded_on_stream(args, torch, nb, pm, vel, eps, stream, world, rank, device)
        else:
            line = _run_ours_on_stream(args, torch, nb, pm, vel, eps, stream, world, rank, device)
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def _run_ours_on_stream(args, torch, nb, pm, vel, eps, stream, world, rank, device):
    solver = nb.QuadrupoleLinearBVHSolver(bodies=pm, rule=nb.Gravity(1.0, eps), velocities=vel, theta=THETA,
                                          max_leaf_size=LEAF, time_step=DT, device=device)
    solver.set_stream(stream.cuda_stream)
    # the traversal's launch shape at the configured leaf size, measured on these bodies
    from nbody_b200 import autotune as at

    shape, shape_ms = at.tune_shape(solver, passes=3)
    acc_info = accuracy(nb, solver, pm, eps, torch, torch.device("cuda", device))
    counts = solver.counts()
    solver.set_bodies(pm, vel)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)

    for _ in range(args.warmup):
        flush_l2(flush)
        solver.step(1)
    torch.cuda.synchronize(device)
    p0, v0 = solver.bodies()
    solver.enable_timing(True)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(device)
    with Clocks(device) as clk:
        for k in range(args.steps):
            flush_l2(flush)
            starts[k].record(stream)
            solver.step(1)
            ends[k].record(stream)
        torch.cuda.synchronize(device)
    if world > 1:
        torch.distributed.barrier()
    step_ms = float(sum(s.elapsed_time(e) for s, e in zip(starts, ends)))
    phases = solver.phase_times()
    solver.enable_timing(False)
    p1, v1 = solver.bodies()
    mom0 = (p0[:, 3:4].astype(np.float64) * v0[:, :3]).sum(0)
    mom1 = (p1[:, 3:4].astype(np.float64) * v1[:, :3]).sum(0)

    # e2e through the C ABI with pinned host buffers
    h_pm = torch.from_numpy(p1.copy()).pin_memory()
    h_vel = torch.from_numpy(v1.copy()).pin_memory()
    out_pm = torch.empty_like(h_pm).pin_memory()
    out_vel = torch.empty_like(h_vel).pin_memory()
    lib = nb.lib()
    torch.cuda.synchronize(device)
    if world > 1:
        torch.distributed.barrier()
    e2e_s = 0.0
    for _ in range(args.e2e_steps):
        t0 = time.perf_counter()
        solver._check(lib.nb_set_bodies(solver.handle, args.n, h_pm.data_ptr(), h_vel.data_ptr()))
        solver._check(lib.nb_step(solver.handle, 1))
        solver._check(lib.nb_get_bodies(solver.handle, out_pm.data_ptr(), out_vel.data_ptr()))
        e2e_s += time.perf_counter() - t0
        h_pm.copy_(out_pm)
        h_vel.copy_(out_vel)

    t_max = step_ms
    e2e_max = e2e_s
    if world > 1:
        t = torch.tensor([step_ms, e2e_s], dtype=torch.float64, device=device)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        t_max, e2e_max = float(t[0]), float(t[1])
    value = args.n * world * args.steps / (t_max / 1000.0)
    e2e_value = args.n * world * args.e2e_steps / e2e_max

    # roofline of the dominant kernel (traversal), per launch
    passes = max(int(phases["passes"]), 1)
    trav_ms = phases["traverse_ms"] / passes
    flops = counts["particle_particle"] * PAIR_FLOPS + counts["node_particle"] * QUAD_NODE_FLOPS
    clk = clk.summary()
    sm_mhz = clk.get("sm_mhz") or 1965.0
    peak = NUM_SMS * FP32_FLOP_PER_CLK_PER_SM * sm_mhz * 1e6 / 1e12
    achieved = flops / (trav_ms / 1000.0) / 1e12
    traffic = read_traffic()
    sort_ms = phases["sort_ms"] / passes
    sort_bytes = 8 * 24 * args.n
    hbm_peak = measured_hbm()
    line = {
        "metric": METRIC, "value": value, "unit": "body-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Plummer sphere)",
        "config": workload_config(args),
        "autotune": {"traversal_shape": list(shape), "ms_per_force_pass_by_shape": shape_ms,
                     "method": "force passes at each launch shape (threads per block x traversal tile) at the "
                               "configured leaf size 16, fastest kept"},
        "e2e": {"value": e2e_value, "unit": "body-steps/s", "h2d_bytes_per_step": 32 * args.n,
                "d2h_bytes_per_step": 32 * args.n, "steps": args.e2e_steps,
                "path": "nb_set_bodies (pinned host) + nb_step + nb_get_bodies, wall clock"},
        "roofline": {"bound": "fp32", "kernel": "bh_kernel<2> (traversal)", "achieved": achieved, "peak": peak,
                     "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
                     "peak_source": f"148 SMs x 256 FP32 flop/clk x {sm_mhz:.0f} MHz SM clock measured under "
                                    "load (no FP32 peak in MEASURED_PEAKS.json; tensor cores do not apply)",
                     "flops_per_launch": flops, "ms_per_launch": trav_ms,
                     "interactions": {"pp": counts["particle_particle"], "np": counts["node_particle"]}},
        "roofline_hbm": {"bound": "hbm", "kernel": "onesweep radix sort (8 passes)",
                         "achieved": sort_bytes / (sort_ms / 1000.0) / 1e9 if sort_ms > 0 else None,
                         "peak": hbm_peak, "unit": "GB/s",
                         "frac": (sort_bytes / (sort_ms / 1000.0) / 1e9) / hbm_peak if sort_ms > 0 and hbm_peak
                         else None, "bytes_per_sort": sort_bytes, "ms_per_sort": sort_ms,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)"},
        "body_step_roofline": body_step_roofline(args.n, counts, t_max / args.steps, sm_mhz, hbm_peak),
        "phases_ms_per_step": {k: phases[k] / passes for k in
                               ("bbox_ms", "morton_ms", "sort_ms", "gather_ms", "build_ms", "traverse_ms",
                                "integrate_ms")},
        "gpu_launches": int(phases["launches"]),
        "accuracy": acc_info,
        "momentum_drift": float(np.linalg.norm(mom1 - mom0)),
        "clocks": clk,
    }
    solver.close()
    if args.emulate_ranks > 1:
        make = lambda: nb.QuadrupoleLinearBVHSolver(rule=nb.Gravity(1.0, eps), theta=THETA, max_leaf_size=LEAF,
                                                    time_step=DT, device=device)
        line["emulated_target_shards"] = shard_emulation(
            nb, torch, make, pm, vel, args.emulate_ranks, device,
            sum(phases[k] for k in phases if k.endswith("_ms") and k != "integrate_ms") / passes)
    line["diagnostics"] = energy_diagnostics(nb, device)
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(pm, vel, eps)
    return line


def body_step_roofline(n, counts, step_ms, sm_mhz, hbm_gbs):
    """Lower bound on one step: the memory-bound phases at the measured copy bandwidth plus the
    interactions at the slower of the FP32 pipe (flop weights) and the MUFU pipe (one rsqrt each)."""
    flops = counts["particle_particle"] * PAIR_FLOPS + counts["node_particle"] * QUAD_NODE_FLOPS
    rsqrt = counts["particle_particle"] + counts["node_particle"]
    t_mem = BODY_STEP_BYTES * n / ((hbm_gbs or 6650.0) * 1e9)
    t_fp32 = flops / (NUM_SMS * FP32_FLOP_PER_CLK_PER_SM * sm_mhz * 1e6)
    t_mufu = rsqrt / (NUM_SMS * MUFU_PER_CLK_PER_SM * sm_mhz * 1e6)
    t_roof = t_mem + max(t_fp32, t_mufu)
    return {"t_roofline_ms": t_roof * 1e3, "t_measured_ms": step_ms, "frac": t_roof * 1e3 / step_ms,
            "memory_ms": t_mem * 1e3, "fp32_ms": t_fp32 * 1e3, "mufu_ms": t_mufu * 1e3,
            "bytes_per_body": BODY_STEP_BYTES,
            "peaks": "HBM: MEASURED_PEAKS.json hbm_gbs; FP32 and MUFU: per-SM rates x 148 SMs x measured SM clock"}


def energy_diagnostics(nb, device, n=65536, steps=100):
    """Energy and momentum drift of the same solver configuration on a 65,536-body Plummer sphere
    over 100 steps, both measured in FP64 on the device (nb_energy is an O(N^2) direct sum, so the
    diagnostic run is smaller than the timed one)."""
    from nbody_b200 import scenarios

    pm, vel = scenarios.plummer(n, seed=SEED + 1000)
    eps = scenarios.softening_to_epsilon(SOFTENING)
    with nb.QuadrupoleLinearBVHSolver(bodies=pm, velocities=vel, rule=nb.Gravity(1.0, eps), theta=THETA,
                                      max_leaf_size=LEAF, time_step=DT, device=device) as s:
        k0, u0 = s.energy()
        p0, v0 = s.bodies()
        s.step(steps)
        k1, u1 = s.energy()
        p1, v1 = s.bodies()
    mom0 = (p0[:, 3:4].astype(np.float64) * v0[:, :3]).sum(0)
    mom1 = (p1[:, 3:4].astype(np.float64) * v1[:, :3]).sum(0)
    e0, e1 = k0 + u0, k1 + u1
    return {"n_bodies": n, "steps": steps, "energy_start": e0, "energy_end": e1,
            "energy_rel_drift": abs(e1 - e0) / abs(e0), "momentum_drift": float(np.linalg.norm(mom1 - mom0)),
            "method": "FP64 direct-sum potential and kinetic energy on the device (nb_energy)"}


def _run_sharded_on_stream(args, torch, nb, pm, vel, eps, stream, world, rank, device):
    """One instance of args.n bodies advanced by all ranks: each evaluates its slice of the
    Morton-ordered targets, then an NCCL in-place all-gather of positions and velocities."""
    solver = nb.QuadrupoleLinearBVHSolver(rule=nb.Gravity(1.0, eps), theta=THETA, max_leaf_size=LEAF,
                                          time_step=DT, device=device)
    solver.set_stream(stream.cuda_stream)
    solver.set_shard(rank, world)
    solver.set_bodies(pm, vel)
    stepper = nb.ShardedStepper(solver)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    for _ in range(max(args.warmup, 3)):
        flush_l2(flush)
        stepper.step(1)
    torch.cuda.synchronize(device)
    solver.enable_timing(True)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    torch.distributed.barrier()
    torch.cuda.synchronize(device)
    with Clocks(device) as clk:
        for k in range(args.steps):
            flush_l2(flush)
            starts[k].record(stream)
            stepper.step(1)
            ends[k].record(stream)
        torch.cuda.synchronize(device)
    torch.distributed.barrier()
    step_ms = float(sum(a.elapsed_time(b) for a, b in zip(starts, ends)))
    phases = solver.phase_times()
    solver.enable_timing(False)
    lib = nb.lib()
    h_pm = torch.from_numpy(pm.copy()).pin_memory()
    h_vel = torch.from_numpy(vel.copy()).pin_memory()
    out_pm = torch.empty_like(h_pm).pin_memory()
    out_vel = torch.empty_like(h_vel).pin_memory()
    torch.distributed.barrier()
    e2e_s = 0.0
    for _ in range(args.e2e_steps):
        t0 = time.perf_counter()
        solver._check(lib.nb_set_bodies(solver.handle, args.n, h_pm.data_ptr(), h_vel.data_ptr()))
        stepper.step(1)
        solver._check(lib.nb_get_bodies(solver.handle, out_pm.data_ptr(), out_vel.data_ptr()))
        e2e_s += time.perf_counter() - t0
    t = torch.tensor([step_ms, e2e_s], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    t_max, e2e_max = float(t[0]), float(t[1])
    solver.close()
    passes = max(int(phases["passes"]), 1)
    chunk, _, _ = nb.shard_range(args.n, rank, world)
    return {
        "metric": METRIC, "value": args.n * args.steps / (t_max / 1000.0), "unit": "body-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Plummer sphere)",
        "config": dict(workload_config(args), parallelism=f"target-sharded over {world} ranks, "
                                                         "NCCL in-place all-gather of positions and velocities"),
        "e2e": {"value": args.n * args.e2e_steps / e2e_max, "unit": "body-steps/s",
                "h2d_bytes_per_step": 32 * args.n, "d2h_bytes_per_step": 32 * args.n, "steps": args.e2e_steps},
        "allgather_bytes_per_step": 2 * 16 * chunk * world,
        "phases_ms_per_step": {k: phases[k] / passes for k in
                               ("bbox_ms", "morton_ms", "sort_ms", "gather_ms", "build_ms", "traverse_ms",
                                "integrate_ms")},
        "gpu_launches": int(phases["launches"]),
        "clocks": clk.summary(),
    }


def measured_hbm():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(path))["hbm_gbs"])
    except Exception:
        return 6650.0


def read_traffic():
    """DRAM bytes per traversal launch from the committed ncu summary, if one exists."""
    path = os.path.join(REPO, "profiles", "traffic.txt")
    try:
        for line in open(path):
            if line.startswith("bh_kernel_traffic_bytes_per_launch"):
                return float(line.split("=")[1])
    except Exception:
        pass
    return None


BATCH_SOFTENING = 0.01
BATCH_DT = 5e-4


def batched_instances(count, seed=44):
    """256 Plummer spheres with N log-uniform in [1024, 200000] and theta uniform in [0.4, 0.7]."""
    from nbody_b200 import scenarios

    return scenarios.batched_plummer(count, seed=seed)


def run_batched(args):
    """Batched workload: every instance advanced by one launch per phase (graph-captured steps),
    against the same instances stepped one after another through the plain single-instance path."""
    import torch

    world, rank, local = dist_env()
    device = local
    torch.cuda.set_device(device)
    import nbody_b200 as nb

    sizes, thetas, bodies, vels = batched_instances(args.instances, seed=44 + rank)
    eps = float(np.float32(BATCH_SOFTENING) * np.float32(BATCH_SOFTENING))
    total = int(sizes.sum())
    stream = torch.cuda.Stream(device)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    with torch.cuda.stream(stream):
        s = nb.QuadrupoleLinearBVHSolver(rule=nb.Gravity(1.0, eps), max_leaf_size=LEAF, time_step=BATCH_DT,
                                         device=device)
        s.set_stream(stream.cuda_stream)
        s.set_instances(sizes, np.concatenate(bodies), np.concatenate(vels), thetas)
        # leaf size and traversal launch shape measured on this batch (force passes only: the
        # state does not change)
        tuned = s.autotune(candidates=(4, 6, 8, 12, 16, 24), passes=2, tolerance=0.02)
        leaf, shape = tuned.leaf, tuned.shape
        accuracy = batched_accuracy(nb, s, sizes, bodies, eps, torch, device)
        batch_acc = s.update_accelerations()
        s.enable_graphs(True)
        s.step(max(args.warmup, 3))
        torch.cuda.synchronize(device)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        flush.zero_()
        with Clocks(device) as clk:
            t0.record(stream)
            s.step(args.steps)
            t1.record(stream)
            torch.cuda.synchronize(device)
        batch_ms = t0.elapsed_time(t1)
        clocks = clk.summary()
        s.enable_timing(True)
        s.step(2)
        phases = s.phase_times()
        s.close()
        # the same instances, one after another, through the plain path (one context each, same
        # theta, leaf size and launch shape: every instance's accelerations are bit-identical to the
        # batch's, so the two runs are at equal accuracy by construction; checked below)
        ctxs = []
        starts = np.concatenate([[0], np.cumsum(sizes)])
        identical = True
        for k in range(len(sizes)):
            c = nb.QuadrupoleLinearBVHSolver(bodies=bodies[k], velocities=vels[k], rule=nb.Gravity(1.0, eps),
                                             theta=float(thetas[k]), max_leaf_size=leaf, time_step=BATCH_DT,
                                             device=device)
            c.set_stream(stream.cuda_stream)
            c.traversal_shape = shape
            identical &= bool(np.array_equal(c.update_accelerations(), batch_acc[starts[k]:starts[k + 1]]))
            c.step(1)
            ctxs.append(c)
        seq_steps = max(1, min(args.steps, 5))
        torch.cuda.synchronize(device)
        flush.zero_()
        t0.record(stream)
        for _ in range(seq_steps):
            for c in ctxs:
                c.step(1)
        t1.record(stream)
        torch.cuda.synchronize(device)
        seq_ms = t0.elapsed_time(t1)
        for c in ctxs:
            c.close()
    value = total * args.steps / (batch_ms / 1000.0)
    seq_value = total * seq_steps / (seq_ms / 1000.0)
    line = {
        "metric": "body-steps/s, 256 batched Plummer instances (N log-uniform 1024..200000, theta 0.4..0.7)",
        "value": value, "unit": "body-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": batch_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded Plummer spheres)",
        "config": {"workload": f"batched-{len(sizes)}-plummer-quadrupole", "instances": int(len(sizes)),
                   "total_bodies": total, "n_min": int(sizes.min()), "n_max": int(sizes.max()),
                   "softening": BATCH_SOFTENING, "leaf_size": leaf, "order": ORDER, "dt": BATCH_DT,
                   "graphs": "two steps per CUDA graph", "l2": "flushed (256 MB write) before the timed steps"},
        "sequential_plain_path": {"value": seq_value, "unit": "body-steps/s", "steps": seq_steps,
                                  "leaf_size": leaf, "traversal_shape": list(shape),
                                  "ratio_batched_over_sequential": value / seq_value,
                                  "accelerations_bit_identical_to_batch": identical,
                                  "accuracy": "equal: the same instances with the same theta, leaf size and launch "
                                              "shape give bit-identical accelerations (force RMS as in accuracy)"},
        "autotune": {"leaf_size": leaf, "ms_per_force_pass": {str(k): v for k, v in tuned.timings_ms.items()},
                     "traversal_shape": list(shape), "ms_per_force_pass_by_shape": tuned.shape_timings_ms,
                     "method": "force passes of this batch at each candidate leaf size (default launch shape), "
                               "then at each launch shape (threads per block x traversal tile), fastest kept"},
        "accuracy": accuracy,
        "clocks": clocks,
        "phases_ms_per_step": {k: phases[k] / max(phases["passes"], 1) for k in
                               ("bbox_ms", "morton_ms", "sort_ms", "gather_ms", "build_ms", "traverse_ms",
                                "integrate_ms")},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def batched_accuracy(nb, s, sizes, bodies, eps, torch, device, picks=(0, 85, 170, 255), targets=2048):
    """Relative RMS force error of the batched pass against an FP64 direct sum, on up to 2048
    seeded targets of four of the instances."""
    acc = s.update_accelerations()
    starts = np.concatenate([[0], np.cumsum(sizes)])
    rng = np.random.default_rng(2024)
    rels = []
    for k in picks:
        if k >= len(sizes):
            continue
        pm = bodies[k]
        idx = np.sort(rng.choice(len(pm), min(targets, len(pm)), replace=False))
        dpm = torch.from_numpy(pm).to(device)
        dt = torch.from_numpy(pm[idx].copy()).to(device)
        out = torch.zeros((len(idx), 3), dtype=torch.float64, device=device)
        s.direct_device(len(pm), dpm.data_ptr(), len(idx), dt.data_ptr(), out.data_ptr(), 64)
        s.synchronize()
        ref = out.cpu().numpy()
        got = acc[starts[k] + idx, :3].astype(np.float64)
        rels.append(np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1))
    r = np.concatenate(rels)
    return {"force_rms_rel": float(np.sqrt(np.mean(r ** 2))), "force_max_rel": float(r.max()),
            "instances_sampled": [int(k) for k in picks if k < len(sizes)], "targets_per_instance": targets,
            "reference": "FP64 direct sum on GPU"}


def serving_pools(seed=45, n_max=1 << 21):
    """Two shuffled body pools (Plummer, uniform ball) that requests take prefixes of: a prefix of
    a shuffled sample is itself a sample of the distribution."""
    from nbody_b200 import scenarios

    rng = np.random.default_rng(seed)
    pools = []
    for kind, gen in (("plummer", scenarios.plummer), ("uniform", scenarios.uniform_ball)):
        pm, vel = gen(n_max, seed=seed)
        perm = rng.permutation(n_max)
        pools.append((kind, pm[perm].copy(), vel[perm].copy()))
    return pools


def serve_run(nb, pools, rate, duration, rng, eps, steps_range=(10, 1000), n_range=(2048, 1 << 21),
              budget=150 * 10 ** 9, drain=0.0, leaf=LEAF, shape=(256, 64)):
    """Open-loop Poisson arrivals for `duration` seconds (then `drain` more seconds of ticks).
    Latency = completion time - arrival time, wall clock."""
    arrivals = []
    t = rng.exponential(1.0 / rate)
    while t < duration:
        kind, pm, vel = pools[rng.integers(0, 2)]
        n = int(np.round(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1])))))
        steps = int(rng.integers(steps_range[0], steps_range[1] + 1))
        theta = float(rng.uniform(0.4, 0.7))
        arrivals.append((t, n, steps, theta, pm, vel))
        t += rng.exponential(1.0 / rate)
    sv = nb.Server(rule=nb.Gravity(1.0, eps), order=ORDER, max_leaf_size=leaf, time_step=DT, hbm_budget_bytes=budget)
    sv.set_traversal_shape(shape)
    pending = {}  # id -> (arrival time, bodies)
    latencies = []
    t0 = time.perf_counter()
    nxt = 0
    while True:
        now = time.perf_counter() - t0
        if now > duration + drain:
            break
        while nxt < len(arrivals) and arrivals[nxt][0] <= now:
            ta, n, steps, theta, pm, vel = arrivals[nxt]
            rid = sv.submit(pm[:n], vel[:n], theta=theta, steps=steps)
            pending[rid] = (ta, n)
            nxt += 1
        st = sv.stats()
        if st["running"] == 0 and st["queued"] == 0:
            if nxt >= len(arrivals):
                break  # everything submitted has completed
            time.sleep(0.0005)
            continue
        if sv.tick():
            done_now = time.perf_counter() - t0
            for rid in list(pending):
                if sv.status(rid)[0] == nb.Server.DONE:
                    ta, n = pending.pop(rid)
                    latencies.append(done_now - ta)
                    sv.take_result(rid, n)
    elapsed = time.perf_counter() - t0
    st = sv.stats()
    sv.close()
    lat = np.array(latencies) if latencies else np.array([np.nan])
    return {
        "arrival_rate_per_s": rate, "duration_s": duration, "submitted": nxt, "completed": len(latencies),
        "running_at_end": st["running"], "queued_at_end": st["queued"], "ticks": st["ticks"],
        "relayouts": st["relayouts"], "body_steps": st["body_steps"],
        "throughput_body_steps_per_s": st["body_steps"] / elapsed,
        "latency_p50_s": float(np.nanpercentile(lat, 50)), "latency_p99_s": float(np.nanpercentile(lat, 99)),
        "offered_body_steps_per_s": float(sum(a[1] * a[2] for a in arrivals) / duration),
    }


def serving_sample(pools, requests=64, seed=47):
    """A sample batch of requests drawn like the stream: sizes, (bodies, velocities), thetas."""
    rng = np.random.default_rng(seed)
    sizes, bodies, thetas = [], [], []
    for _ in range(requests):
        _, pm, vel = pools[rng.integers(0, 2)]
        n = int(np.round(np.exp(rng.uniform(np.log(2048), np.log(1 << 21)))))
        sizes.append(n)
        bodies.append((pm[:n], vel[:n]))
        thetas.append(float(rng.uniform(0.4, 0.7)))
    return sizes, bodies, thetas


def serving_leaf(nb, sample, eps):
    """Leaf size and traversal launch shape for the server, measured on the sample batch of requests."""
    sizes, bodies, thetas = sample
    with nb.QuadrupoleLinearBVHSolver(rule=nb.Gravity(1.0, eps), time_step=DT) as s:
        s.set_instances(sizes, np.concatenate([b[0] for b in bodies]), thetas=np.asarray(thetas, np.float32))
        tuned = s.autotune(candidates=(6, 8, 12, 16, 24), passes=1)
    return tuned.leaf, tuned


def serving_sample_vs_sequential(nb, sample, eps, leaf, torch, steps=2, shape=(256, 64)):
    """The sample batch advanced together (one batched step per tick, as the server runs it) against
    the same requests advanced one after another through the plain single-instance path, on the
    device clock. Both run the same steps of the same bodies, with identical results."""
    sizes, bodies, thetas = sample
    total = int(sum(sizes))
    stream = torch.cuda.Stream()  # the contexts launch on this stream, the events are recorded on it
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    with nb.QuadrupoleLinearBVHSolver(rule=nb.Gravity(1.0, eps), max_leaf_size=leaf, time_step=DT) as s:
        s.set_stream(stream.cuda_stream)
        s.traversal_shape = shape
        s.set_instances(sizes, np.concatenate([b[0] for b in bodies]), np.concatenate([b[1] for b in bodies]),
                        np.asarray(thetas, np.float32))
        s.step(3)
        torch.cuda.synchronize()
        t0.record(stream)
        s.step(steps)
        t1.record(stream)
        torch.cuda.synchronize()
        batched_ms = t0.elapsed_time(t1)
    seq_ms = 0.0
    for n, (pm, vel), theta in zip(sizes, bodies, thetas):
        with nb.QuadrupoleLinearBVHSolver(bodies=pm, velocities=vel, rule=nb.Gravity(1.0, eps), theta=theta,
                                          max_leaf_size=leaf, time_step=DT) as c:
            c.set_stream(stream.cuda_stream)
            c.traversal_shape = shape
            c.step(1)
            torch.cuda.synchronize()
            t0.record(stream)
            c.step(steps)
            t1.record(stream)
            torch.cuda.synchronize()
            seq_ms += t0.elapsed_time(t1)
    batched = total * steps / (batched_ms / 1000.0)
    sequential = total * steps / (seq_ms / 1000.0)
    return {"requests": len(sizes), "total_bodies": total, "steps": steps, "leaf_size": leaf,
            "traversal_shape": list(shape),
            "batched_body_steps_per_s": batched, "sequential_plain_body_steps_per_s": sequential,
            "ratio_batched_over_sequential": batched / sequential,
            "ratio_served_over_sequential": None}


def run_serving(args):
    import torch

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    import nbody_b200 as nb

    eps = float(np.float32(BATCH_SOFTENING) * np.float32(BATCH_SOFTENING))
    pools = serving_pools()
    rng = np.random.default_rng(46 + rank)
    sample = serving_sample(pools)
    leaf, tuned = serving_leaf(nb, sample, eps)
    shape = tuned.shape
    versus = serving_sample_vs_sequential(nb, sample, eps, leaf, torch, shape=shape)
    with Clocks(local) as clk:
        overload = serve_run(nb, pools, args.rate, args.duration, rng, eps, leaf=leaf, shape=shape)
    overload["clocks"] = clk.summary()
    # the server's own throughput (re-layouts, admission and retirement included) on the stream
    versus["ratio_served_over_sequential"] = (overload["throughput_body_steps_per_s"] /
                                              versus["sequential_plain_body_steps_per_s"])
    # calibrated run: arrival rate at 70 % of the measured capacity for the mean request size
    mean_work = np.mean([np.exp(rng.uniform(np.log(2048), np.log(1 << 21))) for _ in range(20000)]) * 505.0
    rate = max(0.7 * overload["throughput_body_steps_per_s"] / mean_work, 0.05)
    with Clocks(local) as clk:
        calibrated = serve_run(nb, pools, rate, args.duration, rng, eps, drain=args.duration, leaf=leaf, shape=shape)
    calibrated["clocks"] = clk.summary()
    line = {
        "metric": "serving: aggregate body-steps/s and request latency p50/p99 (Poisson arrivals)",
        "value": overload["throughput_body_steps_per_s"], "unit": "body-steps/s", "n_gpus": world,
        "steps": overload["ticks"], "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (Plummer or uniform ball, 50/50)",
        "config": {"workload": "serving-poisson", "n_range": [2048, 1 << 21], "steps_range": [10, 1000],
                   "theta_range": [0.4, 0.7], "softening": BATCH_SOFTENING, "hbm_budget_bytes": 150 * 10 ** 9,
                   "order": ORDER, "leaf_size": leaf},
        "autotune": {"leaf_size": leaf, "ms_per_force_pass": {str(k): v for k, v in tuned.timings_ms.items()},
                     "traversal_shape": list(shape), "ms_per_force_pass_by_shape": tuned.shape_timings_ms,
                     "method": "force passes of a 64-request sample batch at each candidate leaf size, then at "
                               "each launch shape"},
        "sample_batch_vs_sequential": versus,
        "overload_run": overload,
        "calibrated_run": calibrated,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


DUAL_HALF = 1 << 21
DUAL_THETA = 0.4
DUAL_LEAF = 64           # LinearBVH's default maxLeafSize (LinearBVH.h:88)
DUAL_SOFTENING = 0.005
# FP64 combination of the moments of nodes with at least this many bodies (the top levels: about
# 6 of them at 2 x 2^21 bodies); the configuration asks for FP64 root-level moments
DUAL_FP64_SUMMARIES = 65536
# Flop weights of the dual-tree interactions, counted from n-body_b200/csrc/dualtree.cu and
# stensor.cuh after unrolling (FMA = 2): pair 20; M2P with octupole moments (the two contractions
# grouped for symmetric moments) 125; P2L into an order-4 field (D2..D4) 440; M2L (D2..D4, three
# contractions) 820.
DUAL_PAIR_FLOPS = 20
DUAL_NP_FLOPS = 125
DUAL_PN_FLOPS = 440
DUAL_NN_FLOPS = 820


def colliding_hernquist(half, seed=46):
    """Two Hernquist spheres (a = 1, total mass 1 each, truncated at 100 a) centred at x = -10 and
    x = +10, approaching at 0.5 along x (+-0.25 each)."""
    from nbody_b200 import scenarios

    return scenarios.colliding_hernquist(half, seed=seed)


def dual_cpu_baseline(half_sample, eps):
    """The oracle's dual-tree solver (CPU restatement, OpenMP over the host cores) on the same scene
    at a reduced body count: one full force evaluation, timed."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O

    O.lib()
    pm, _ = colliding_hernquist(half_sample, seed=146)
    t0 = time.perf_counter()
    O.dual_accelerations(pm, eps=eps, theta=DUAL_THETA, leaf=DUAL_LEAF, order=3)
    dt = time.perf_counter() - t0
    return {"value": len(pm) / dt, "unit": "body-steps/s", "cores": O.max_threads(), "kind": "port",
            "sample": f"one force pass of the same scene at 2 x {half_sample} bodies ({dt:.1f} s); the "
                      "per-body cost grows with N, so this overstates the CPU rate at 2 x 2^21"}


def run_dual(args):
    """Precision-study scene: two colliding Hernquist spheres of 2^21 bodies each, dual-tree solver
    with octupole moments and order-4 local fields (MultipoleImplicitLinearBVHFMMSolver<3>),
    theta 0.4. Error vs an FP64 direct sum on a seeded 65,536-body subsample."""
    import torch

    world, rank, local = dist_env()
    device = local
    torch.cuda.set_device(device)
    import nbody_b200 as nb

    half = args.n // 2 if args.n != N_BODIES else DUAL_HALF
    pm, vel = colliding_hernquist(half, seed=46 + rank)
    n = len(pm)
    eps = float(np.float32(DUAL_SOFTENING) * np.float32(DUAL_SOFTENING))
    stream = torch.cuda.Stream(device)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=device)
    with torch.cuda.stream(stream):
        s = nb.OctupoleImplicitLinearBVHFMMSolver(bodies=pm, velocities=vel, rule=nb.Gravity(1.0, eps),
                                                  theta=DUAL_THETA, max_leaf_size=DUAL_LEAF, time_step=DT,
                                                  device=device)
        s.set_stream(stream.cuda_stream)
        fp64_min = DUAL_FP64_SUMMARIES if args.fp64_summaries is None else args.fp64_summaries
        # accuracy of the first force pass vs FP64 direct summation, with the FP32 top-level
        # summaries of the reference for comparison
        rng = np.random.default_rng(65536)
        idx = np.sort(rng.choice(n, min(65536, n), replace=False))
        dpm = torch.from_numpy(pm).to(device)
        dt_ = torch.from_numpy(pm[idx].copy()).to(device)
        out = torch.zeros((len(idx), 3), dtype=torch.float64, device=device)
        s.direct_device(n, dpm.data_ptr(), len(idx), dt_.data_ptr(), out.data_ptr(), 64)
        s.synchronize()
        ref = out.cpu().numpy()
        del dpm, dt_, out
        rel32 = None
        if fp64_min > 0:
            got32 = s.update_accelerations()[idx, :3].astype(np.float64)
            rel32 = np.linalg.norm(got32 - ref, axis=1) / np.linalg.norm(ref, axis=1)
        s.set_fp64_summaries(fp64_min)
        acc = s.update_accelerations()
        counts = s.counts()
        got = acc[idx, :3].astype(np.float64)
        rel = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
        abs_rms = float(np.sqrt(np.mean(np.sum((got - ref) ** 2, axis=1))))
        for _ in range(max(args.warmup, 3)):
            flush.zero_()
            s.step(1)
        s.enable_timing(True)
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        torch.cuda.synchronize(device)
        with Clocks(device) as clk:
            for k in range(args.steps):
                flush.zero_()
                starts[k].record(stream)
                s.step(1)
                ends[k].record(stream)
            torch.cuda.synchronize(device)
        step_ms = float(sum(a.elapsed_time(b) for a, b in zip(starts, ends)))
        phases = s.phase_times()
        s.close()
    passes = max(int(phases["passes"]), 1)
    trav_ms = phases["traverse_ms"] / passes
    flops = (counts["particle_particle"] * DUAL_PAIR_FLOPS + counts["node_particle"] * DUAL_NP_FLOPS +
             counts["particle_node"] * DUAL_PN_FLOPS + counts["node_node"] * DUAL_NN_FLOPS)
    clk = clk.summary()
    sm_mhz = clk.get("sm_mhz") or 1965.0
    peak = NUM_SMS * FP32_FLOP_PER_CLK_PER_SM * sm_mhz * 1e6 / 1e12
    achieved = flops / (trav_ms / 1000.0) / 1e12
    value = n * args.steps / (step_ms / 1000.0)
    line = {
        "metric": "body-steps/s, 2 x 2^21 colliding Hernquist spheres, dual tree (octupole, field order 4), "
                  "theta=0.4",
        "value": value, "unit": "body-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": step_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded Hernquist spheres)",
        "config": {"workload": f"dual-hernquist-2x{half}-octupole", "n_bodies": n, "theta": DUAL_THETA,
                   "leaf_size": DUAL_LEAF, "softening": DUAL_SOFTENING, "dt": DT,
                   "solver": "implicit-linear-bvh-fmm-8p", "l2": "flushed (256 MB write) before every timed step",
                   "summaries": f"FP32, FP64 combination for nodes of at least {fp64_min} bodies" if fp64_min
                   else "FP32 (the reference's operations)"},
        "accuracy": {"force_rms_rel": float(np.sqrt(np.mean(rel ** 2))), "force_max_rel": float(rel.max()),
                     "force_rms_abs": abs_rms, "sample_targets": int(len(idx)),
                     "reference": "FP64 direct sum on GPU",
                     "fp64_summaries_min_bodies": fp64_min,
                     "force_rms_rel_fp32_summaries": None if rel32 is None else float(np.sqrt(np.mean(rel32 ** 2)))},
        "interactions": counts,
        "roofline": {"bound": "fp32",
                     "kernel": "traversal phase: dual_kernel<0>, dual_kernel<1> (tasks) and near_kernel (near field)",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "flops_per_launch": flops, "ms_per_launch": trav_ms,
                     "peak_source": f"148 SMs x 256 FP32 flop/clk x {sm_mhz:.0f} MHz measured under load"},
        "phases_ms_per_step": {k: phases[k] / passes for k in
                               ("bbox_ms", "morton_ms", "sort_ms", "gather_ms", "build_ms", "traverse_ms",
                                "integrate_ms")},
        "gpu_launches": int(phases["launches"]),
        "clocks": clk,
    }
    if args.emulate_ranks > 1:
        make = lambda: nb.OctupoleImplicitLinearBVHFMMSolver(rule=nb.Gravity(1.0, eps), theta=DUAL_THETA,
                                                             max_leaf_size=DUAL_LEAF, time_step=DT, device=device)
        line["emulated_target_shards"] = shard_emulation(
            nb, torch, make, pm, vel, args.emulate_ranks, device,
            sum(phases[k] for k in phases if k.endswith("_ms") and k != "integrate_ms") / passes)
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = dual_cpu_baseline(1 << 16, eps)
    if rank == 0:
        print(json.dumps(line), flush=True)


def shard_emulation(nb, torch, make, pm, vel, world, device, unsharded_ms):
    """Each of `world` target shards' force pass (nb_set_shard(r, world)) run alone on this GPU,
    device time per pass. A rank of a real run takes its pass plus the all-gather of its chunk of
    positions and velocities over NVLink, which this does not include."""
    n = len(pm)
    chunk, _, _ = nb.shard_range(n, 0, world)
    per_rank = []
    for r in range(world):
        s = make()
        try:
            s.set_shard(r, world)
            s.set_bodies(pm, vel)
            s.update_accelerations_async()  # sizes the pools for this shard
            s.synchronize()
            s.enable_timing(True)
            s.update_accelerations_async()
            t = s.phase_times()
            per_rank.append(sum(v for k, v in t.items() if k.endswith("_ms")) / max(t["passes"], 1))
        finally:
            s.close()
        torch.cuda.synchronize(device)
    worst = max(per_rank)
    return {"ranks": world, "force_pass_ms_per_rank": per_rank, "max_ms": worst,
            "unsharded_force_pass_ms": unsharded_ms, "speedup_of_slowest_rank": unsharded_ms / worst,
            "allgather_bytes_per_rank": 32 * chunk * (world - 1),
            "method": "each shard's force pass run alone on one GPU (device time, sort and build over all "
                      "bodies included); the all-gather over NVLink is not included"}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batched":
        run_batched(args)
    elif args.workload == "serving":
        run_serving(args)
    elif args.workload == "dual-4m":
        run_dual(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
