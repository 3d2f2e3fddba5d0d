"""Benchmark of the CUDA cloth step: sim steps/s on the floor-drape workload.

python bench.py --gpus N --steps K --warmup W [--impl cuda|reference]
                [--workload floor_drape|strip_pull|sphere_drape|batch_sheets|material_fit]
                [--precision fp64|mixed|both]
                [--skip S]   # S extra untimed steps before timing (e.g. to reach contact)

One process per GPU (torchrun for N > 1); every rank steps its own replica of
the workload (a single sheet does not shard: "replicas only", weak scaling).
Timing: per step, L2 is flushed (a 256 MiB write on the solver's stream), then
the step is bracketed by CUDA events on the solver's stream; the reported
time is the max over ranks. rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

HBM_FALLBACK_GBS = 6650.0


def max_over_ranks(values, device, world):
    """Max of each timing over all ranks (the job is as slow as its slowest
    replica); identity when world == 1."""
    import torch
    import torch.distributed as dist
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def replica_throughput(world, steps, ms):
    """Whole-job steps/s of `world` independent replicas that each ran `steps`
    steps, timed as the slowest rank's `ms`."""
    return world * steps / (ms / 1000.0)


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.dev)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        # nvidia-smi's start-up (NVML initialization) can stall the GPU's
        # clients for tens of ms: wait for its first sample, so the start-up
        # falls before the warm-up steps that follow, not inside timed steps.
        t0 = time.time()
        while not self.lines and time.time() - t0 < 10 and self.proc.poll() is None:
            time.sleep(0.01)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def workload(name: str, steps_hint: int):
    from closim_b200 import configs
    if name == "floor_drape":
        return configs.floor_drape()
    if name == "strip_pull":
        return configs.strip_pull()
    if name == "sphere_drape":
        return configs.sphere_drape()
    raise SystemExit(f"unknown workload {name}")


def cpu_baseline(cfg, budget_s: float, max_steps: int):
    """The oracle (single-threaded C++ port of the reference CpuSolver) on a
    bounded sample: the first steps of the same workload, up to budget_s."""
    from tests.helpers import oracle_scene, oracle_step_kwargs
    from closim_b200 import configs
    sc = oracle_scene(cfg)
    kw = oracle_step_kwargs(cfg)
    t0 = time.perf_counter()
    k = 0
    while k < max_steps:
        sc.set_pins(configs.pins_at(cfg, k))
        sc.step(cfg["h"], **kw)
        k += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return {"value": k / dt, "unit": "steps/s", "cores": 1, "kind": "port",
            "sample": f"first {k} steps of {cfg['name']} ({dt:.1f} s, 1 thread)"}


def run_reference(args, rank):
    if rank != 0:
        return 0
    cfg = workload(args.workload, args.steps)
    from oracle import oracle as O
    O.lib()
    per = []
    for i in range(args.warmup + args.steps):
        b = cpu_baseline(cfg, budget_s=max(5.0, 60.0 / max(1, args.warmup + args.steps)), max_steps=cfg["steps"])
        if i >= args.warmup:
            per.append(b["value"])
    v = statistics.mean(per)
    line = {"metric": "sim steps/s", "value": v, "unit": "steps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "impl": "reference", "scaling": "weak",
            "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": cfg["name"], "n": len(cfg["x"]) // 3, "h": cfg["h"]},
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": 1, "kind": "port", "sample": b["sample"]},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "vs_baseline": None}
    print(json.dumps(line), flush=True)
    return 0


def step_algorithmic_bytes(st, mesh, precision, cfg):
    """Algorithmic bytes of one step from its measured counts (Newton
    iterations, PCG iterations, Armijo trials, contacts): per Newton iteration a
    gradient pass, per PCG iteration an HVP and the vector updates, per trial an
    energy pass, and per broadphase query the boxes, sort passes and nodes; f is
    the PCG vector width (4 mixed, 8 FP64), constants 4 B, 64 B per frozen
    contact record, 48 B per CCD candidate primitive."""
    f = 4 if precision == "mixed" else 8
    n, m, hg = mesh.count, mesh.triCount, mesh.hinges.shape[0]
    c = st.contact["activePairs"] if st.contact else 0
    cand = st.contact["candidatePairs"] if st.contact else 0
    D = (n + 7) // 8 if cfg["options"]["precond"] == "schwarz" else 0
    b_grad = (9 * f + 4) * n + 32 * m + (16 + 3 * f) * hg + 64 * c
    b_e = (6 * f + 4) * n + 32 * m + (16 + 3 * f) * hg + 64 * c
    b_hvp = (9 * f + 4) * n + 32 * m + 64 * c
    b_vec = 24 * f * n + D * 300 * 4
    newton = max(st.newtonItersUsed, 1)
    trials = st.armijoTrials
    b = newton * b_grad + st.pcgIters * (b_hvp + b_vec) + trials * b_e
    if st.contact:
        queries = newton + trials + 2
        b += queries * (6 * f * n + 12 * m + 24 * m + 8 * m + 2 * 8 * m * 4 + 2 * m * 40) + trials * 48 * cand
    return float(b)


def pcg_kernel_name(precision, prof):
    if precision != "mixed":
        return "k_pcg"
    info = prof.get("launch_info") or {}
    return "k_mx_pcg_cluster" if info.get("pcgClusterCtas") else "k_mx_pcg"


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of
# the headline PCG kernel on the 64x64 floor drape, from one ncu --set full
# capture; the command and the other counters are in
# profiles/k_mx_pcg_cluster_floor_drape_64x64.md.
PCG_DRAM_BYTES = {"k_mx_pcg_cluster": 3.418e6}


def run_precision(cfg, precision, local, args, ext_stream_cb, flush, sampler=None, prof_out=None):
    """Warm-up W steps, then K device-resident steps, each bracketed by CUDA
    events on the solver's stream after an L2 flush. Returns (ms_total, solver,
    scene, final positions, kernel launches)."""
    import torch
    import closim_b200 as cb
    from closim_b200 import configs
    sc = configs.make_scene(cfg)
    solver = cb.CudaSolver(precision, device=local, **cfg["options"])
    solver.initialize(sc)
    ext = torch.cuda.ExternalStream(solver.stream(), device=local)
    k = [0]

    def set_pins():
        sc.pinned.clear()
        sc.pinned.update(configs.pins_at(cfg, k[0] % cfg["steps"]))
        k[0] += 1

    if sampler:
        sampler.start()  # before the warm-up steps (see ClockSampler.start)
    for _ in range(args.warmup + args.skip):
        set_pins()
        solver.advance(cfg["h"], 1)
    torch.cuda.synchronize()
    ext_stream_cb()
    launches0 = solver.kernelLaunches()
    if args.profiler_range:
        torch.cuda.profiler.start()  # ncu --profile-from-start off captures the timed steps only
    solver.profile(True)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    total = 0.0
    step_bytes = 0.0
    mesh = configs.make_scene(cfg).mesh
    for _ in range(args.steps):
        set_pins()
        with torch.cuda.stream(ext):
            flush.fill_(1.0)
        ev0.record(ext)
        solver.advance(cfg["h"], 1)
        ev1.record(ext)
        ev1.synchronize()
        total += ev0.elapsed_time(ev1)
        step_bytes += step_algorithmic_bytes(solver.lastStats, mesh, precision, cfg)
    torch.cuda.synchronize()
    if args.profiler_range:
        torch.cuda.profiler.stop()
    if prof_out is not None:
        prof_out.update(solver.profileRead())
    solver.profile(False)
    launches = solver.kernelLaunches() - launches0
    if prof_out is not None:
        prof_out["launch_info"] = solver.launchInfo()
        prof_out["step_bytes"] = step_bytes
    if prof_out is not None and args.phase_steps > 0:
        # wall-time breakdown over a few extra (untimed) steps
        solver.profile(True, phases=True)
        for _ in range(args.phase_steps):
            set_pins()
            solver.advance(cfg["h"], 1)
        torch.cuda.synchronize()
        prof_out["phases_ms_per_step"] = {k: v / args.phase_steps for k, v in solver.profilePhases().items()}
        solver.profile(False)
    solver.pull()
    return total, solver, sc, sc.positions.copy(), launches, ext, set_pins


def run_batch(args, world, rank, local):
    """512 uneven sheets stepped by the batched solver: one persistent launch
    per step, K steps graph-replayed; value = whole-job sheet-steps/s."""
    import torch
    import torch.distributed as dist
    from closim_b200 import configs
    from closim_b200.batch import BatchSolver
    sheets = configs.batch_sheets(count=args.sheets)
    h = sheets[0]["h"]
    bs = BatchSolver(sheets, device=local)
    threads = bs.autotune(h)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")
    ext = torch.cuda.ExternalStream(bs.stream(), device=local)
    sampler = ClockSampler(local)
    sampler.start()  # before the warm-up steps (see ClockSampler.start)
    bs.step(h, args.warmup)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    total = 0.0
    for _ in range(args.steps):
        with torch.cuda.stream(ext):
            flush.fill_(1.0)
        ev0.record(ext)
        bs.step(h)
        ev1.record(ext)
        ev1.synchronize()
        total += ev0.elapsed_time(ev1)
    clocks = sampler.stop()
    # graph-replayed multi-step call (the production path)
    ev0.record(ext)
    bs.step(h, args.steps)
    ev1.record(ext)
    ev1.synchronize()
    graph_ms = ev0.elapsed_time(ev1)
    st = bs.stats()
    # the same sheets stepped one by one by the single-sheet mixed solver (a
    # sample of 8, scaled to the batch by triangle count)
    import closim_b200 as cb
    sample = sheets[:: max(1, len(sheets) // 8)][:8]
    single_ms, single_m = 0.0, 0
    for cfg in sample:
        sc = configs.make_scene(dict(cfg, contact=None))  # no self-contact search in the comparison
        so = cb.CudaSolver("mixed", device=local, **dict(cfg["options"], precond="jacobi"))
        so.initialize(sc)
        so.advance(h, 2)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        so.advance(h, 3)
        torch.cuda.synchronize()
        single_ms += (time.perf_counter() - t0) * 1000.0 / 3
        single_m += len(cfg["idx"]) // 3
        so.close()
    total_m = int(sum(len(c["idx"]) // 3 for c in sheets))
    single_est_ms = single_ms * total_m / max(single_m, 1)
    total, graph_ms = max_over_ranks([total, graph_ms], f"cuda:{local}", world)
    if rank == 0:
        S = len(sheets)
        line = {"metric": "sim steps/s", "value": replica_throughput(world, args.steps, total), "unit": "steps/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
                "data": "synthetic (seeded)", "impl": "cuda",
                "config": {"workload": "batch_sheets", "sheets": S, "n": bs.N,
                           "m": int(sum(len(c["idx"]) // 3 for c in sheets)), "h": h,
                           "parallelism": f"replicas x{world}", "threads_per_sheet": threads,
                           "resident_blocks": bs.launchShape()["blocks"],
                           "l2": "flushed between timed steps (256 MiB write)"},
                "sheet_steps_per_s": world * S * args.steps / (total / 1000.0),
                "graph_replay": {"steps": args.steps, "ms_per_step": graph_ms / args.steps},
                "converged_sheets_last_step": int(sum(1 for x in st if x["converged"] == 1)),
                "mean_newton_iters": float(np.mean([x["newtonIters"] for x in st])),
                "mean_pcg_iters": float(np.mean([x["pcgIters"] for x in st])),
                "single_sheet_solver_ms_per_batch_step": single_est_ms,
                "single_sheet_solver_note": "8 sheets stepped one by one by the single-sheet mixed solver (Jacobi, "
                                            "no contact), scaled to the batch by triangle count",
                "speedup_vs_single_sheet_solver": single_est_ms / (total / args.steps),
                "gpu_launches": 2 * args.steps, "clocks": clocks}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_material_fit(args, world, rank, local):
    """Adjoint cost: a rollout of the material-fit sheet (96 x 96, exact-Newton
    forward, checkpoints every 20 steps) and its backward; value = forward
    sim steps/s, plus the backward / forward time ratio."""
    import torch
    import closim_b200 as cb
    from closim_b200 import configs
    cfg = configs.material_fit(steps=args.rollout_steps, grad_tol=1e-9)
    sc = configs.make_scene(cfg)
    s = cb.CudaSolver("fp64", device=local, **cfg["options"])
    s.initialize(sc)
    s.setNewtonMode("exact", 1e-8)
    s.setAdjointOptions(4000, 1e-10)
    x0 = sc.positions.copy()
    ext = torch.cuda.ExternalStream(s.stream(), device=local)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record(ext)
    xN = s.forward(cfg["h"], cfg["steps"], cfg["checkpoint_every"]).copy()
    ev[1].record(ext)
    fwd_conv = s.adjointStats()["forwardConverged"]
    gx = 2 * (xN - x0) / (len(x0) // 3)
    dth, dv0 = s.backward(gx)
    ev[2].record(ext)
    ev[2].synchronize()
    f_ms = ev[0].elapsed_time(ev[1])
    b_ms = ev[1].elapsed_time(ev[2])
    st = s.adjointStats()
    if rank == 0:
        line = {"metric": "sim steps/s", "value": cfg["steps"] / (f_ms / 1000.0), "unit": "steps/s", "n_gpus": 1,
                "steps": cfg["steps"], "warmup": 0, "ms_per_step": f_ms / cfg["steps"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "impl": "cuda",
                "config": {"workload": "material_fit", "n": len(x0) // 3, "m": len(cfg["idx"]) // 3,
                           "checkpoint_every": cfg["checkpoint_every"], "newton": "exact, gradTol 1e-9"},
                "adjoint": {"backward_ms": b_ms, "forward_ms": f_ms, "backward_over_forward": b_ms / f_ms,
                            "forward_converged_steps": fwd_conv, "adjoint_pcg_iters": st["pcgIters"],
                            "max_rel_residual": st["maxRelResidual"],
                            "dL_dtheta": [dth["C00"], dth["C11"], dth["G"], dth["kBend"]]}}
        print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cuda", choices=["cuda", "reference"])
    ap.add_argument("--workload", default="floor_drape",
                    choices=["floor_drape", "strip_pull", "sphere_drape", "batch_sheets", "material_fit"])
    ap.add_argument("--rollout-steps", type=int, default=40, help="material_fit: steps of the timed rollout")
    ap.add_argument("--sheets", type=int, default=512, help="batch_sheets: number of sheets (512 in the workload)")
    ap.add_argument("--skip", type=int, default=0, help="extra untimed steps before the timed region")
    ap.add_argument("--phase-steps", type=int, default=3, help="extra steps for the per-phase wall-time breakdown")
    ap.add_argument("--small", action="store_true", help="32x32 floor drape (for profiler captures)")
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profiler-range", action="store_true",
                    help="mark the timed steps for ncu --profile-from-start off")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)

    import torch
    import torch.distributed as dist
    import datetime
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from closim_b200 import configs
    if args.workload == "batch_sheets":
        return run_batch(args, world, rank, local)
    if args.workload == "material_fit":
        return run_material_fit(args, world, rank, local)
    if args.small:
        cfg = configs.floor_drape(nx=31, ny=31, w=0.4, hgt=0.4)
    else:
        cfg = workload(args.workload, args.steps)
    n = len(cfg["x"]) // 3
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")  # 256 MiB > 126 MB L2

    def barrier():
        if world > 1:
            dist.barrier()

    headline = "mixed" if args.precision in ("both", "mixed") else "fp64"
    res = {}
    if args.precision in ("both", "fp64"):
        t, _, _, pos, la, _, _ = run_precision(cfg, "fp64", local, args, barrier, flush)
        res["fp64"] = dict(ms=t, pos=pos, launches=la)
    sampler = ClockSampler(local)
    prof = {}
    t, solver, sc, pos, la, ext, set_pins = run_precision(cfg, headline, local, args, barrier, flush, sampler, prof)
    clocks = sampler.stop()
    res[headline] = dict(ms=t, pos=pos, launches=la)

    # ---- end to end through the public API: host state in, host state out ----
    px = torch.empty(n * 3, dtype=torch.float64).pin_memory()
    pv = torch.empty(n * 3, dtype=torch.float64).pin_memory()
    px.numpy()[:] = sc.positions
    pv.numpy()[:] = sc.velocities
    sc.positions = px.numpy()
    sc.velocities = pv.numpy()
    solver.syncFromScene = True
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    e2e_ms = 0.0
    e_steps = max(3, args.steps // 2)
    for _ in range(e_steps):
        set_pins()
        ev0.record(ext)
        solver.step(cfg["h"])
        ev1.record(ext)
        ev1.synchronize()
        e2e_ms += ev0.elapsed_time(ev1)
    h2d = 2 * n * 3 * 8 + len(sc.pinned) * (4 + 24)
    d2h = 2 * n * 3 * 8

    times = [res[headline]["ms"], e2e_ms, res.get("fp64", {}).get("ms", 0.0)]
    total_ms, e2e_ms, fp64_ms = max_over_ranks(times, f"cuda:{local}", world)
    if world > 1:
        dist.barrier()
    value = replica_throughput(world, args.steps, total_ms)
    e2e_value = replica_throughput(world, e_steps, e2e_ms)

    if rank == 0:
        peak, peak_kind = measured_peak()
        achieved = (prof["bytes"] / prof["launches"] / (prof["ms_per_launch"] / 1000.0) / 1e9
                    if prof.get("launches") else 0.0)
        line = {
            "metric": "sim steps/s", "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if headline == "mixed" else "f64",
            "data": "synthetic (seeded)", "impl": "cuda",
            "config": {"workload": cfg["name"] + ("_32x32" if args.small else ""), "n": n, "m": len(cfg["idx"]) // 3,
                       "h": cfg["h"], "precision": headline, "precond": cfg["options"]["precond"],
                       "parallelism": f"replicas x{world}", "l2": "flushed between timed steps (256 MiB write)"},
            "roofline": {"bound": "hbm", "kernel": pcg_kernel_name(headline, prof),
                         "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": PCG_DRAM_BYTES.get(pcg_kernel_name(headline, prof))
                         if cfg["name"] == "floor_drape" and not args.small else None,
                         "traffic_source": "profiles/k_mx_pcg_cluster_floor_drape_64x64.md (one ncu capture)",
                         "launches": prof.get("launches"),
                         "ms_per_launch": prof.get("ms_per_launch"), "pcg_iters": prof.get("iters"),
                         "alg_bytes_per_launch": prof["bytes"] / max(1, prof["launches"]) if prof else None,
                         "share_of_step": prof["ms"] / total_ms if total_ms and prof else None},
            "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": res[headline]["launches"],
            "clocks": clocks,
            "phases_ms_per_step": prof.get("phases_ms_per_step"),
            "step_roofline": {"bound": "hbm", "alg_bytes_per_step": prof.get("step_bytes", 0.0) / args.steps,
                              "achieved": prof.get("step_bytes", 0.0) / (total_ms / 1000.0) / 1e9,
                              "peak": measured_peak()[0], "unit": "GB/s",
                              "frac": prof.get("step_bytes", 0.0) / (total_ms / 1000.0) / 1e9 / measured_peak()[0]},
            "launch_info": prof.get("launch_info"),
        }
        if args.skip:
            line["config"]["untimed_steps_before"] = args.warmup + args.skip
        if "fp64" in res and headline == "mixed":
            a, b = res["fp64"]["pos"], res["mixed"]["pos"]
            line["fp64_path"] = {"value": world * args.steps / (fp64_ms / 1000.0), "unit": "steps/s",
                                 "ms_per_step": fp64_ms / args.steps,
                                 "gpu_launches": res["fp64"]["launches"]}
            line["mixed_vs_fp64_rel_pos_err"] = float(np.max(np.abs(b - a)) / np.max(np.abs(a)))
            line["mixed_vs_fp64_steps"] = args.warmup + args.skip + args.steps
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(cfg, budget_s=20.0, max_steps=cfg["steps"])
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
