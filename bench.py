"""Benchmark of the B200 IISPH step: particle-updates/s on the 1,000,000-particle dam break.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One step = one full IISPH time step (neighbor build, density, non-pressure, source/diagonal,
relaxed-Jacobi loop to the density-error target, pressure acceleration, integration) of the
100^3 dam break (dx = 0.01 m, 5 x 2 x 2 m tank, 2 wall layers, dt = 5e-4 s, omega = 0.5,
2..100 iterations, average positive density error <= 0.1 %), seeded +-0.01 dx jitter. The
working set (~0.3 GB) is larger than L2, so no flush is needed between steps.

value: fluid particles x steps / device time (CUDA events on the backend stream, timed region
bracketed by a barrier and device synchronisation, max over ranks). The K timed steps run as one
tsp_b200_step(h, p, K) call (the interface's N_steps); p50/p99 come from the backend's per-step
history (tsp_b200_get_step_history), the phase split from 20 further steps. Multi-GPU:
independent replicas (one scene per GPU, no inter-GPU traffic) -> weak scaling.
developed: the same run continued to step 1,000 (the collapse under way, more Jacobi sweeps per
step), then 20 steps timed the same way.
tuned: the autotuner's launch configurations (tune.cu), chosen during the first warm-up step.
other_configs: the 32K dam for its 1,000 steps, the 2M-fluid rigid dam (50 steps) and the
neighbor-search-only builds at 1M / 4M points, uniform and clustered (--no-configs skips them).
e2e: the same metric through the C ABI with pinned host buffers: per step pull_state (H2D of
the step's particle state) + step + push_state (D2H of positions, velocities, pressure,
density).
served: the seeded mixed-size served stream (continuous batching, turbospharticles_b200.serve;
256 scenes x 500 steps, the full stream, by default; --served-scenes 0 skips it) against the
same scenes one at a time on the plain one-scene path for the same 500 steps each, both
device-timed; value_wall is the served loop's host wall clock (admission, relayout and
read-back included).
--impl reference: the CPU restatement of the reference step (oracle/, OpenMP over all host
threads) on the same workload; the reference's own CPU backend cannot be built here.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-updates/s @1M (plain vs served batch, same B200); p50/p99 step ms"
UNIT = "particle-updates/s"


from turbospharticles_b200.replicas import (dist_env, init as init_dist_group, barrier, max_over_ranks,
                                            aggregate_rate, replica_seed)


def init_dist(ws, backend):
    return init_dist_group(backend, ws)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 100 ms; sampling starts before the
    timed region (the first sample is awaited) and only samples received inside the region
    (`mark_start` .. `mark_end`, plus one interval of read-out lag) are summarised."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    INTERVAL_S = 0.1

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", str(int(self.INTERVAL_S * 1000))], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            deadline = time.perf_counter() + 3.0
            while not self.rows and time.perf_counter() < deadline:
                time.sleep(0.01)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append((time.perf_counter(), [x.strip() for x in line.split(",")]))

    def mark_start(self):
        self.t0 = time.perf_counter()

    def mark_end(self):
        self.t1 = time.perf_counter()
        time.sleep(self.INTERVAL_S * 1.5)  # let the sample covering the end arrive

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        lo = self.t0 if self.t0 is not None else float("-inf")
        hi = (self.t1 + self.INTERVAL_S) if self.t1 is not None else float("inf")
        inside = [r for t, r in self.rows if lo <= t <= hi]
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        rows = inside
        sm = [float(r[1]) for r in rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows if len(r) >= 9 for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes (read + write) of one KJacobi launch on this workload, from the ncu summary
    committed beside the kernel's profile (line `traffic_bytes_per_launch = N`)."""
    p = os.path.join(ROOT, "profiles", "KJacobi_iisph_dam_1M.md")
    try:
        with open(p) as f:
            for line in f:
                if line.strip().startswith("traffic_bytes_per_launch"):
                    return {"bytes_per_launch_scaled": int(line.split("=")[1].strip().split()[0])}
    except (OSError, ValueError, IndexError):
        pass
    return None


def profiled_issue(name="KJacobi_iisph_dam_1M.md",
                   keys=("issue_active_pct", "l1_wavefronts_pct_of_peak", "warp_instructions_per_pair_slot")):
    """Issue and L1 figures of a kernel from its committed ncu summary (lines `key = value`):
    what bounds it besides HBM."""
    p = os.path.join(ROOT, "profiles", name)
    out = {}
    try:
        with open(p) as f:
            for line in f:
                t = line.strip()
                for key in keys:
                    if t.startswith(key + " "):
                        out[key] = float(t.split("=")[1].strip().split()[0])
    except (OSError, ValueError, IndexError):
        pass
    return out or None


def cpu_description():
    """Host CPU model and the widest x86 SIMD extension it reports (for the CPU baselines)."""
    model, flags = None, set()
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name") and model is None:
                    model = line.split(":", 1)[1].strip()
                elif line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    break
    except OSError:
        pass
    simd = "avx512f" if "avx512f" in flags else "avx2" if "avx2" in flags else "sse4_2" if "sse4_2" in flags else None
    return {"cpu_model": model, "simd": simd}


DEVELOPED_AT = 1000
DEVELOPED_STEPS = 20
PHASE_SAMPLE = 20  # steps after the timed region whose per-phase device times give phase_ms_p50


def build_workload(rank=0):
    from turbospharticles_b200 import scene as S
    st, dmin, dmax, p = S.dam_1m(seed=replica_seed(42, rank))
    return st, dmin, dmax, p


def pinned_state(st):
    """Copy of a UniversalSimState whose arrays live in pinned (page-locked) host memory."""
    import torch
    out = st.copy()
    for k, v in st.arrays().items():
        t = torch.empty(v.shape, dtype=getattr(torch, str(v.dtype)) if v.dtype != np.uint64 else torch.int64,
                        pin_memory=True)
        a = t.numpy().view(v.dtype)
        a[...] = v
        setattr(out, k, a)
        out.__dict__.setdefault("_pins", []).append(t)
    return out


def run_b200(args):
    import torch
    from turbospharticles_b200 import abi
    from turbospharticles_b200.backend import SimBackendB200

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = init_dist(ws, "nccl")
    if args.tuning:
        with open(args.tuning) as f:
            abi.pin_tuning(json.load(f), local)
    for spec in args.pin or []:  # KERNEL:SLOTS:MINBLOCKS at every particle count
        kernel, slots, mb = spec.split(":")
        abi.pin_tuning({f"{kernel}/n{1 << k}": {"slots": int(slots), "min_blocks": int(mb)} for k in range(22)}, local)
    dev = torch.device("cuda", local)
    st, dmin, dmax, p = build_workload(rank)
    be = SimBackendB200(p, device=local)
    be.set_sim_domain_bounds(dmin, dmax)
    be.pull(st, p)
    be.run_stage(abi.STAGE_BOUNDARY_VOLUMES, p)
    stream = torch.cuda.ExternalStream(be.stream_handle(), device=dev)
    for _ in range(args.warmup):
        be.step(p)  # the first step also runs the autotuner (tune.cu) for this size class
    tuned = abi.tuning(local)
    # ---- device-timed region (clock sampling already running when it starts)
    # K steps in one tsp_b200_step call (the interface's N_steps); each step's device time and
    # iteration count come from the backend's step history after the region
    with ClockSampler(local) as clk:
        barrier(dist, dev)
        torch.cuda.synchronize(dev)
        l0 = be.launch_count()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        clk.mark_start()
        e0.record(stream)
        be.step(p, args.steps)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        clk.mark_end()
    barrier(dist, dev)
    elapsed_ms = max_over_ranks(dist, e0.elapsed_time(e1), dev)
    launches = be.launch_count() - l0
    hist = be.step_history(args.steps)
    step_ms = [r["ms"] for r in hist]
    iters = [r["solverIters"] - 1 for r in hist]
    # phase split: PHASE_SAMPLE further steps, one call each, phase times read after each
    phases = []
    for _ in range(PHASE_SAMPLE):
        be.step(p)
        phases.append(be.phase_times())
    nF = st.N_F
    value = aggregate_rate(nF * args.steps, ws, elapsed_ms)
    sweeps = int(np.sum(iters))
    # ---- roofline of the dominant kernel: the relaxed-Jacobi sweep (KJacobi)
    s = be.stats()
    L = s.sellPackedBytes / nF + 6.0
    bytes_per_particle = 32.0 + L + 4.0
    jac_ms = be.time_stage(abi.STAGE_JACOBI_UPDATE, reps=20, params=p)
    pacc_ms = be.time_stage(abi.STAGE_PRESSURE_ACC, reps=20, params=p)
    phase_p50 = {k: float(np.median([ph[k] for ph in phases if k in ph])) for k in (phases[-1] if phases else {})}
    largest = max(phase_p50, key=phase_p50.get) if phase_p50 else None
    achieved = bytes_per_particle * nF / (jac_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    traffic = profiled_traffic()
    roof = {"kernel": "KJacobi (relaxed Jacobi sweep + FP64 residual reduction)", "bound": "hbm",
            "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "peak_source": peak_kind, "traffic": (traffic or {}).get("bytes_per_launch_scaled"),
            "algorithmic_bytes_per_launch": int(bytes_per_particle * nF), "ms_per_launch": round(jac_ms, 4),
            "pressure_acc_ms_per_launch": round(pacc_ms, 4),
            "bytes_per_particle": round(bytes_per_particle, 2), "list_bytes_per_particle": round(L, 2),
            "issue": profiled_issue(),
            "largest_phase_of_window": {"phase": largest, "p50_ms": round(phase_p50.get(largest, 0.0), 4)}}
    # the neighbor build of a step (keys, sort, reorder, cell tables, count, finalize, fill) against
    # the same peak: algorithmic bytes per particle keys 24 + sort 24 x passes + reorder 68 + cell
    # table 8 + count 18 + fill 12 + list bytes, time = the build phases' p50 of the phase sample
    nb_phases = ("sort_reorder_tables", "query_count", "finalize_readback", "query_fill")
    if all(k in phase_p50 for k in nb_phases):
        passes = (int(s.keyBits) + 7) // 8
        nb_bpp = 24.0 + 24.0 * passes + 68.0 + 8.0 + 18.0 + 12.0 + L
        nb_ms = sum(phase_p50[k] for k in nb_phases)
        nb_gbs = nb_bpp * nF / (nb_ms * 1e-3) / 1e9
        roof["neighbor_build"] = {
            "phases_ms": {k: round(phase_p50[k], 4) for k in nb_phases}, "ms_per_build": round(nb_ms, 4),
            "bytes_per_particle": round(nb_bpp, 2), "sort_passes": passes, "achieved": round(nb_gbs, 1),
            "frac": round(nb_gbs / peak, 4), "bound": "SM issue (count pass: ~216 candidate tests per particle)",
            "count_pass": profiled_issue("KQueryFluid_iisph_dam_1M.md",
                                         ("count_issue_active_pct", "count_warps_active_pct"))}
    # ---- developed flow: the same run continued to step DEVELOPED_AT (the collapse under way,
    # more Jacobi sweeps per step), then DEVELOPED_STEPS steps timed the same way
    developed = None
    if not args.no_developed:
        done = args.warmup + args.steps + PHASE_SAMPLE
        if DEVELOPED_AT > done:
            be.step(p, DEVELOPED_AT - done)
        barrier(dist, dev)
        torch.cuda.synchronize(dev)
        e4 = torch.cuda.Event(enable_timing=True)
        e5 = torch.cuda.Event(enable_timing=True)
        e4.record(stream)
        be.step(p, DEVELOPED_STEPS)
        e5.record(stream)
        torch.cuda.synchronize(dev)
        dev_ms = max_over_ranks(dist, e4.elapsed_time(e5), dev)
        dh = be.step_history(DEVELOPED_STEPS)
        d_ms = [r["ms"] for r in dh]
        d_it = [r["solverIters"] - 1 for r in dh]
        dq = np.percentile(d_ms, [50, 99])
        developed = {"from_step": max(DEVELOPED_AT, done), "steps": DEVELOPED_STEPS, "unit": UNIT,
                     "value": round(aggregate_rate(nF * DEVELOPED_STEPS, ws, dev_ms), 1),
                     "p50_step_ms": round(float(dq[0]), 4), "p99_step_ms": round(float(dq[1]), 4),
                     "jacobi_sweeps_per_step": round(float(np.mean(d_it)), 2)}
    # ---- end to end through the C ABI with pinned host buffers
    e2e = None
    if not args.no_e2e:
        host = pinned_state(be.push())
        out = pinned_state(be.push())
        for n in ("xVelPredF", "yVelPredF", "zVelPredF", "xAccPressF", "yAccPressF", "zAccPressF",
                  "sourceTermF", "diagElemF"):
            setattr(out, n, np.zeros(0, np.float32))
            setattr(host, n, np.zeros(0, np.float32))
        h2d = host.N_F * (8 + 12 + 12 + 4 + 4) + host.N_B * (8 + 12 + 4 + 4)
        d2h = host.N_F * (8 + 12 + 12 + 4 + 4) + host.N_B * (8 + 12 + 4 + 4)
        barrier(dist, dev)
        torch.cuda.synchronize(dev)
        k_e2e = max(1, min(args.steps, 10))
        e2 = torch.cuda.Event(enable_timing=True)
        e3 = torch.cuda.Event(enable_timing=True)
        e2.record(stream)
        for _ in range(k_e2e):
            be.pull(host, p)
            be.step(p)
            be.push(out)
            host, out = out, host
        e3.record(stream)
        torch.cuda.synchronize(dev)
        e2e_ms = max_over_ranks(dist, e2.elapsed_time(e3), dev)
        e2e = {"value": round(nF * k_e2e * ws / (e2e_ms / 1e3), 1), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "steps": k_e2e,
               "path": "tsp_b200_pull_state + tsp_b200_step + tsp_b200_push_state, pinned host SoA"}
    # ---- CPU baseline: the oracle port on this host, one step from the current GPU state
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_baseline_from(be, p, dmin, dmax)
    # ---- the other configurations of the workload set, timed the same way (device events)
    others = None
    if rank == 0 and ws == 1 and not args.no_configs:
        be.close()
        others = other_configs_measure(torch, dev)
    # ---- served mixed-size stream (continuous batching) vs the same scenes one at a time
    served = None
    if rank == 0 and ws == 1 and args.served_scenes > 0:
        be.close()
        served = served_stream_measure(args.served_scenes, args.served_steps)
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return
    q = np.percentile(step_ms, [50, 99])
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(elapsed_ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 residual and rigid sums)",
        "data": "synthetic (seeded dam-break scene restated from the reference builder)",
        "config": {"workload": "iisph_dam_1M", "n_fluid": nF, "n_boundary": st.N_B, "dx_m": 0.01, "dt_s": 5e-4,
                   "tank_m": [5, 2, 2], "omega": 0.5, "iters": "2..100, avg positive density error <= 0.001",
                   "parallelism": f"replicas x{ws}", "l2": "working set > L2 (126 MB), no flush"},
        "p50_step_ms": round(float(q[0]), 4), "p99_step_ms": round(float(q[1]), 4),
        "jacobi_sweeps": sweeps, "jacobi_iters_per_s": round(sweeps * ws / (elapsed_ms / 1e3), 1),
        "neighbor_ms_last": round(s.lastNeighborMs, 4), "jacobi_ms_last": round(s.lastJacobiMs, 4),
        "phase_ms_p50": {k: round(v, 4) for k, v in phase_p50.items()},
        "phase_sample": f"{PHASE_SAMPLE} steps after the timed region",
        "roofline": roof, "developed": developed, "tuned": tuned, "e2e": e2e, "cpu_baseline": cpu,
        "gpu_launches": int(launches), "clocks": clk.summary(), "other_configs": others, "served": served,
        "impl": "b200",
    }
    print(json.dumps(line), flush=True)


def _timed_steps(torch, dev, be, p, steps):
    stream = torch.cuda.ExternalStream(be.stream_handle(), device=dev)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    be.step(p, steps)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    h = be.step_history(steps)
    return e0.elapsed_time(e1), [r["ms"] for r in h], sum(r["solverIters"] - 1 for r in h)


def other_configs_measure(torch, dev):
    """The workload set's other configurations on this GPU: the 32K dam for its full 1,000
    steps, the full-size rigid dam (2,000,000 fluid, 8 cubes) for 50 steps after 5 warm-up, and
    the neighbor-search-only case (Morton keys, sort, reorder, cell tables, SELL32 count + fill)
    at 1,048,576 and 4,194,304 points, uniform and clustered, 5 builds each after one warm-up
    build; algorithmic bytes of a build per point: keys 24 + sort 24 x passes + reorder of every
    field 68 + cell table 8 + count 18 + fill 12 + list bytes."""
    from turbospharticles_b200 import abi, scene as S
    from turbospharticles_b200.backend import SimBackendB200
    out = {}
    for name, builder, warm, steps in (("iisph_dam_32k_1000_steps", S.dam_32k, 0, 1000),
                                       ("rigid_dam_2M_8_cubes", S.rigid_dam, 5, 50)):
        st, dmin, dmax, p = builder()
        be = SimBackendB200(p)
        be.set_sim_domain_bounds(dmin, dmax)
        be.pull(st, p)
        be.run_stage(abi.STAGE_BOUNDARY_VOLUMES, p)
        if warm:
            be.step(p, warm)
        el, ms, sweeps = _timed_steps(torch, dev, be, p, steps)
        q = np.percentile(ms, [50, 99])
        out[name] = {"n_fluid": st.N_F, "n_boundary": st.N_B, "n_rigid": st.N_R, "steps": steps,
                     "from_step": warm + 1, "value": round(st.N_F * steps / (el / 1e3), 1), "unit": UNIT,
                     "p50_step_ms": round(float(q[0]), 4), "p99_step_ms": round(float(q[1]), 4),
                     "jacobi_sweeps_per_step": round(sweeps / steps, 2)}
        be.close()
    ns = {}
    for n in (1 << 20, 1 << 22):
        for dist in ("uniform", "clustered"):
            st, dmin, dmax, p = S.neighbor_search_scene(n, dist, seed=7)
            be = SimBackendB200(p)
            be.set_sim_domain_bounds(dmin, dmax)
            be.pull(st, p)
            be.neighbor_search(p)
            stream = torch.cuda.ExternalStream(be.stream_handle(), device=dev)
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            reps = 5
            e0.record(stream)
            for _ in range(reps):
                be.neighbor_search(p)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            ms = e0.elapsed_time(e1) / reps
            s = be.stats()
            L = s.sellPackedBytes / n + 6.0
            passes = (s.keyBits + 7) // 8
            bpp = 24 + 24 * passes + 68 + 8 + 18 + 12 + L
            ns[f"{dist}_{n}"] = {"ms_per_build": round(ms, 4), "points_per_s": round(n / (ms / 1e3), 1),
                                 "algorithmic_GBps": round(bpp * n / (ms / 1e3) / 1e9, 1),
                                 "neighbors_per_point": round(s.nNbrFF / n, 1), "sort_passes": int(passes)}
            be.close()
    out["neighbor_search_only"] = ns
    return out


def served_stream_measure(n_scenes, steps):
    """Served-stream figures (turbospharticles_b200.serve): the seeded mixed-size stream
    (N_F log-uniform in [4,096, 262,144], Poisson arrivals at 64 scenes/s, 16 GB budget) run
    with continuous batching, and the same scenes one at a time on the plain path."""
    from turbospharticles_b200 import scene as S, serve
    specs = S.served_stream(n_scenes)
    prepared = serve.prepare(specs)
    sv = serve.run_served(prepared, steps, 16 << 30)
    pl = serve.run_plain(prepared, steps, full=True)
    return {"workload": f"served_stream_{n_scenes}x{steps}", "scenes": n_scenes, "steps_per_scene": steps,
            "n_fluid_total": int(sum(sp.n_fluid for sp in specs)), "unit": UNIT,
            "value": sv["value"], "value_wall": sv["value_wall"], "p50_step_ms": sv["p50_step_ms"],
            "p99_step_ms": sv["p99_step_ms"], "mean_active_scenes": sv["mean_active_scenes"],
            "latency_split": sv["latency_split"], "longest_substeps_ms": sv["longest_substeps_ms"],
            "substeps_over_20ms_s": sv["substeps_over_20ms_s"], "accuracy": sv["accuracy"],
            "plain_value": pl["value"], "plain_p50_step_ms": pl["p50_step_ms"],
            "plain_p99_step_ms": pl["p99_step_ms"], "plain_sampling": pl["sampling"],
            "served_over_plain": round(sv["value"] / pl["value"], 3)}


def cpu_baseline_from(be, p, dmin, dmax):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import OracleBackend
    st = be.push()
    threads = os.cpu_count() or 1
    o = OracleBackend(p, threads=threads)
    o.set_sim_domain_bounds(dmin, dmax)
    o.pull(st, p)
    # bounded sample: whole steps until about 12 s of CPU work (at least 3 steps)
    t0 = time.perf_counter()
    steps, sweeps = 0, 0
    while steps < 3 or time.perf_counter() - t0 < 12.0:
        o.step(p)
        steps += 1
        sweeps += o.stats().solverIters - 1
    dt = time.perf_counter() - t0
    return {"value": round(st.N_F * steps / dt, 1), "unit": UNIT, "cores": threads, "kind": "port",
            **cpu_description(),
            "sample": f"{steps} IISPH steps of the 1M dam from the GPU state after warm-up ({sweeps} Jacobi "
                      f"sweeps, {dt:.1f} s, oracle/ CPU restatement, scalar per particle (the compiler may "
                      f"vectorise), OpenMP over {threads} threads)"}


def run_reference(args):
    ws, rank, _ = dist_env()
    if ws > 1 and rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import OracleBackend
    st, dmin, dmax, p = build_workload()
    threads = os.cpu_count() or 1
    o = OracleBackend(p, threads=threads)
    o.set_sim_domain_bounds(dmin, dmax)
    o.pull(st, p)
    from turbospharticles_b200 import abi
    o.run_stage(abi.STAGE_BOUNDARY_VOLUMES, p)
    budget_s = 150.0
    t_start = time.perf_counter()
    for _ in range(args.warmup):
        o.step(p)
        if time.perf_counter() - t_start > budget_s / 2:
            break
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        o.step(p)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start > budget_s:
            break
    value = st.N_F * len(times) / sum(times)
    q = np.percentile(np.array(times) * 1e3, [50, 99])
    line = {"metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": ws, "steps": len(times),
            "warmup": args.warmup, "ms_per_step": round(1e3 * sum(times) / len(times), 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 residual sums)",
            "data": "synthetic (seeded dam-break scene restated from the reference builder)",
            "config": {"workload": "iisph_dam_1M", "n_fluid": st.N_F, "n_boundary": st.N_B,
                       "parallelism": f"{threads} host threads"},
            "p50_step_ms": round(float(q[0]), 2), "p99_step_ms": round(float(q[1]), 2), "impl": "reference",
            "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": threads, "kind": "port",
                             **cpu_description(),
                             "sample": f"{len(times)} IISPH steps of the 1M dam after {args.warmup} warm-up steps "
                                       "(oracle/ CPU restatement; the reference CPU backend needs oneTBB/xsimd/"
                                       "glm/Boost which are not installed)"},
            "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-developed", action="store_true", help="skip the developed-flow sub-measure")
    ap.add_argument("--no-configs", action="store_true", help="skip the other configurations' sub-measure")
    ap.add_argument("--tuning", default=None,
                    help="JSON file of launch configurations (a bench line's `tuned` object) to pin instead of tuning")
    ap.add_argument("--pin", action="append", default=None, metavar="KERNEL:SLOTS:MINBLOCKS",
                    help="pin one kernel's configuration at every particle count (repeatable), "
                         "e.g. KQueryFluidCount:1:5 for the staged count pass")
    ap.add_argument("--served-scenes", type=int, default=256,
                    help="scenes of the served-stream sub-measure (0: skip; 256 = the full stream)")
    ap.add_argument("--served-steps", type=int, default=500)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "b200" else args.warmup
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
