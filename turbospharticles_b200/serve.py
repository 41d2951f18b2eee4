"""Served mixed-size stream: continuous batching of independent dam-break scenes on one GPU.

Request loop: scenes arrive (seeded Poisson process, `scene.served_stream`), wait in a FIFO
queue, and are admitted into the batch when the batch's device-memory budget has room; every
loop iteration advances all admitted scenes by one step (`ServedBatchB200.substep`); a scene
that has run its steps is retired and its slot and memory are reused. Arrival times are
compared with the loop's own clock (device-timed substeps), so arrivals that happen while
other scenes are on the GPU are admitted at the next substep.

Accuracy: after every substep each active scene's average positive density error (the solver's
own termination measure) must be at most the target (0.1 %) unless the scene's solver stopped at
its iteration limit; the run reports the largest error seen, the count of scene-steps at the
limit and `accuracy_ok`.

The comparison path runs the same scenes one at a time on the one-scene backend
(`SimBackendB200`), the plain path, each for the same number of steps as in the served run;
its device time is the sum of its steps' CUDA-event times. (`--plain-sample K` instead times
steps 3..K+2 of every scene, charges the full step count at that rate and reports the bias of
that sampling from 16 scenes run in full: the flow develops and later steps need more Jacobi
sweeps, so a sample of early steps makes the plain path look faster than it is.)

    python -m turbospharticles_b200.serve --scenes 256 --steps 500        # the full stream
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import abi, scene as S
from .backend import ServedBatchB200, SimBackendB200, TspError


def prepare(specs):
    """Builds every scene and computes its boundary volumes once (ComputeParticleCoefficients,
    which the reference runs when it builds a scene)."""
    out = []
    for sp in specs:
        st, dmin, dmax, p = sp.build()
        be = SimBackendB200(p)
        be.set_sim_domain_bounds(dmin, dmax)
        be.pull(st, p)
        be.run_stage(abi.STAGE_BOUNDARY_VOLUMES, p)
        st = be.push()
        be.close()
        out.append((sp, st, dmin, dmax, p))
    return out


def run_served(prepared, steps, budget_bytes, max_substeps=None):
    """Continuous batching of the prepared scenes; returns throughput and latency figures."""
    p = prepared[0][4]
    batch = ServedBatchB200(p, budget_bytes)
    queue = list(range(len(prepared)))
    queue.sort(key=lambda k: prepared[k][0].arrival_s)
    active = {}   # slot -> (scene index, steps done)
    clock_s = 0.0
    sub_ms, n_active, particles_per_sub, changed_sub = [], [], [], []
    done_updates = 0
    refused = 0
    it = 0
    target = float(np.float32(p.densityDevTarget))
    max_err, at_limit, over_target, checked = 0.0, 0, 0, 0
    changed = True  # admissions or retirements since the last substep (the batch relayouts then)
    t0 = time.perf_counter()
    while queue or active:
        # admit arrived scenes in arrival order while they fit
        while queue and (prepared[queue[0]][0].arrival_s <= clock_s or not active):
            k = queue[0]
            sp, st, dmin, dmax, _ = prepared[k]
            try:
                slot = batch.admit(st, dmin, dmax)
            except TspError as e:
                if e.status != -3 or not active:
                    raise
                refused += 1
                break
            active[slot] = [k, 0]
            queue.pop(0)
            changed = True
        batch.substep(1)
        info = batch.info()
        ms = info["last_substep_ms"]
        sub_ms.append(ms)
        changed_sub.append(changed)
        changed = False
        clock_s += ms / 1e3
        nf = sum(prepared[k][0].n_fluid for k, _ in active.values())
        particles_per_sub.append(nf)
        n_active.append(len(active))
        done_updates += nf
        for slot in list(active):
            s_ = batch.stats(slot)
            checked += 1
            if s_.solverIters >= p.maxSolverIters:
                at_limit += 1
            else:
                max_err = max(max_err, float(s_.avgRelDensityErrPos))
                over_target += 1 if s_.avgRelDensityErrPos > target else 0
            active[slot][1] += 1
            if active[slot][1] >= steps:
                batch.retire(slot)
                del active[slot]
                changed = True
        it += 1
        if max_substeps and it >= max_substeps:
            break
    wall_s = time.perf_counter() - t0
    batch.close()
    dev_s = float(np.sum(sub_ms)) / 1e3
    q = np.percentile(sub_ms, [50, 99])
    ms_a = np.asarray(sub_ms)
    ch = np.asarray(changed_sub, bool)
    # substep latency split: substeps after an admission or retirement include the relayout
    # (whole chunks moved into the alternate arena, new scenes' boundaries sorted and gridded)
    split = {"relayout_substeps": int(ch.sum()),
             "relayout_p50_ms": round(float(np.percentile(ms_a[ch], 50)), 4) if ch.any() else None,
             "steady_p50_ms": round(float(np.percentile(ms_a[~ch], 50)), 4) if (~ch).any() else None,
             "steady_p99_ms": round(float(np.percentile(ms_a[~ch], 99)), 4) if (~ch).any() else None}
    # what the slowest 1 % of substeps have in common: fluid particles in flight and relayouts
    pp = np.asarray(particles_per_sub, np.float64)
    tail = ms_a >= q[1]
    split.update({"tail_substeps": int(tail.sum()), "tail_after_relayout": int((tail & ch).sum()),
                  "tail_mean_fluid": int(pp[tail].mean()), "all_mean_fluid": int(pp.mean()),
                  "tail_us_per_1k_fluid": round(float((ms_a[tail] / pp[tail]).mean()) * 1e6, 3),
                  "all_us_per_1k_fluid": round(float((ms_a / pp).mean()) * 1e6, 3)})
    return {"particle_updates": int(done_updates), "device_s": round(dev_s, 4), "wall_s": round(wall_s, 3),
            "value": round(done_updates / dev_s, 1), "value_wall": round(done_updates / wall_s, 1),
            "substeps": it, "p50_step_ms": round(float(q[0]), 4), "p99_step_ms": round(float(q[1]), 4),
            "latency_split": split,
            "longest_substeps_ms": [round(float(x), 2) for x in np.sort(ms_a)[-8:][::-1]],
            "substeps_over_20ms_s": round(float(ms_a[ms_a > 20.0].sum()) / 1e3, 3),
            "mean_active_scenes": round(float(np.mean(n_active)), 1), "max_active_scenes": int(np.max(n_active)),
            "admissions_deferred": refused, "budget_bytes": int(budget_bytes),
            "accuracy": {"target": target, "max_avg_density_error": max_err, "scene_steps_checked": checked,
                         "scene_steps_at_iteration_limit": at_limit, "scene_steps_over_target": over_target,
                         "accuracy_ok": over_target == 0}}


def run_plain(prepared, steps, sample_steps=10, warmup=2, calibrate=16, full=True):
    """The same scenes one at a time on the one-scene backend, device time per step (the
    backend's CUDA events around each step, summed). full: every scene runs all `steps` steps
    (the same steps the served run makes), its device time the sum of its steps; the first
    `calibrate` scenes are stepped one call per step for the per-step percentiles. Otherwise
    steps warmup+1 .. warmup+sample_steps of every scene are timed and charged for `steps` steps,
    and the calibration scenes also run in full to show the sampling's bias."""
    total_updates, total_s, step_ms = 0, 0.0, []
    cal_full, cal_sampled = [], []
    for idx, (sp, st, dmin, dmax, p) in enumerate(prepared):
        be = SimBackendB200(p)
        be.set_sim_domain_bounds(dmin, dmax)
        be.pull(st, p)
        if full:
            if idx < calibrate:
                for _ in range(steps):
                    be.step(p)
                    step_ms.append(be.stats().lastStepMs)
            else:
                be.step(p, steps)
            ms_total, n = be.step_time_total()
            be.close()
            total_updates += sp.n_fluid * steps
            total_s += ms_total / 1e3
            continue
        for _ in range(warmup):
            be.step(p)
        ms = []
        for _ in range(sample_steps):
            be.step(p)
            ms.append(be.stats().lastStepMs)
        if idx < calibrate:
            fl = list(ms)
            for _ in range(steps - warmup - sample_steps):
                be.step(p)
                fl.append(be.stats().lastStepMs)
            cal_full.append(float(np.mean(fl)))
            cal_sampled.append(float(np.mean(ms)))
        be.close()
        per = float(np.mean(ms))
        step_ms.extend(ms)
        total_updates += sp.n_fluid * steps
        total_s += per * steps / 1e3
    q = np.percentile(step_ms, [50, 99])
    out = {"particle_updates": int(total_updates), "device_s": round(total_s, 4),
           "value": round(total_updates / total_s, 1), "p50_step_ms": round(float(q[0]), 4),
           "p99_step_ms": round(float(q[1]), 4)}
    if full:
        out["sampling"] = (f"every scene all {steps} steps (device time = sum of the per-step CUDA-event times); "
                           f"percentiles from the first {min(calibrate, len(prepared))} scenes' steps")
    else:
        out["sampling"] = f"steps {warmup + 1}-{warmup + sample_steps} of each scene timed, charged for {steps} steps"
        out["calibration_scenes"] = len(cal_full)
        out["full_over_sampled"] = round(float(np.sum(cal_full) / np.sum(cal_sampled)), 3) if cal_full else None
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scenes", type=int, default=256)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--rate", type=float, default=64.0, help="Poisson arrival rate, scenes per second")
    ap.add_argument("--budget-gb", type=float, default=16.0)
    ap.add_argument("--plain-sample", type=int, default=0, help="time a sample of K steps per scene (0: all steps)")
    ap.add_argument("--seed", type=int, default=2024)
    args = ap.parse_args()
    specs = S.served_stream(args.scenes, rate_hz=args.rate, seed=args.seed)
    prepared = prepare(specs)
    served = run_served(prepared, args.steps, int(args.budget_gb * (1 << 30)))
    plain = run_plain(prepared, args.steps, args.plain_sample or 10, full=args.plain_sample == 0)
    print(json.dumps({"workload": "served_stream", "scenes": args.scenes, "steps_per_scene": args.steps,
                      "rate_hz": args.rate, "n_fluid_total": int(sum(s.n_fluid for s in specs)),
                      "served": served, "plain": plain,
                      "served_over_plain": round(served["value"] / plain["value"], 3)}))


if __name__ == "__main__":
    main()
