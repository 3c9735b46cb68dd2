#!/usr/bin/env python
"""Benchmark: registered frames/s for one stage of series matching at 513^2.

Workload (per GPU): 20 frames of a hexagonal Gaussian-column lattice, 513x513
(level 9), Poisson peak 30, smooth displacements <= 3 px plus 0.7 px row
jitter, registered to a reference frame of the same series on levels 5..9
(maxGDIterations 30, lambda 0.1, reference preprocessing with saturation
0.15 %), followed by the warped-frame average.  One bench step = one such
stage (all 20 registrations + the average).  Seeded synthetic data.

  value : frames/s with the images resident in HBM (device entry point)
  e2e   : frames/s through the host entry point msgpu_match_series_stage with
          pinned host buffers (uploads and downloads inside the timed region)

--impl reference times the reference's own CPU code (oracle/_ref/ms_ref, the
quocmesh templates built from the reference sources) on a bounded sample of
the same workload, one process per host core.

--series times the whole of matchSeries' first stage instead
(msgpu_match_series, accumulated deformations): the 20 templates are
registered to their predecessors in one batch, then composed and refined
against frame 0 one after the other, then averaged.  Its CPU baseline is the
reference's own stage loop on the first 3 templates (a sequential chain, one
core).

--files times series read from disk: FILE_SERIES series of 21 frames each,
stored as the reference's bzip2-compressed double arrays (.q2bz), are decoded
by host threads and registered stage by stage through the host entry point,
the decoding of the next series overlapping the GPU work on the current one.
Its CPU baseline is the reference's own loader on the same files.

--ragged times uneven series in one batch (msgpu_register_ragged): 16
series of 8 templates each, sizes drawn from 129², 257², 513², 1025², levels
4 to each series' own finest level, one launch per level for all series;
beside it the same series registered one batch after the other.

--seismic times the seismic line-shift model (matchSeismicSeries'
findXShift): 32 synthetic gathers of 257 traces x 2049 samples, each
registered to the mean gather by shifts along the time axis (line-wise NCC,
anisotropic regulariser, exact H1 metric), maxGDIterations 500; its CPU
baseline is the oracle port on a 257-sample x 33-trace crop (the reference's
own solver needs SuiteSparse, which it does not vendor).

Multi-GPU (torchrun): weak scaling; every rank registers its own series.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "match-series_b200"))

METRIC = "registered frames/s at 513² to stated energy tol: warm-start+batched vs plain GPU"
UNIT = "frames/s"
LEVEL, START, FRAMES, MAX_ITER, LAMBDA = 9, 5, 20, 30, 0.1
DATA_TERM = 0   # 0: SSD (deformationModel 22); 1: normalized cross-correlation (--ncc)


def use_tuning(ctx):
    """Loads the committed scheduler table (measured on B200) when it exists."""
    if os.path.exists(os.path.join(ROOT, "match-series_b200", "msgpu", "tuning_b200.json")):
        ctx.load_tuning()


def workload(rank: int):
    """One series: frame FRAMES is the stage's reference on every rank; rank
    0 registers frames 0..FRAMES-1, rank r > 0 the next FRAMES frames after
    the reference (a shard of one series of FRAMES * world + 1 frames)."""
    from msgpu import synthetic as syn
    n = (1 << LEVEL) + 1
    if rank == 0:
        frames, clean, _ = syn.make_series(n, FRAMES + 1, syn.HEX_513, seed=2000)
        return frames[FRAMES].reshape(-1).copy(), frames[:FRAMES].reshape(FRAMES, -1).copy(), clean[FRAMES]
    rf, rc, _ = syn.make_series(n, 1, syn.HEX_513, seed=2000, first=FRAMES)
    frames, _, _ = syn.make_series(n, FRAMES, syn.HEX_513, seed=2000, first=FRAMES + 1 + FRAMES * (rank - 1))
    return rf[0].reshape(-1).copy(), frames.reshape(FRAMES, -1).copy(), rc[0]


SUM_ORDER = 0   # 0: the reference's sequential order (bit-exact); 1: parallel order (--sum-order 1)
CERTIFIED = True   # sum order 0: control steps on bounded sums where the bounds settle them
WARM_COARSE_ITERS = 4   # warm leg: step limit below the stop level (0: maxGDIterations); 4 measured best


def params(fp64: bool):
    import msgpu
    return msgpu.default_params(precision_level=LEVEL, input_level=LEVEL, start_level=START, stop_level=LEVEL,
                                max_gd_iterations=MAX_ITER, use_fp64=int(fp64), data_term=DATA_TERM,
                                sum_order=SUM_ORDER)


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while running."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                t = [x.strip() for x in line.split(",")]
                if len(t) >= 9 and t[1].replace(".", "").isdigit():
                    rows.append(t)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows]
        mx = max(float(r[2]) for r in rows)
        load = [s for s in sm if s > 0.5 * mx] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


def measured_peak():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def level_traffic(fp64: bool):
    """DRAM bytes per launch of the finest-level kernel from the committed ncu summary (or None)."""
    try:
        d = json.load(open(os.path.join(ROOT, "profiles", "level_kernel_traffic.json")))
        key = ("f64" if fp64 else "f32") + ("_ncc" if DATA_TERM else "")
        if key == "f64" and SUM_ORDER == 0:
            key = "f64_exact"   # the reference's sum order: terms stored for the ordered sums
        return d.get(key, {}).get("bytes_per_launch_513x20")
    except Exception:
        return None


def algorithmic_bytes(steps: int, evals: int, real_bytes: int) -> float:
    """Per-level algorithmic bytes, per node and frame in FP32 units (scaled by
    real_bytes/4).  SSD: 24 B per energy trial (phi, d, R, gathered T), 24 B
    gradient, 20 B NCG/update, 2 x 96 B V-cycle per step.  NCC: an energy
    evaluation is three passes (phi, d, gathered T, Td write; Td; Td and the
    normalised R) = 40 B, the gradient adds them to its force pass (phi, Td,
    normalised R, gathered T, DE write = 28 B) = 68 B."""
    n = (1 << LEVEL) + 1
    if DATA_TERM:
        return n * n * (40.0 * evals + (68.0 + 20.0 + 2 * 96.0) * steps) * (real_bytes / 4.0)
    return n * n * (24.0 * evals + (24.0 + 20.0 + 2 * 96.0) * steps) * (real_bytes / 4.0)


# --- CPU baseline: the reference binary on a bounded sample ------------------

def run_reference_sample(ref, tmpl, procs: int, workdir: str):
    """Registers `procs` templates with the reference (one process each, in
    parallel); returns (frames, seconds, phis, energies, kind)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import msor
    n = (1 << LEVEL) + 1
    N = n * n
    if msor.have_ref():
        jobs = []
        for i in range(procs):
            d = os.path.join(workdir, f"r{i}")
            os.makedirs(d, exist_ok=True)
            fr = np.stack([ref, tmpl[i]])
            fr.tofile(os.path.join(d, "frames.bin"))
            cmd = [msor.REF_BIN, "series_ncc" if DATA_TERM else "series", str(LEVEL), str(START), str(LEVEL), repr(LAMBDA), "1.0", str(MAX_ITER),
                   "0.0", "0.15", "1", "2", os.path.join(d, "frames.bin"), os.path.join(d, "phis.bin"),
                   os.path.join(d, "mean.bin"), os.path.join(d, "info.txt")]
            jobs.append(subprocess.Popen(cmd, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL))
        t0 = time.perf_counter()
        for j in jobs:
            j.wait()
        wall = time.perf_counter() - t0
        secs, phis, energies = [], [], []
        for i in range(procs):
            d = os.path.join(workdir, f"r{i}")
            info = {}
            for line in open(os.path.join(d, "info.txt")):
                t = line.split()
                info[t[0] + (t[1] if t[0] == "energy" else "")] = float(t[-1])
            secs.append(info["registration_seconds"])
            phis.append(np.fromfile(os.path.join(d, "phis.bin")).reshape(2, 2, N)[1])
            energies.append(info["energy1"])
        # registration phase only (the driver's own clock, file I/O excluded)
        return procs, max(secs), np.array(phis), np.array(energies), "reference", wall
    # the CPU restatement when the reference binary is not available here
    import multiprocessing as mp
    msor.lib()
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        res = pool.starmap(_oracle_one, [(ref, tmpl[i]) for i in range(procs)])
    wall = time.perf_counter() - t0
    phis = np.array([[r[0], r[1]] for r in res])
    energies = np.array([r[2] for r in res])
    return procs, wall, phis, energies, "port", wall


def _oracle_one(ref, tpl):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import msor
    R = msor.normalize(ref)
    T = msor.normalize(tpl)
    px, py, e, _ = msor.register(LEVEL, START, LEVEL, R, T, lam=LAMBDA, max_iter=MAX_ITER, ncc=bool(DATA_TERM))
    return px, py, e


def cpu_procs():
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except Exception:
        return max(1, os.cpu_count() or 1)


# --- main ---------------------------------------------------------------------

def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    return world, rank, local


def allreduce_max(x: float, world: int):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def run_reference_arm(args, world, rank):
    if rank != 0:
        return 0
    ref, tmpl, _ = workload(0)
    procs = min(cpu_procs(), FRAMES)
    values = []
    kind = None
    with tempfile.TemporaryDirectory() as wd:
        for it in range(args.warmup + args.steps):
            nfr, secs, _, _, kind, _ = run_reference_sample(ref, tmpl, procs, wd)
            if it >= args.warmup:
                values.append(nfr / secs)
    v = statistics.mean(values)
    out = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * procs / v,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": f"stage registration of {procs} of the 20 hex-lattice frames 513x513 (level 9) "
                                  f"to a reference frame, levels {START}-{LEVEL}, maxGDIterations {MAX_ITER}, "
                                  f"lambda {LAMBDA}, {'NCC' if DATA_TERM else 'SSD'} data term; one process per "
                                  f"host core", "frames_per_step": procs, "data_term": "ncc" if DATA_TERM else "ssd"},
           "cpu_baseline": {"value": v, "unit": UNIT, "cores": procs, "kind": kind,
                            "sample": f"{procs} frames 513x513 per step, one per process"},
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return 0


TRACE_KINDS = {0: "energy0", 1: "gradient", 2: "vdown", 3: "vcoarse", 4: "vup", 5: "ncg", 6: "trial",
               7: "flush", 8: "ncc1", 9: "ncc2", 10: "ncc3", 11: "ncc_var", 12: "xsum"}


def trace_summary(tr: dict, ctas: int) -> dict:
    """Figures of a level kernel's pass timeline (Context.trace()): CTA time
    spent waiting for work (all of it, and after the first instance
    finished), the ordered walks, and per pass kind the mean time from
    publication to completion and from completion to the next publication
    (the control step, with any ordered walk it waits for)."""
    import numpy as np
    t, ev, val = tr["t"], tr["event"], tr["value"]
    span = float(t.max()) if t.size else 0.0
    pub, com = ev == 1, ev == 2
    fin = t[pub & ((val & 255) == 13)]
    idle, walk = ev == 3, ev == 4
    out = {"span_ms": span / 1e6, "ctas": ctas,
           "idle_cta_ms": float(val[idle].sum()) / 1e6,
           "idle_frac": float(val[idle].sum()) / (span * ctas) if span else 0.0,
           "idle_cta_ms_after_first_finish": float(val[idle & (t >= fin.min())].sum()) / 1e6 if fin.size else 0.0,
           "finish_ms": [float(fin.min()) / 1e6, float(np.median(fin)) / 1e6, float(fin.max()) / 1e6] if fin.size else [],
           "walks": int(walk.sum()), "walk_us_mean": float(val[walk].mean()) / 1e3 if walk.any() else 0.0,
           "walk_us_max": float(val[walk].max()) / 1e3 if walk.any() else 0.0}
    dur, lat = {}, {}
    for i in np.unique(val[pub] >> 8):
        P = pub & ((val >> 8) == i)
        C = com & ((val >> 8) == i)
        tp, kp, tc = t[P], val[P] & 255, t[C]
        for j in range(min(len(tp), len(tc))):
            dur.setdefault(int(kp[j]), []).append(tc[j] - tp[j])
            if j + 1 < len(tp):
                lat.setdefault(int(kp[j]), []).append(tp[j + 1] - tc[j])
    out["pass_us"] = {TRACE_KINDS.get(k, str(k)): [len(v), float(np.mean(v)) / 1e3] for k, v in sorted(dur.items())}
    out["control_us"] = {TRACE_KINDS.get(k, str(k)): float(np.mean(v)) / 1e3 for k, v in sorted(lat.items())}
    return out


def profile_case(level: int, iters: int, fp64: bool, trace_out: str = ""):
    """One launch of the level kernel on the bench's frames generated at
    `level` (start = stop = level, `iters` steps): the case ncu captures."""
    import numpy as np
    import msgpu
    from msgpu import build as mbuild
    from msgpu import synthetic as syn
    mbuild.build()
    n = (1 << level) + 1
    frames, _, _ = syn.make_series(n, FRAMES + 1, syn.HEX_513, seed=2000)
    ctx = msgpu.Context(0)
    p = msgpu.default_params(precision_level=level, input_level=level, start_level=level, stop_level=level,
                             max_gd_iterations=iters, use_fp64=int(fp64), data_term=DATA_TERM, sum_order=SUM_ORDER)
    ctx.set_certified_steps(CERTIFIED)
    ctx.set_profiling(True)
    if trace_out:
        ctx.set_trace(level, 1 << 22)
    ctx.register_batch(p, frames[FRAMES], frames[:FRAMES])
    print(json.dumps({"profile_level": level, "frames": FRAMES, "iters": iters, "fp64": fp64,
                      "stats": ctx.stats()}))
    if trace_out:
        tr = ctx.trace()
        np.savez_compressed(trace_out, **tr)
        print(json.dumps({"trace": trace_summary(tr, ctx.stats()["level_cluster"][0])}))


SERIES_SAMPLE = 3   # templates of the chain the CPU reference runs in --series


def profile_series(compose_level: int, fp64: bool):
    """Small cases for ncu: with compose_level > 0 one composition at that
    level (smooth displacements of 3 px and 2 px, the second shifted so that a
    band of nodes leaves the domain); otherwise one msgpu_match_series call on
    the bench's frames (no timing)."""
    import numpy as np
    import msgpu
    from msgpu import build as mbuild
    from msgpu import synthetic as syn
    mbuild.build()
    ctx = msgpu.Context(0)
    if compose_level:
        n = (1 << compose_level) + 1
        rng = np.random.default_rng(compose_level)
        d1 = syn.smooth_field(n, rng, 3.0)
        d2 = syn.smooth_field(n, rng, 2.0, shift_px=(-3.0, 2.0))
        _, it = ctx.compose(compose_level, d1, d2)
        print(json.dumps({"profile_compose_level": compose_level, "pcg_iterations": it.tolist()}))
        return 0
    p = params(fp64)
    ref, tmpl, _ = workload(0)
    frames = np.concatenate([ref[None], tmpl])
    ctx.match_series(p, msgpu.default_series_params(p), frames)
    print(json.dumps({"profile_series_frames": int(frames.shape[0]), "launches": ctx.stats()["kernel_launches"]}))
    return 0


def reference_series_sample(frames, workdir: str):
    """The reference's stage loop on frames[0..SERIES_SAMPLE] (one process);
    returns (seconds of the registration phase, phis, energies)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import msor
    r = msor.RefRunner()
    phis, _, _, _, energies, timing = r.match_series(LEVEL, START, LEVEL, frames[:SERIES_SAMPLE + 1], lam=LAMBDA,
                                                     max_iter=MAX_ITER, refine_start=START, ncc=bool(DATA_TERM))
    return timing[1]["registration_seconds"], phis, energies[0]


def main_series(args, world, rank, local):
    """--series: msgpu_match_series (stage 1 with accumulated deformations)."""
    import numpy as np
    import torch
    import msgpu
    from msgpu import build as mbuild

    torch.cuda.set_device(local)
    mbuild.build()
    fp64 = not args.fp32
    p = params(fp64)
    sp = msgpu.default_series_params(p)
    ref, tmpl, _ = workload(rank)
    frames = np.concatenate([ref[None], tmpl])            # frame 0 is the stage's reference
    F = frames.shape[0]
    m = F - 1
    n = (1 << LEVEL) + 1
    N = n * n
    ctx = msgpu.Context(local)
    use_tuning(ctx)
    dev = torch.device("cuda", local)
    d_frames = torch.from_numpy(frames).to(dev)
    d_phis = torch.empty((m, 2, N), dtype=torch.float64, device=dev)
    d_e = torch.empty(m, dtype=torch.float64, device=dev)
    d_avg = torch.empty(N, dtype=torch.float64, device=dev)
    d_med = torch.empty(N, dtype=torch.float64, device=dev)
    d_cnt = torch.empty(N, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        ctx.match_series_device(p, sp, d_frames.data_ptr(), F, d_phis.data_ptr(), d_e.data_ptr(), d_avg.data_ptr(),
                                d_med.data_ptr(), d_cnt.data_ptr(), stream.cuda_stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    start_ev = torch.cuda.Event(enable_timing=True)
    stop_ev = torch.cuda.Event(enable_timing=True)
    launches = 0
    barrier(world)
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clocks:
        start_ev.record(stream)
        for _ in range(args.steps):
            step()
            launches += ctx.stats()["kernel_launches"]
        stop_ev.record(stream)
        torch.cuda.synchronize(dev)
    barrier(world)
    elapsed_ms = allreduce_max(start_ev.elapsed_time(stop_ev), world)
    value = world * m * args.steps / (elapsed_ms / 1000.0)
    phis = d_phis.cpu().numpy()
    energies = d_e.cpu().numpy()
    # one profiled call: per-level launch times of its last solve (a single-frame refinement)
    ctx.set_profiling(True)
    step()
    torch.cuda.synchronize(dev)
    st = ctx.stats()
    ctx.set_profiling(False)
    # end to end through the host entry point, pinned host buffers
    h_frames = torch.from_numpy(frames).pin_memory().numpy()
    ctx.match_series(p, sp, h_frames)
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ctx.match_series(p, sp, h_frames)
    e2e_s = allreduce_max(time.perf_counter() - t0, world)
    e2e_value = world * m * args.steps / e2e_s
    h2d = F * N * 8
    d2h = (2 * m * N + 3 * N + m) * 8
    if rank == 0:
        peak, peak_kind = measured_peak()
        real_bytes = 8 if fp64 else 4
        lv = LEVEL - st["first_level"]
        lvl_ms = st["level_ms"][lv]
        alg = algorithmic_bytes(st["level_steps"][lv], st["level_evals"][lv], real_bytes)
        achieved = alg / (lvl_ms / 1000.0) / 1e9
        clk = clocks.summary()
        cpu = accuracy = None
        if world == 1 and not args.no_cpu_baseline:
            with tempfile.TemporaryDirectory() as wd:
                secs, rphis, ren = reference_series_sample(frames, wd)
            cpu = {"value": SERIES_SAMPLE / secs, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": f"the reference's stage loop on frames 0..{SERIES_SAMPLE} (the first {SERIES_SAMPLE} "
                             f"templates of the chain, 513x513, levels {START}-{LEVEL}), registration phase "
                             f"{secs:.1f} s; the chain is sequential, one core"}
            fp = frames.copy()
            up = np.random.default_rng(7).random(fp.shape) < 0.5
            fp = np.where(up, np.nextafter(fp, np.inf), np.nextafter(fp, -np.inf))
            with tempfile.TemporaryDirectory() as wd:
                _, pphis, pen = reference_series_sample(fp, wd)
            k = SERIES_SAMPLE
            accuracy = {"templates_checked": k,
                        "max_dphi_px": float(np.abs(phis[:k] - rphis).max()) * (n - 1),
                        "max_rel_energy": float(np.max(np.abs(energies[:k] - ren) / np.abs(ren))),
                        "tolerance": {"dphi_px": 1e-3, "rel_energy": 1e-6},
                        "reference_1ulp_spread": {"max_dphi_px": float(np.abs(pphis - rphis).max()) * (n - 1),
                                                  "max_rel_energy": float(np.max(np.abs(pen - ren) / np.abs(ren))),
                                                  "perturbation": "every pixel of every frame +-1 ulp"}}
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if fp64 else "f32+f64-reductions",
            "data": "synthetic",
            "config": {"workload": f"matchSeries stage 1 with accumulated deformations: {m} hex-lattice templates "
                                   f"513x513 (level {LEVEL}) and frame 0, pairwise batch, composition and "
                                   f"refinement (levels {START}-{LEVEL}) per template, average and median; "
                                   f"maxGDIterations {MAX_ITER}, lambda {LAMBDA}, "
                                   f"{'NCC' if DATA_TERM else 'SSD'} data term",
                       "data_term": "ncc" if DATA_TERM else "ssd",
                       "sum_order": "reference sequential order (bit-exact)"
                       if (SUM_ORDER == 0 and fp64 and not DATA_TERM) else "parallel order", "templates_per_gpu": m, "level": LEVEL,
                       "l2": "no flush: per-step working set exceeds the 126 MB L2",
                       "parallelism": f"weak, {world} independent series"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": f"level_kernel<{'double' if fp64 else 'float'}> level {LEVEL}, "
                                                   f"single-frame refinement",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "traffic": None, "algorithmic_bytes_per_launch": alg,
                         "avg_launch_ms": lvl_ms},
            "cpu_baseline": cpu,
            "accuracy": accuracy,
            "clocks": {k2: clk[k2] for k2 in ("sm_mhz", "sm_max_mhz", "reasons")},
        }
        print(json.dumps(out), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


FILE_SERIES = 4


def main_files(args, world, rank, local):
    """--files: series decoded from .q2bz files, overlapped with the GPU stages."""
    import numpy as np
    import torch
    import msgpu
    from concurrent.futures import ThreadPoolExecutor
    from msgpu import build as mbuild
    from msgpu import synthetic as syn

    torch.cuda.set_device(local)
    mbuild.build()
    fp64 = not args.fp32
    p = params(fp64)
    n = (1 << LEVEL) + 1
    N = n * n
    nlev = LEVEL - START + 1
    threads = cpu_procs()
    ctx = msgpu.Context(local)
    use_tuning(ctx)
    with tempfile.TemporaryDirectory() as wd:
        # --- the files (untimed): FILE_SERIES series, reference frame first
        series = []
        with ThreadPoolExecutor(threads) as pool:
            for k in range(FILE_SERIES):
                fr, _, _ = syn.make_series(n, FRAMES + 1, syn.HEX_513, seed=2000 + 1000 * rank + 17 * k)
                paths = [os.path.join(wd, f"s{k}_f{i:02d}.q2bz") for i in range(FRAMES + 1)]
                order = [FRAMES] + list(range(FRAMES))
                list(pool.map(lambda a: msgpu.write_array(a[0], fr[a[1]]), zip(paths, order)))
                series.append(paths)
        file_bytes = sum(os.path.getsize(q) for q in series[0])
        bufs = [torch.zeros((FRAMES + 1, N), dtype=torch.float64).pin_memory().numpy() for _ in range(2)]
        outs = (torch.zeros((FRAMES, 2, N), dtype=torch.float64).pin_memory().numpy(),
                torch.zeros(FRAMES, dtype=torch.float64).pin_memory().numpy(),
                torch.zeros((FRAMES, nlev), dtype=torch.int32).pin_memory().numpy(),
                torch.zeros(N, dtype=torch.float64).pin_memory().numpy(),
                torch.zeros(N, dtype=torch.float64).pin_memory().numpy())

        def stage(buf):
            ctx.match_series_stage(p, buf[0], buf[1:], out=outs)
            return ctx.stats()["kernel_launches"]

        # warm-up: decoding and one stage
        for _ in range(args.warmup):
            msgpu.read_arrays(series[0], n, n, threads)
        bufs[0][:] = msgpu.read_arrays(series[0], n, n, threads).reshape(FRAMES + 1, N)
        stage(bufs[0])
        # decoding alone
        t0 = time.perf_counter()
        for k in range(FILE_SERIES):
            msgpu.ReadTask(series[k], n, n, bufs[k % 2], threads).wait()
        t_dec = time.perf_counter() - t0
        # decode then register, series after series
        barrier(world)
        t0 = time.perf_counter()
        for k in range(FILE_SERIES):
            msgpu.ReadTask(series[k], n, n, bufs[0], threads).wait()
            stage(bufs[0])
        t_seq = allreduce_max(time.perf_counter() - t0, world)
        # decoding of series k+1 overlapping the stage of series k (the timed value)
        launches = 0
        barrier(world)
        with ClockSampler(local) as clocks:
            t0 = time.perf_counter()
            task = msgpu.ReadTask(series[0], n, n, bufs[0], threads)
            for k in range(FILE_SERIES):
                task.wait()
                task = msgpu.ReadTask(series[k + 1], n, n, bufs[(k + 1) % 2], threads) if k + 1 < FILE_SERIES else None
                launches += stage(bufs[k % 2])
            t_ovl = allreduce_max(time.perf_counter() - t0, world)
        # the reference's own loader on 3 of the files, one after the other (one core)
        cpu = None
        if rank == 0 and not args.no_cpu_baseline:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import msor
            if msor.have_ref():
                r = msor.RefRunner()
                t0 = time.perf_counter()
                for q in series[0][:3]:
                    r.load_array(q)
                t_ref = (time.perf_counter() - t0) / 3
                cpu = {"value": 1.0 / t_ref, "unit": "frames/s", "cores": 1, "kind": "reference",
                       "sample": "the reference's loader (qc::ScalarArray<QC_2D>::load via aol::Bzipifstream) on 3 "
                                 "of the .q2bz frames, one process each, process start included; decoding only"}
    if rank == 0:
        frames_total = world * FRAMES * FILE_SERIES
        clk = clocks.summary()
        out = {
            "metric": METRIC, "value": frames_total / t_ovl, "unit": UNIT, "n_gpus": world, "steps": FILE_SERIES,
            "warmup": args.warmup, "ms_per_step": 1000.0 * t_ovl / FILE_SERIES, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if fp64 else "f32+f64-reductions",
            "data": "synthetic, stored as .q2bz files",
            "config": {"workload": f"{FILE_SERIES} series of {FRAMES} hex-lattice templates 513x513 and a reference "
                                   f"frame, each frame a bzip2-compressed double array file (.q2bz, "
                                   f"{file_bytes / (FRAMES + 1) / 1e6:.2f} MB); per series: decode on {threads} "
                                   f"host threads, then msgpu_match_series_stage (levels {START}-{LEVEL}, "
                                   f"maxGDIterations {MAX_ITER}); a step is one series",
                       "decode_threads": threads,
                       "parallelism": f"weak, {world} ranks"},
            "e2e": {"value": frames_total / t_ovl, "unit": UNIT,
                    "h2d_bytes_per_step": (FRAMES + 1) * N * 8,
                    "d2h_bytes_per_step": (2 * FRAMES * N + 2 * N + FRAMES) * 8 + FRAMES * nlev * 4},
            "gpu_launches": launches,
            "files": {"overlapped_frames_per_s": frames_total / t_ovl,
                      "sequential_frames_per_s": frames_total / t_seq,
                      "decode_only_frames_per_s": FRAMES * FILE_SERIES / t_dec,
                      "decode_MB_per_s": (FILE_SERIES * (FRAMES + 1) * N * 8 / 1e6) / t_dec,
                      "compressed_MB_per_series": file_bytes / 1e6},
            "roofline": None,
            "cpu_baseline": cpu,
            "clocks": {k2: clk[k2] for k2 in ("sm_mhz", "sm_max_mhz", "reasons")},
        }
        print(json.dumps(out), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main_ragged(args, world, rank, local):
    """--ragged: uneven series in one ragged batch (msgpu_register_ragged)."""
    import numpy as np
    import torch
    import msgpu
    from msgpu import build as mbuild
    from msgpu import synthetic as syn

    torch.cuda.set_device(local)
    mbuild.build()
    fp64 = not args.fp32
    series = syn.ragged_workload(seed=3000 + 1000 * rank)
    levels = [int(round(np.sqrt(r.size))) - 1 for r, _ in series]
    levels = [l.bit_length() - 1 for l in levels]
    F = [t.shape[0] for _, t in series]
    total = sum(F)
    p = msgpu.default_params(start_level=4, max_gd_iterations=MAX_ITER, use_fp64=int(fp64), lambda_=LAMBDA,
                             sum_order=SUM_ORDER)
    ctx = msgpu.Context(local)
    use_tuning(ctx)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    keep, descs = [], []
    for (ref, tm), l in zip(series, levels):
        N = ((1 << l) + 1) ** 2
        d_ref = torch.from_numpy(ref).to(dev)
        d_tm = torch.from_numpy(tm).to(dev)
        d_ph = torch.empty((tm.shape[0], 2, N), dtype=torch.float64, device=dev)
        d_e = torch.empty(tm.shape[0], dtype=torch.float64, device=dev)
        keep += [d_ref, d_tm, d_ph, d_e]
        descs.append(msgpu.SeriesDesc(l, tm.shape[0], d_ref.data_ptr(), d_tm.data_ptr(), d_ph.data_ptr(),
                                      d_e.data_ptr()))

    def step():
        ctx.register_ragged_device(p, descs, stream.cuda_stream)

    def separate():
        for d in descs:
            q = msgpu.default_params(precision_level=d.level, input_level=d.level, start_level=4, stop_level=d.level,
                                     max_gd_iterations=MAX_ITER, use_fp64=int(fp64), lambda_=LAMBDA, sum_order=SUM_ORDER)
            ctx.register_batch_device(q, d.reference, d.templates, d.num_templates, d.phis_out, d.energies_out,
                                      0, 0, stream.cuda_stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    start_ev = torch.cuda.Event(enable_timing=True)
    stop_ev = torch.cuda.Event(enable_timing=True)
    launches = 0
    barrier(world)
    with ClockSampler(local) as clocks:
        start_ev.record(stream)
        for _ in range(args.steps):
            step()
            launches += ctx.stats()["kernel_launches"]
        stop_ev.record(stream)
        torch.cuda.synchronize(dev)
    elapsed_ms = allreduce_max(start_ev.elapsed_time(stop_ev), world)
    value = world * total * args.steps / (elapsed_ms / 1000.0)
    # the same series one batch after the other
    separate()
    torch.cuda.synchronize(dev)
    start_ev.record(stream)
    separate()
    stop_ev.record(stream)
    torch.cuda.synchronize(dev)
    sep_ms = start_ev.elapsed_time(stop_ev)
    # end to end through the host entry point
    host = [(r, t) for r, t in series]
    ctx.register_ragged(p, host)
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ctx.register_ragged(p, host)
    e2e_s = allreduce_max(time.perf_counter() - t0, world)
    h2d = sum((1 + f) * ((1 << l) + 1) ** 2 * 8 for f, l in zip(F, levels))
    d2h = sum((2 * f * ((1 << l) + 1) ** 2 + f) * 8 for f, l in zip(F, levels))
    if rank == 0:
        clk = clocks.summary()
        sizes = {}
        for f, l in zip(F, levels):
            sizes[(1 << l) + 1] = sizes.get((1 << l) + 1, 0) + f
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if fp64 else "f32+f64-reductions",
            "data": "synthetic",
            "config": {"workload": f"ragged batch: {len(series)} series, {total} templates, frames per size "
                                   f"{dict(sorted(sizes.items()))}, square/hex lattices with spacing 8-16 px and "
                                   f"Poisson peak 20-100, levels 4 to each series' finest, maxGDIterations "
                                   f"{MAX_ITER}, lambda {LAMBDA}, one level-kernel launch per level",
                       "sum_order": "reference sequential order (bit-exact)" if SUM_ORDER == 0 else "parallel order",
                       "parallelism": f"weak, {world} ranks"},
            "e2e": {"value": world * total * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "separate_batches_frames_per_s": total / (sep_ms / 1000.0),
            "roofline": None,
            "cpu_baseline": None,
            "clocks": {k: clk[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        }
        print(json.dumps(out), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


SEIS_GATHERS, SEIS_LAMBDA, SEIS_YREG, SEIS_ITER, SEIS_WORKERS = 32, 0.1, 1.0, 500, 8


def main_seismic(args, world, rank, local):
    """--seismic: findXShift for 32 gathers (msgpu_find_xshift_batch)."""
    import numpy as np
    import torch
    import msgpu
    from msgpu import build as mbuild
    from msgpu import synthetic as syn

    torch.cuda.set_device(local)
    mbuild.build()
    gathers = syn.seismic_gathers(SEIS_GATHERS, seed=4000 + 1000 * rank)
    R = gathers.mean(axis=0)
    G, ny, nx = gathers.shape
    ctx = msgpu.Context(local)

    def step():
        return ctx.find_xshift_batch(R, gathers, SEIS_LAMBDA, SEIS_YREG, SEIS_ITER, workers=SEIS_WORKERS)

    for _ in range(max(1, args.warmup - 2)):
        step()
    launches = 0
    barrier(world)
    with ClockSampler(local) as clocks:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            ph, en, st = step()
            launches += ctx.stats()["kernel_launches"]
        elapsed = allreduce_max(time.perf_counter() - t0, world)
    value = world * G * args.steps / elapsed
    # the data term's kernel (k_lineshift with its derivative) over all gathers in
    # one launch: R, T, phi read and DE written once per gather (inputs > L2)
    dev = torch.device("cuda", local)
    N = nx * ny
    d_R = torch.from_numpy(np.ascontiguousarray(np.broadcast_to(R, gathers.shape))).to(dev)
    d_T = torch.from_numpy(gathers).to(dev)
    d_phi = torch.from_numpy(ph).to(dev)
    d_de = torch.empty_like(d_T)
    d_e = torch.empty(G, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)

    def data_term():
        ctx.lineshift_energy_device(nx, ny, G, d_R.data_ptr(), d_T.data_ptr(), d_phi.data_ptr(), d_e.data_ptr(),
                                    d_de.data_ptr(), stream.cuda_stream)

    for _ in range(3):
        data_term()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 20
    torch.cuda.synchronize(dev)
    ev0.record(stream)
    for _ in range(reps):
        data_term()
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    ls_ms = ev0.elapsed_time(ev1) / reps
    ls_bytes = G * N * 8 * 4 + G * ny * 8
    peak, peak_kind = measured_peak()
    if rank == 0:
        clk = clocks.summary()
        cpu = accuracy = None
        if not args.no_cpu_baseline:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import msor
            crop = (slice(0, 33), slice(0, 257))
            t0 = time.perf_counter()
            rph, re, rsteps, _ = msor.xshift(R[crop], gathers[0][crop], SEIS_LAMBDA, SEIS_YREG, SEIS_ITER)
            t_cpu = time.perf_counter() - t0
            gph, ge, gsteps = ctx.find_xshift(R[crop], gathers[0][crop], SEIS_LAMBDA, SEIS_YREG, SEIS_ITER)
            # the oracle's own sensitivity: every template pixel of the crop moved by one ulp
            tc = gathers[0][crop]
            up = np.random.default_rng(7).random(tc.shape) < 0.5
            tp = np.where(up, np.nextafter(tc, np.inf), np.nextafter(tc, -np.inf))
            pph, pe, psteps, _ = msor.xshift(R[crop], tp, SEIS_LAMBDA, SEIS_YREG, SEIS_ITER)
            cpu = {"value": 1.0 / t_cpu, "unit": "crops/s", "cores": 1, "kind": "port",
                   "sample": f"the oracle (band Cholesky for the H1 metric) on a 257-sample x 33-trace crop of one "
                             f"gather, {rsteps} steps in {t_cpu:.1f} s; the reference's own CholeskyBasedInverseH1Metric "
                             f"needs SuiteSparse, which it does not vendor"}
            accuracy = {"crop": "257 x 33", "steps_gpu": int(gsteps), "steps_oracle": int(rsteps),
                        "max_dphi_px": float(np.abs(gph - rph).max() * 256),
                        "rel_energy": float(abs(ge - re) / abs(re)),
                        "oracle_1ulp_spread": {"steps": int(psteps),
                                               "max_dphi_px": float(np.abs(pph - rph).max() * 256),
                                               "rel_energy": float(abs(pe - re) / abs(re)),
                                               "perturbation": "every template pixel of the crop +-1 ulp"}}
        out = {
            "metric": METRIC, "value": value, "unit": "gathers/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * elapsed / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic seismic gathers",
            "config": {"workload": f"findXShift of {G} gathers ({ny} traces x {nx} samples, 0.25 ms, 50 Hz Ricker, "
                                   f"hyperbolic moveout, +-2 ms statics, 10 dB SNR) to their mean gather, lambda "
                                   f"{SEIS_LAMBDA}, yRegFactor {SEIS_YREG}, maxGDIterations {SEIS_ITER}, "
                                   f"{SEIS_WORKERS} concurrent descents",
                       "mean_steps": float(np.mean(st)), "parallelism": f"weak, {world} ranks"},
            "e2e": {"value": value, "unit": "gathers/s", "h2d_bytes_per_step": 2 * G * nx * ny * 8 + nx * ny * 8,
                    "d2h_bytes_per_step": G * nx * ny * 8},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": f"k_lineshift with its derivative, all {G} gathers in one launch "
                                                   f"(timed after the descents, {reps} launches)",
                         "achieved": ls_bytes / (ls_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": ls_bytes / (ls_ms * 1e-3) / 1e9 / peak, "peak_kind": peak_kind, "traffic": None,
                         "algorithmic_bytes_per_launch": ls_bytes, "avg_launch_ms": ls_ms},
            "cpu_baseline": cpu,
            "accuracy": accuracy,
            "clocks": {k: clk[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        }
        print(json.dumps(out), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


# --- learned warm start (--warm) -------------------------------------------
# --warm: the metric's own configuration, 20 frames 513^2 (levels 5-9); the
# network sees the prepared 513^2 pair and predicts level 8 (--warm-level 10:
# 50 frames 1025^2, levels 4-10, network input 1025^2, prediction level 9)
WARM_LEVEL, WARM_NET, WARM_START, WARM_FRAMES = 9, 9, 5, 20
WARM_TRAIN_SERIES, WARM_FPS, WARM_STEPS, WARM_BATCH, WARM_LR = 64, 8, 600, 8, 2e-3
WARM_TOL = 1e-6


def net_forward_flops(n0: int) -> float:
    """Algorithmic FLOPs of one network forward pass at input grid n0 (real channels)."""
    spec = [(2, 16, 1, 0), (16, 16, 1, 0), (16, 32, 2, 1), (32, 32, 1, 1), (32, 64, 2, 2), (64, 64, 1, 2),
            (64, 128, 2, 3), (128, 128, 1, 3), (192, 64, 1, 2), (64, 64, 1, 2), (96, 32, 1, 1), (32, 32, 1, 1),
            (32, 2, 1, 1)]
    grids = [n0]
    for _ in range(3):
        grids.append((grids[-1] + 1) // 2)
    return sum(2.0 * 9 * ci * co * grids[g] ** 2 for ci, co, _, g in spec)


def metric_legs(ctx, p, d_ref, d_tmpl, F, plain_ms, plain_e, fp64, local, rank):
    """The metric's two legs on the stage's own frames (one GPU): the plain
    GPU gradient flow one frame at a time, and warm start + batch to the
    stated energy tolerance (the plain batch's final energies + WARM_TOL
    relative; a frame that does not reach it is registered again from the
    plain start, counted in the time).  The network (input 513^2, output
    level 8) is trained first on pairs the plain method registers (untimed,
    reported)."""
    import numpy as np
    import torch
    import msgpu
    from msgpu import warmstart as ws
    dev = torch.device("cuda", local)
    st = torch.cuda.current_stream(dev)
    R, T, tgt, t_data = ws.training_set(ctx, level=LEVEL, net_level=LEVEL, num_series=WARM_TRAIN_SERIES,
                                        frames_per_series=WARM_FPS, seed=9000 + 1000 * rank, fp64=fp64,
                                        start_level=START)
    net = msgpu.Net(ctx, LEVEL, seed=1)
    _, t_train = ws.train(net, R, T, tgt, steps=WARM_STEPS, batch=WARM_BATCH, lr=WARM_LR, seed=rank)
    del R, T, tgt
    torch.cuda.empty_cache()
    N = d_tmpl.shape[1]
    nlev = LEVEL - START + 1
    phis = torch.empty((F, 2, N), dtype=torch.float64, device=dev)
    e = torch.empty(F, dtype=torch.float64, device=dev)
    s = torch.empty((F, nlev), dtype=torch.int32, device=dev)
    d_plain = torch.from_numpy(np.ascontiguousarray(plain_e)).to(dev)

    ctx.set_warm_schedule(WARM_COARSE_ITERS)

    def warm():
        return ctx.register_batch_warm_device(p, net, d_ref.data_ptr(), d_tmpl.data_ptr(), F, phis.data_ptr(),
                                              e.data_ptr(), s.data_ptr(), d_plain_energies=d_plain.data_ptr(),
                                              rel_tol=WARM_TOL, stream=st.cuda_stream)

    one = torch.empty((1, 2, N), dtype=torch.float64, device=dev)

    def single():
        for f in range(F):
            ctx.register_batch_device(p, d_ref.data_ptr(), d_tmpl[f].data_ptr(), 1, one.data_ptr(),
                                      stream=st.cuda_stream)

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            r = fn()
        e1.record(st)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / reps, r

    t_warm, used = timed(warm, 3)
    t_single, _ = timed(single, 1)
    ew = e.cpu().numpy()
    rel = (ew - plain_e) / np.abs(plain_e)
    net.close()
    return {
        "plain_gpu_batched_frames_per_s": F / (plain_ms * 1e-3),
        "plain_gpu_single_frame_frames_per_s": F / (t_single * 1e-3),
        "warm_batched_to_energy_tol_frames_per_s": F / (t_warm * 1e-3),
        "ratio_vs_plain_gpu_single_frame": t_single / t_warm,
        "ratio_vs_plain_gpu_batched": plain_ms / t_warm,
        "energy_tol_rel": WARM_TOL,
        "frames_within_tol": int(np.sum(rel <= WARM_TOL)),
        "fallback_frames": int(F - int(np.sum(used))),
        "steps_per_level_warm_to_tol": [round(float(x), 1) for x in s.float().mean(0).cpu().numpy()],
        "coarse_level_step_limit": WARM_COARSE_ITERS or None,
        "training": {"pairs": WARM_TRAIN_SERIES * WARM_FPS, "steps": WARM_STEPS, "seconds": t_train,
                     "data_seconds": t_data},
        "note": "the plain batch's final energies are the targets; frames that end above them by more than the "
                "tolerance are registered again from the plain start inside the timed region",
    }


def main_warm(args, world, rank, local):
    """--warm: registration started from the learned network's prediction, to
    the stated energy tolerance: the plain batch's final energies are the
    targets; the warm-started solve of the finest level stops as soon as a
    frame is within WARM_TOL of its target, and a frame that ends above it is
    registered again from the plain start (counted in the time)."""
    global WARM_LEVEL, WARM_NET, WARM_START, WARM_FRAMES
    if args.warm_level == 10:
        WARM_LEVEL, WARM_NET, WARM_START, WARM_FRAMES = 10, 10, 4, 50
    import numpy as np
    import torch
    import msgpu
    from msgpu import build as mbuild
    from msgpu import synthetic as syn
    from msgpu import warmstart as ws

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    mbuild.build()
    ctx = msgpu.Context(local)
    fp64 = not args.fp32
    # 1. training set from the plain method, training (untimed for the metric, reported)
    R, T, tgt, t_data = ws.training_set(ctx, level=WARM_LEVEL, net_level=WARM_NET, num_series=WARM_TRAIN_SERIES,
                                        frames_per_series=WARM_FPS, seed=9000 + 1000 * rank, fp64=fp64,
                                        start_level=WARM_START)
    Rv, Tv, tv, _ = ws.training_set(ctx, level=WARM_LEVEL, net_level=WARM_NET, num_series=2,
                                    frames_per_series=WARM_FPS, seed=9500 + 1000 * rank, fp64=fp64,
                                    start_level=WARM_START)
    net = msgpu.Net(ctx, WARM_NET, seed=1)
    losses, t_train = ws.train(net, R, T, tgt, steps=WARM_STEPS, batch=WARM_BATCH, lr=WARM_LR, seed=rank,
                               log_every=WARM_STEPS // 4)
    pred_mse, zero_mse = ws.prediction_error(net, Rv, Tv, tv)
    train_flops = 3.0 * net_forward_flops(msgpu.n_of(WARM_NET)) * WARM_BATCH * WARM_STEPS
    del R, T, tgt, Rv, Tv, tv
    torch.cuda.empty_cache()
    # 2. the evaluation series (device resident)
    n = msgpu.n_of(WARM_LEVEL)
    N = n * n
    F = WARM_FRAMES
    spec = syn.random_spec(np.random.default_rng(7000 + rank))
    frames = syn.make_series_torch(n, F + 1, spec, 7001 + 1000 * rank, dev).reshape(F + 1, N).contiguous()
    p = msgpu.default_params(precision_level=WARM_LEVEL, input_level=WARM_LEVEL, start_level=WARM_START,
                             stop_level=WARM_LEVEL, max_gd_iterations=MAX_ITER, use_fp64=int(fp64), lambda_=LAMBDA,
                             sum_order=SUM_ORDER)
    nlev = WARM_LEVEL - WARM_START + 1
    st = torch.cuda.current_stream(dev)
    outs = {k: (torch.empty((F, 2, N), dtype=torch.float64, device=dev),
                torch.empty(F, dtype=torch.float64, device=dev),
                torch.empty((F, nlev), dtype=torch.int32, device=dev)) for k in ("plain", "warm", "fallback")}
    launches = {}

    def plain():
        o = outs["plain"]
        ctx.register_batch_device(p, frames[0].data_ptr(), frames[1].data_ptr(), F, o[0].data_ptr(),
                                  o[1].data_ptr(), o[2].data_ptr(), stream=st.cuda_stream)
        launches["plain"] = ctx.stats()["kernel_launches"]

    def warm():
        o = outs["warm"]
        ctx.register_batch_warm_device(p, net, frames[0].data_ptr(), frames[1].data_ptr(), F, o[0].data_ptr(),
                                       o[1].data_ptr(), o[2].data_ptr(), stream=st.cuda_stream)
        launches["warm"] = ctx.stats()["kernel_launches"]

    def fallback():
        o = outs["fallback"]
        used = ctx.register_batch_warm_device(p, net, frames[0].data_ptr(), frames[1].data_ptr(), F,
                                              o[0].data_ptr(), o[1].data_ptr(), o[2].data_ptr(),
                                              d_plain_energies=outs["plain"][1].data_ptr(), rel_tol=WARM_TOL,
                                              stream=st.cuda_stream)
        launches["fallback"] = ctx.stats()["kernel_launches"]
        return used

    def timed(fn, reps):
        for _ in range(max(1, args.warmup - 2)):
            fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            r = fn()
        e1.record(st)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / reps, r

    barrier(world)
    with ClockSampler(local) as clocks:
        t_plain, _ = timed(plain, args.steps)
        t_warm, _ = timed(warm, args.steps)
        t_fb, used = timed(fallback, args.steps)
    # the network alone on the evaluation pairs (prepared images at its input level)
    prep = torch.empty((F + 1, msgpu.n_of(WARM_NET) ** 2), dtype=torch.float64, device=dev)
    ctx.prepare_images_device(p, frames.data_ptr(), F + 1, WARM_NET, prep.data_ptr(), st.cuda_stream)
    pred = torch.empty((F, 2, msgpu.n_of(WARM_NET - 1) ** 2), dtype=torch.float64, device=dev)
    t_net, _ = timed(lambda: net.predict_device(prep[0].data_ptr(), 0, prep[1].data_ptr(), F, pred.data_ptr(),
                                                st.cuda_stream), 5)
    # the plain method one frame at a time (the unbatched plain GPU flow), on 5 frames
    one = (torch.empty((1, 2, N), dtype=torch.float64, device=dev),)

    def single():
        for f in range(5):
            ctx.register_batch_device(p, frames[0].data_ptr(), frames[1 + f].data_ptr(), 1, one[0].data_ptr(),
                                      stream=st.cuda_stream)

    t_single, _ = timed(single, 1)
    t_single /= 5
    # end to end through the host entry point, host buffers (pinned)
    h_ref = frames[0].cpu().pin_memory()
    h_tm = frames[1:].cpu().pin_memory()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        wh, we, _, _ = ctx.register_batch_warm(p, net, h_ref.numpy(), h_tm.numpy())
    t_e2e = (time.perf_counter() - t0) / args.steps
    t_fb_max = allreduce_max(t_fb, world)
    ep = outs["plain"][1].cpu().numpy()
    ew = outs["warm"][1].cpu().numpy()
    ef = outs["fallback"][1].cpu().numpy()
    r = (ew - ep) / np.abs(ep)
    d_px = (outs["warm"][0] - outs["plain"][0]).abs().amax(dim=(1, 2)).cpu().numpy() * (n - 1)
    steps_w = outs["warm"][2].float().mean(0).cpu().numpy()
    steps_p = outs["plain"][2].float().mean(0).cpu().numpy()
    net_flops = net_forward_flops(msgpu.n_of(WARM_NET)) * F
    peak_tf = None
    try:
        peak_tf = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops"])
        peak_kind = "measured"
    except Exception:
        peak_tf, peak_kind = 1590.0, "fallback"
    if rank == 0:
        clk = clocks.summary()
        out = {
            "metric": METRIC, "value": world * F / (t_fb_max * 1e-3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_fb_max, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if fp64 else "f32+f64-reductions",
            "data": "synthetic lattice series (GPU generator), random lattice per series",
            "config": {"workload": f"{F} frames {n}x{n} registered to a reference frame, levels {WARM_START}-"
                                   f"{WARM_LEVEL}, maxGDIterations {MAX_ITER}; warm start: the network (input level "
                                   f"{WARM_NET}) predicts level {WARM_NET - 1}, the flow refines "
                                   f"{WARM_NET - 1}-{WARM_LEVEL} to the plain batch's final energies "
                                   f"(+{WARM_TOL} relative: the finest level stops there); frames that end above "
                                   f"are registered again from the plain start (counted in the time); a step is "
                                   f"the whole batch",
                       "lattice": {"kind": spec.kind, "spacing_px": round(spec.spacing, 2),
                                   "peak": round(spec.peak, 1), "max_disp_px": round(spec.max_disp, 2)},
                       "inputs": f"larger than L2 ({F} frames of {N * 8 / 1e6:.1f} MB)",
                       "parallelism": f"weak, {world} ranks"},
            "e2e": {"value": world * F / t_e2e, "unit": UNIT, "h2d_bytes_per_step": (F + 1) * N * 8,
                    "d2h_bytes_per_step": F * 2 * N * 8 + F * 8 + F * nlev * 4,
                    "note": "warm start without the fallback (the host entry point, pinned host buffers)"},
            "gpu_launches": launches.get("fallback"),
            "warm_start": {
                "plain_batched_frames_per_s": F / (t_plain * 1e-3),
                "warm_batched_frames_per_s": F / (t_warm * 1e-3),
                "warm_with_fallback_frames_per_s": F / (t_fb * 1e-3),
                "plain_single_frame_frames_per_s": 1.0 / (t_single * 1e-3),
                "gain_vs_plain_batched": t_plain / t_fb,
                "gain_vs_plain_single_frame": t_single * F / t_fb,
                "fallback_frames": int(F - int(np.sum(used))),
                "rel_energy_warm_vs_plain": {"median": float(np.median(r)), "min": float(r.min()),
                                             "max": float(r.max()), "within_tol": int(np.sum(r <= WARM_TOL)),
                                             "lower": int(np.sum(r <= 0))},
                "after_fallback_max_rel_energy": float(np.max((ef - ep) / np.abs(ep))),
                "max_dphi_px_warm_vs_plain": float(d_px.max()),
                "steps_per_level_plain": [round(float(x), 1) for x in steps_p],
                "steps_per_level_warm": [round(float(x), 1) for x in steps_w],
                "network_ms": t_net,
                "training": {"pairs": WARM_TRAIN_SERIES * WARM_FPS, "steps": WARM_STEPS, "batch": WARM_BATCH,
                             "seconds": t_train, "data_seconds": t_data,
                             "loss": [[k, round(l, 6)] for k, l in losses],
                             "heldout_mse_px2": pred_mse, "zero_start_mse_px2": zero_mse,
                             "tflops": train_flops / t_train / 1e12},
            },
            "roofline": {"bound": "tensor", "kernel": f"network forward (k_conv and its up/pack kernels), {F} "
                                                      f"pairs at {msgpu.n_of(WARM_NET)}^2",
                         "achieved": net_flops / (t_net * 1e-3) / 1e12, "peak": peak_tf, "unit": "TFLOP/s",
                         "frac": net_flops / (t_net * 1e-3) / 1e12 / peak_tf, "peak_kind": peak_kind,
                         "traffic": None, "algorithmic_flops_per_launch": net_flops, "avg_launch_ms": t_net},
            "cpu_baseline": None,
            "clocks": {k2: clk[k2] for k2 in ("sm_mhz", "sm_max_mhz", "reasons")},
        }
        print(json.dumps(out), flush=True)
    net.close()
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--fp32", action="store_true", help="FP32 bulk with FP64 reductions (outside the energy tol)")
    ap.add_argument("--no-warm-leg", action="store_true",
                    help="skip the metric's warm-start leg (network training + warm-started batch) of the default run")
    ap.add_argument("--autotune", action="store_true",
                    help="tune the level scheduler on the workload first (msgpu_autotune_device); writes the table "
                         "to gpurun_out/tuning.json when that folder exists")
    ap.add_argument("--sum-order", type=int, default=0, choices=[0, 1],
                    help="0: global sums in the reference's sequential order (bit-exact, default); "
                         "1: fixed parallel order")
    ap.add_argument("--no-certified", action="store_true",
                    help="with sum order 0: add every pass's sums in order before its control step (the results "
                         "are the same; for comparisons)")
    ap.add_argument("--warm-coarse-iters", type=int, default=4,
                    help="warm leg: step limit of the levels below the stop level (0: maxGDIterations; "
                         "default 4, the best of 0, 3, 4, 6, 8, 12 measured on B200)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ncc", action="store_true",
                    help="normalized cross-correlation data term (matchSeries' default model) instead of SSD")
    ap.add_argument("--profile-level", type=int, default=0,
                    help="small case for ncu captures: one level solve of FRAMES frames at this level, "
                         "--profile-iters gradient steps, no timing")
    ap.add_argument("--profile-iters", type=int, default=5)
    ap.add_argument("--trace-out", default="",
                    help="with --profile-level: save the level kernel's pass timeline (msgpu_set_trace) "
                         "to this .npz")
    ap.add_argument("--profile-compose", type=int, default=0,
                    help="small case for ncu: one displacement composition at this level, no timing")
    ap.add_argument("--profile-series", action="store_true",
                    help="small case for ncu: one msgpu_match_series call on the bench's frames, no timing")
    ap.add_argument("--profile-seismic", type=int, default=0,
                    help="small case for ncu: findXShift of one gather 257 x 2049 with this many steps, no timing")
    ap.add_argument("--seismic", action="store_true",
                    help="the seismic line-shift model: findXShift of 32 gathers 257 x 2049")
    ap.add_argument("--ragged", action="store_true",
                    help="uneven series of 129^2..1025^2 in one ragged batch (msgpu_register_ragged)")
    ap.add_argument("--files", action="store_true",
                    help="series read from .q2bz files, decoding overlapped with the GPU stages")
    ap.add_argument("--warm-level", type=int, default=9, choices=[9, 10],
                    help="--warm at 513^2 x 20 frames (9, the metric's configuration) or 1025^2 x 50 frames (10)")
    ap.add_argument("--warm", action="store_true",
                    help="the learned warm start: train the network, then 50 frames 1025^2 warm-started vs plain")
    ap.add_argument("--profile-net", type=int, default=0,
                    help="small case for ncu: this many network training steps at input level 9, batch 4")
    ap.add_argument("--profile-predict", type=int, default=0,
                    help="case for the ncu launch list: network predictions of 8 pairs at 1025^2, this many times")
    ap.add_argument("--series", action="store_true",
                    help="time matchSeries' whole first stage with accumulated deformations (msgpu_match_series)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    global DATA_TERM, SUM_ORDER, CERTIFIED, WARM_COARSE_ITERS
    DATA_TERM = 1 if args.ncc else 0
    SUM_ORDER = args.sum_order
    CERTIFIED = not args.no_certified
    WARM_COARSE_ITERS = args.warm_coarse_iters
    if args.profile_level:
        return profile_case(args.profile_level, args.profile_iters, not args.fp32, args.trace_out)
    if args.profile_compose or args.profile_series:
        return profile_series(args.profile_compose, not args.fp32)
    if args.profile_predict:
        import torch
        import msgpu
        from msgpu import build as mbuild
        mbuild.build()
        ctx = msgpu.Context(0)
        net = msgpu.Net(ctx, 10, seed=1)
        B, n0, n1 = 8, msgpu.n_of(10), msgpu.n_of(9)
        g = torch.Generator(device="cuda").manual_seed(0)
        R = torch.rand((B, n0 * n0), dtype=torch.float64, device="cuda", generator=g)
        T = torch.rand((B, n0 * n0), dtype=torch.float64, device="cuda", generator=g)
        phi = torch.empty((B, 2, n1 * n1), dtype=torch.float64, device="cuda")
        for _ in range(args.profile_predict):
            net.predict_device(R.data_ptr(), n0 * n0, T.data_ptr(), B, phi.data_ptr())
        torch.cuda.synchronize()
        print(json.dumps({"profile_predict": args.profile_predict, "launches": ctx.stats()["kernel_launches"]}))
        return 0
    if args.profile_net:
        import torch
        import msgpu
        from msgpu import build as mbuild
        mbuild.build()
        ctx = msgpu.Context(0)
        net = msgpu.Net(ctx, 9, seed=1)
        B, n0, n1 = 4, msgpu.n_of(9), msgpu.n_of(8)
        g = torch.Generator(device="cuda").manual_seed(0)
        R = torch.rand((B, n0 * n0), dtype=torch.float64, device="cuda", generator=g)
        T = torch.rand((B, n0 * n0), dtype=torch.float64, device="cuda", generator=g)
        t = torch.randn((B, 2, n1 * n1), dtype=torch.float64, device="cuda", generator=g) / (n1 - 1)
        for _ in range(args.profile_net):
            loss = net.train_step_device(R.data_ptr(), n0 * n0, T.data_ptr(), t.data_ptr(), B, 1e-3)
        print(json.dumps({"profile_net_steps": args.profile_net, "loss": loss,
                          "launches_per_step": ctx.stats()["kernel_launches"]}))
        return 0
    if args.profile_seismic:
        import msgpu
        from msgpu import build as mbuild
        from msgpu import synthetic as syn
        mbuild.build()
        g = syn.seismic_gathers(2, seed=4000)
        ctx = msgpu.Context(0)
        _, e, st = ctx.find_xshift(g.mean(axis=0), g[0], SEIS_LAMBDA, SEIS_YREG, args.profile_seismic)
        print(json.dumps({"profile_seismic_steps": st, "energy": e, "launches": ctx.stats()["kernel_launches"]}))
        return 0
    world, rank, local = dist_setup()
    if args.impl == "reference":
        return run_reference_arm(args, world, rank)
    if args.series:
        return main_series(args, world, rank, local)
    if args.files:
        return main_files(args, world, rank, local)
    if args.ragged:
        return main_ragged(args, world, rank, local)
    if args.seismic:
        return main_seismic(args, world, rank, local)
    if args.warm:
        return main_warm(args, world, rank, local)

    import numpy as np
    import torch
    import msgpu
    from msgpu import build as mbuild
    from msgpu import synthetic as syn

    torch.cuda.set_device(local)
    mbuild.build()
    fp64 = not args.fp32
    p = params(fp64)
    ref, tmpl, clean_ref = workload(rank)
    n = (1 << LEVEL) + 1
    N = n * n
    nlev = LEVEL - START + 1
    ctx = msgpu.Context(local)
    ctx.set_certified_steps(CERTIFIED)
    dev = torch.device("cuda", local)
    d_ref = torch.from_numpy(ref).to(dev)
    d_tmpl = torch.from_numpy(tmpl).to(dev)
    d_phis = torch.empty((FRAMES, 2, N), dtype=torch.float64, device=dev)
    d_e = torch.empty(FRAMES, dtype=torch.float64, device=dev)
    d_s = torch.empty((FRAMES, nlev), dtype=torch.int32, device=dev)
    d_mean = torch.empty(N, dtype=torch.float64, device=dev)
    d_count = torch.empty(N + 1, dtype=torch.float64, device=dev)   # slot N: fill of pixels without samples
    d_sum = torch.empty(N, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)

    tuned = None
    if args.autotune:
        scratch = torch.empty_like(d_phis)
        tuned = ctx.autotune_device(p, d_ref.data_ptr(), d_tmpl.data_ptr(), FRAMES, scratch.data_ptr(),
                                    stream.cuda_stream)
        if rank == 0 and os.path.isdir(os.path.join(ROOT, "gpurun_out")):
            key = "fp64" if fp64 else "fp32"
            json.dump({"device": torch.cuda.get_device_name(dev),
                       "workload": f"{FRAMES} frames 513x513, levels {START}-{LEVEL}, sum order {SUM_ORDER}",
                       "levels": {key: {str(k): v for k, v in tuned.items()}}},
                      open(os.path.join(ROOT, "gpurun_out", "tuning.json"), "w"), indent=1)
    elif os.path.exists(os.path.join(ROOT, "match-series_b200", "msgpu", "tuning_b200.json")):
        ctx.load_tuning()

    def step():
        if world == 1:
            ctx.match_series_stage_device(p, d_ref.data_ptr(), d_tmpl.data_ptr(), FRAMES, d_phis.data_ptr(),
                                          d_e.data_ptr(), d_s.data_ptr(), d_mean.data_ptr(), d_count.data_ptr(),
                                          stream.cuda_stream)
            return
        # sharded stage: every rank registers its frames; the average needs the
        # ranks' per-pixel sums and counts added (one NCCL all-reduce each)
        import torch.distributed as dist
        ctx.register_batch_device(p, d_ref.data_ptr(), d_tmpl.data_ptr(), FRAMES, d_phis.data_ptr(), d_e.data_ptr(),
                                  d_s.data_ptr(), 0, stream.cuda_stream)
        last = rank == world - 1   # holds the series' last frame: its mean fills empty pixels
        ctx.warp_sum_device(LEVEL, d_tmpl.data_ptr(), d_phis.data_ptr(), FRAMES, d_sum.data_ptr(), d_count.data_ptr(),
                            d_count[N:].data_ptr() if last else 0, stream.cuda_stream)
        if not last:
            d_count[N:].zero_()
        dist.all_reduce(d_sum)
        dist.all_reduce(d_count)
        ctx.mean_from_sums_device(LEVEL, d_sum.data_ptr(), d_count.data_ptr(), d_count[N:].data_ptr(),
                                  d_mean.data_ptr(), stream.cuda_stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    # ---- device-resident timed region (profiling events per level launch)
    ctx.set_profiling(True)
    lvl_ms, lvl_steps, lvl_evals, launches = [], [], [], 0
    start_ev = torch.cuda.Event(enable_timing=True)
    stop_ev = torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clocks:
        start_ev.record(stream)
        for _ in range(args.steps):
            step()
            st = ctx.stats()
            lvl_ms.append(st["level_ms"][-1])
            lvl_steps.append(st["level_steps"][-1])
            lvl_evals.append(st["level_evals"][-1])
            launches += st["kernel_launches"]
        stop_ev.record(stream)
        torch.cuda.synchronize(dev)
    barrier(world)
    ctx.set_profiling(False)
    elapsed_ms = allreduce_max(start_ev.elapsed_time(stop_ev), world)
    ms_per_step = elapsed_ms / args.steps
    value = world * FRAMES * args.steps / (elapsed_ms / 1000.0)
    phis = d_phis.cpu().numpy()
    energies = d_e.cpu().numpy()
    mean = d_mean.cpu().numpy()
    steps_per_level = d_s.cpu().numpy()

    # ---- end to end through the host entry point, pinned host buffers
    h_ref = torch.from_numpy(ref).pin_memory().numpy()
    h_tmpl = torch.from_numpy(tmpl).pin_memory().numpy()
    outs = (torch.zeros((FRAMES, 2, N), dtype=torch.float64).pin_memory().numpy(),
            torch.zeros(FRAMES, dtype=torch.float64).pin_memory().numpy(),
            torch.zeros((FRAMES, nlev), dtype=torch.int32).pin_memory().numpy(),
            torch.zeros(N, dtype=torch.float64).pin_memory().numpy(),
            torch.zeros(N, dtype=torch.float64).pin_memory().numpy())
    def e2e_step():
        if world == 1:
            ctx.match_series_stage(p, h_ref, h_tmpl, out=outs)
            return
        # host buffers in and out around the sharded device step
        d_ref.copy_(torch.from_numpy(h_ref), non_blocking=True)
        d_tmpl.copy_(torch.from_numpy(h_tmpl), non_blocking=True)
        step()
        outs[0][...] = d_phis.cpu().numpy()
        outs[1][...] = d_e.cpu().numpy()
        outs[2][...] = d_s.cpu().numpy()
        outs[3][...] = d_mean.cpu().numpy()
        outs[4][...] = d_count[:N].cpu().numpy()

    e2e_step()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = allreduce_max(time.perf_counter() - t0, world)
    e2e_value = world * FRAMES * args.steps / e2e_s
    h2d = (1 + FRAMES) * N * 8
    d2h = (2 * FRAMES * N + 2 * N + FRAMES) * 8 + FRAMES * nlev * 4

    out = None
    if rank == 0:
        peak, peak_kind = measured_peak()
        real_bytes = 8 if fp64 else 4
        avg_ms = statistics.mean(lvl_ms)
        alg = statistics.mean(algorithmic_bytes(s, e, real_bytes) for s, e in zip(lvl_steps, lvl_evals))
        achieved = alg / (avg_ms / 1000.0) / 1e9
        traffic = level_traffic(fp64)
        clk = clocks.summary()
        cpu = None
        accuracy = None
        if world == 1 and not args.no_cpu_baseline:
            procs = min(cpu_procs(), FRAMES)
            with tempfile.TemporaryDirectory() as wd:
                nfr, secs, rphis, renergies, kind, wall = run_reference_sample(ref, tmpl, procs, wd)
            cpu = {"value": nfr / secs, "unit": UNIT, "cores": procs, "kind": kind,
                   "sample": f"{nfr} of the 20 frames (513x513, levels {START}-{LEVEL}), one process per core, "
                             f"registration phase {secs:.1f} s"}
            dphi = float(np.abs(phis[:nfr] - rphis).max()) * (n - 1)
            rel = float(np.max(np.abs(energies[:nfr] - renergies) / np.abs(renergies)))
            identical = int(sum(np.array_equal(phis[f], rphis[f]) and energies[f] == renergies[f]
                                for f in range(nfr)))
            # the reference's own sensitivity: the same frames with every pixel
            # of the reference frame moved by one ulp in a random direction (a
            # perturbation of the size of a reordered floating-point sum)
            ref_p = ref.copy()
            up = np.random.default_rng(7).random(ref_p.size) < 0.5
            ref_p = np.where(up, np.nextafter(ref_p, np.inf), np.nextafter(ref_p, -np.inf))
            with tempfile.TemporaryDirectory() as wd:
                _, _, pphis, penergies, _, _ = run_reference_sample(ref_p, tmpl, procs, wd)
            sp_dphi = float(np.abs(pphis - rphis).max()) * (n - 1)
            sp_rel = float(np.max(np.abs(penergies - renergies) / np.abs(renergies)))
            accuracy = {"frames_checked": nfr, "frames_bit_identical": identical,
                        "max_dphi_px": dphi, "max_rel_energy": rel,
                        "tolerance": {"dphi_px": 1e-3, "rel_energy": 1e-6},
                        "within_tolerance": bool(dphi <= 1e-3 and rel <= 1e-6),
                        "reference_1ulp_spread": {"max_dphi_px": sp_dphi, "max_rel_energy": sp_rel,
                                                  "perturbation": "every pixel of the reference frame "
                                                                  "+-1 ulp (random signs)"}}
        legs = None
        if world == 1 and not args.no_warm_leg:
            legs = metric_legs(ctx, p, d_ref, d_tmpl, FRAMES, ms_per_step, energies, fp64, local, rank)
        psnr = syn.psnr(mean.reshape(n, n), clean_ref)
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if fp64 else "f32+f64-reductions", "data": "synthetic",
            "config": {"workload": f"stage registration: {FRAMES} hex-lattice frames 513x513 (level {LEVEL}) to a "
                                   f"reference frame, levels {START}-{LEVEL}, maxGDIterations {MAX_ITER}, "
                                   f"lambda {LAMBDA}, saturation 0.15%, {'NCC' if DATA_TERM else 'SSD'} data term, "
                                   f"plus warped-frame average",
                       "data_term": "ncc" if DATA_TERM else "ssd",
                       "frames_per_gpu": FRAMES, "level": LEVEL, "start_level": START,
                       "max_gd_iterations": MAX_ITER, "lambda": LAMBDA,
                       "l2": "no flush: per-step working set (~0.6 GB) exceeds the 126 MB L2",
                       "parallelism": ("one GPU" if world == 1 else
                                       f"weak: {world} ranks register {FRAMES} frames each of one series against "
                                       f"its reference; the average adds the ranks' per-pixel sums and counts "
                                       f"(NCCL all-reduce)")},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "tuning": tuned if tuned is not None else "table" if os.path.exists(
                os.path.join(ROOT, "match-series_b200", "msgpu", "tuning_b200.json")) else "defaults",
            "roofline": {"bound": "hbm", "kernel": f"level_kernel<{'double' if fp64 else 'float'}> level {LEVEL}",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "traffic": traffic,
                         "algorithmic_bytes_per_launch": alg, "avg_launch_ms": avg_ms,
                         "steps_per_launch": statistics.mean(lvl_steps),
                         "energy_evals_per_launch": statistics.mean(lvl_evals)},
            "cpu_baseline": cpu,
            "metric_legs": legs,
            "accuracy": accuracy,
            "reconstruction_psnr_db": psnr,
            "steps_per_level_frame0": steps_per_level[0].tolist(),
            "clocks": {k: clk[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        }
        print(json.dumps(out), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
