#!/usr/bin/env python
"""Train rays/s of the NeAT forward-projection training step on B200.

A step = one fused neat_train_step over a batch of rays: camera rays,
ray-octree intersection + stratified sampling, IGS + decoder + softplus, line
integral, MSE, hand-written backward, Adam on grid and decoder.

Default workload (N=1): the plain FP32 full-size configuration -- phantom of
64 random ellipsoids + 200 void spheres, 360 projections of 512x512 with
Poisson noise (I0 = 1e4), octree of max depth 4 refined by density variance
to ~1500 active nodes, C=8 features on G=17 grids, decoder 8->64->64->1,
32 samples per node segment, 2^18 rays per batch.  Synthetic data stands in
for the reference's measured scans.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Multi-GPU: the path is data parallel over rays with no exchange in this
build (replicas only): every rank trains its own replica on its own batches,
timing is the max over ranks, value = all rays processed / that time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from neat_b200.workloads import WORKLOADS, build_workload, phantom  # noqa: E402

METRIC = "train rays/s (fwd+bwd)"
DECODER_DESC = {"simt": "FP32 FFMA (CUDA cores)",
                "bf16x3": "tcgen05, FP32-accurate: operands split in 3 BF16 pieces, 6 products, FP32 accumulation",
                "bf16": "tcgen05, BF16 operands, FP32 accumulation (precision variant)"}
CPU_PATH_DESC = ("reference CPU IGS fwd/bwd compiled from its source (oracle/_ref), OpenMP C port of the CUDA-only "
                 "ComputeRaySamples, libtorch-CPU decoder/softplus/index_add/MSE/autograd/Adam")
PHASES = ["segments", "forward_tiles", "loss", "backward_tiles", "adam"]
# kernels one neat_train_step launches: step scalars, rays, hit lists, 2 scans
# x 3 kernels and the one-block scan of the node counts, placement (with the
# segment capacity check and the partials' zeroing), tile map (with the
# sample capacity check), forward tiles, ray loss, loss total, backward tiles,
# decoder Adam, grid Adam
STEP_LAUNCHES = 18
# DRAM bytes per sample of the records backward (k_bwd_rec), dram__bytes_read.sum +
# dram__bytes_write.sum of one launch in a single-pass ncu capture, scaled to the
# measured launch by its samples:
TRAFFIC_BYTES_PER_SAMPLE = {
    # BF16x3 at the full-size workload itself (2^18 rays, 11.64 M samples): 886.6 + 176.5 MB
    ("full", "bf16x3"): (1063.1e6 / 11.6376e6, "ncu capture of a full-size launch (2^18 rays), per sample"),
    # BF16, same scene at 2^16 rays (2.908 M samples): 344.3 + 120.8 MB -- an upper bound at
    # larger batches, which reuse more of the grid gradient in L2
    ("full", "bf16"): (465.1e6 / 2.908e6, "ncu capture at 2^16 rays scaled by samples (upper bound)")}
KERNEL_NAME = {"simt": "k_step_tiles<C=%d, backward> (FP32 SIMT)",
               "bf16x3": "k_bwd_rec<C=%d, BF16x3> (backward from the forward's records, MMA warp)",
               "bf16": "k_bwd_rec<C=%d, BF16> (backward from the forward's records, MMA warp)"}
PSNR_TARGET_DB = 40.0


PROPOSAL_ITERS = 10  # proposal Adam iterations on a TRAIN step (FusedTrainer default)
PREFETCH = True      # timed steps build the next batch's segment lists under their Adam (--no-prefetch: off)


def step_launches(decoder, C, proposal, train):
    """Kernels one neat_train_step launches: STEP_LAUNCHES, plus the records
    backward (three pieces at C = 4, 8; BF16 at C = 4, 8, 16; the plain
    backward kernel then returns at once); with the learned proposal a SAMPLE step adds the CDF
    kernel and a TRAIN step the histogram zeroing, the segments' density
    variation, the node descriptors and 3 kernels per proposal iteration."""
    records = (decoder == "bf16x3" and C in (4, 8)) or (decoder == "bf16" and C in (4, 8, 16))
    n = STEP_LAUNCHES + (1 if records else 0)
    if proposal:
        n += (3 + 3 * PROPOSAL_ITERS) if train else 1
    return n


def hidden_flops(C, H=64):
    return C * H + H * H + H  # multiply-adds of one decoder forward


def step_roofline(S, R, P, C, ms_step, peaks, simt_peak_tflops, H=64):
    """Whole-step roofline of the path: T* = max(F / peak flops, B / HBM bandwidth) and
    achieved = T* / measured step time.  F = 6 (C H + H^2 + H) flops per sample (the decoder
    forward, its dX and its weight-gradient products); B = 16 R + 36 P bytes (per ray: target,
    ray key, prediction; per FP32 grid parameter: the step's grid read and gradient write, 8 B,
    and Adam's reads of p, g, m, v and writes of p, m, v, 28 B).  Reported against the measured
    tensor-core (BF16, sustained) and the FP32 CUDA-core flop peaks."""
    F = 6.0 * hidden_flops(C, H) * S
    B = 16.0 * R + 36.0 * P
    t_hbm = B / (peaks["hbm_gbs"] * 1e9)
    t_tc = F / (peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops")) * 1e12)
    t_simt = F / (simt_peak_tflops * 1e12)
    t = ms_step / 1000.0
    return {"flops": F, "bytes": B,
            "t_star_ms_tensor": 1e3 * max(t_tc, t_hbm), "bound_tensor": "hbm" if t_hbm >= t_tc else "tensor",
            "frac_tensor": max(t_tc, t_hbm) / t,
            "t_star_ms_fp32_simt": 1e3 * max(t_simt, t_hbm), "bound_fp32_simt": "hbm" if t_hbm >= t_simt else "fp32",
            "frac_fp32_simt": max(t_simt, t_hbm) / t}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


# --------------------------------------------------------------------------
# clocks
# --------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples of the SM clock and throttle reasons taken while the
    timed region runs.  The sampler is started, and its first sample awaited,
    before the region begins (nvidia-smi needs a few hundred ms to start); a
    sample counts when it arrives between begin() and end() (plus one
    interval).  If the region is shorter than an interval, the sample on each
    side of it is reported instead, and `samples_in_region` says so."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    INTERVAL_MS = 20

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []  # (arrival time, line)
        self.t_begin = self.t_end = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.INTERVAL_MS)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
            return
        t0 = time.monotonic()
        while not self.lines and time.monotonic() - t0 < 10.0 and self.proc.poll() is None:
            time.sleep(0.005)

    def begin(self):
        self.t_begin = time.monotonic()

    def end(self):
        self.t_end = time.monotonic()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(3 * self.INTERVAL_MS / 1000.0)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        lines = list(self.lines)
        tb = self.t_begin if self.t_begin is not None else -1e30
        te = (self.t_end if self.t_end is not None else 1e30) + self.INTERVAL_MS / 1000.0
        inside = [ln for t, ln in lines if tb <= t <= te]
        n_inside = len(inside)
        if not inside:
            before = [ln for t, ln in lines if t < tb][-1:]
            after = [ln for t, ln in lines if t > te][:1]
            inside = before + after
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in inside:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "samples_in_region": n_inside, "interval_ms": self.INTERVAL_MS}


# --------------------------------------------------------------------------
# workload
# --------------------------------------------------------------------------
def cpu_tree(cfg, objs):
    """The configuration's octree refined with the oracle's density (the CPU
    leg has no device projector)."""
    from oracle import oracle as O
    from neat_b200.tree import HyperTreeBase
    tree = HyperTreeBase(3, cfg["depth"])
    if cfg["active"]:
        tree.RefineByVariance(lambda p: O.phantom_density(objs, p), cfg["active"], samples_per_axis=4)
    else:
        tree.SetActive(cfg["depth"])
    return tree


# --------------------------------------------------------------------------
# CPU path (oracle port of the reference's CPU execution) -- baseline only
# --------------------------------------------------------------------------
def cpu_reference_rays_per_s(cfg, steps, warmup, budget_s=None, min_s=None):
    """Times the CPU restatement of the step: C oracle rays + samples + IGS
    (reference CPU semantics), libtorch-CPU decoder / softplus / index_add /
    MSE / autograd / Adam, with all host threads.  Runs `steps` steps, fewer
    once budget_s is spent, more (up to 4x) until min_s is reached.
    Returns (rays/s, info)."""
    from oracle import cpu_reference as CR
    objs = phantom(cfg)
    tree = cpu_tree(cfg, objs)
    runner = CR.CpuReferenceStep(objs, tree, cfg)
    R = cfg["cpu_rays"]
    max_steps = steps if min_s is None else 4 * steps
    batches = [runner.batch(R) for _ in range(warmup + max_steps)]  # host data loading is not timed
    for i in range(warmup):
        runner.run(*batches[i], i + 1)
    t0 = time.perf_counter()
    done = 0
    for i in range(max_steps):
        runner.run(*batches[warmup + i], warmup + i + 1)
        done += 1
        el = time.perf_counter() - t0
        if budget_s is not None and el > budget_s:
            break
        if done >= steps and (min_s is None or el >= min_s):
            break
    dt = time.perf_counter() - t0
    kind = "reference" if CR.reference_igs() is not None else "port"
    return R * done / dt, dict(cores=torch.get_num_threads(), rays=R, steps=done, seconds=dt,
                               samples_per_ray=runner.last_samples / R, kind=kind)


# --------------------------------------------------------------------------
# time to PSNR (small workload, CUDA-graph steps)
# --------------------------------------------------------------------------
def time_to_psnr(dev, decoders, target_db=PSNR_TARGET_DB, max_steps=3000, every=50):
    """Train the small workload (config-1 shapes) from the same initial state
    with each decoder path until the projection PSNR of 4 held-out views
    (every 8th of the 32) reaches target_db.  PSNR = 10 log10(1 / MSE), MSE
    the mean over the views of each view's pixel mean (EvalStepProjection,
    samples/reconstruct.cpp:504-707), squared errors summed in f64.  Training
    time = CUDA-event time of the graph-replayed steps; evaluation not counted."""
    from neat_b200 import _lib
    from neat_b200.trainer import FusedTrainer
    cfg = dict(WORKLOADS["small"])
    scene, tree, cam = build_workload(cfg, dev)
    n = cfg["n_angles"]
    eval_ids = list(range(0, n, 8))
    train_ids = [i for i in range(n) if i not in eval_ids]
    gen = torch.Generator(device=dev)
    gen.manual_seed(77)
    batches = [scene.sample_batch(cfg["R"], gen, images=train_ids) for _ in range(max_steps)]
    out = {}
    for name in decoders:
        path = {"simt": _lib.NEAT_DECODER_SIMT_FP32, "bf16x3": _lib.NEAT_DECODER_TC_BF16X3,
                "bf16": _lib.NEAT_DECODER_TC_BF16}[name]
        tr = FusedTrainer(tree, cam, cfg["C"], cfg["G"], cfg["M"], lr_grid=1e-2, lr_decoder=5e-5, seed=cfg["seed"],
                          decoder_path=path, device=dev)
        tr.graph_step(*batches[0])  # captures the graph (and runs step 1, not timed)
        torch.cuda.synchronize()
        ms, k, curve, reached, psnr = 0.0, 1, [], False, 0.0
        while k < max_steps and not reached:
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(min(every, max_steps - k)):
                tr.graph_step(*batches[k])
                k += 1
            e1.record()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
            psnr = tr.eval_projection(eval_ids, scene.projection)["psnr"]
            curve.append([k, round(ms, 3), round(psnr, 3)])
            reached = psnr >= target_db
        tr.check_status()
        out[name] = {"reached": reached, "steps": k, "train_ms": ms, "psnr_db": psnr,
                     "ms_per_step": ms / max(k - 1, 1), "curve_every_%d_steps" % every: curve}
    return {"workload": cfg["desc"], "target_psnr_db": target_db, "lr_grid": 1e-2,
            "eval": "4 held-out views (every 8th of 32), all pixels, a = 0.5 samples; PSNR = 10 log10(1/MSE)",
            "timing": "CUDA events around CUDA-graph replays of the fused step (batches pre-staged on the "
                      "device); evaluation excluded", "paths": out}


# --------------------------------------------------------------------------
# variants of the step at the full-size workload
# --------------------------------------------------------------------------
PATH_NAMES = ("simt", "bf16x3", "bf16")


def decoder_path(name):
    from neat_b200 import _lib
    return {"simt": _lib.NEAT_DECODER_SIMT_FP32, "bf16x3": _lib.NEAT_DECODER_TC_BF16X3,
            "bf16": _lib.NEAT_DECODER_TC_BF16}[name]


# the count head's tolerance: a segment gets ceil(exp(v) / eps) samples (at most
# the budget, at least 2), v its predicted log(length x density variation); the
# midpoint rule then misses about eps / 2 of its integral at density jumps,
# below the projections' Poisson noise at I0 = 1e4 (about 0.01)
COUNT_EPS = 0.05
# uniform share of the proposal's placement density in training: the more
# uniform the placement, the sooner the volume-PSNR race's target is reached
# (with the count head at 0.05: 3800 steps at mix 0.25, 3500 at 0.75)
PROPOSAL_MIX = 0.75
# proposal lines are timed over one 50-step cycle after this many: the count
# head's sample counts settle within about 1000 steps (3.4 M samples a step
# over the first 100 steps of the race, 2.3 M from step 1000 on)
PROPOSAL_WARM_CYCLES = 20


def make_trainer(cfg, tree, cam, dev, decoder, proposal, seed):
    """FusedTrainer of a workload: decoder path by name; with the learned
    proposal the BF16 grid copy, the workload's sample budget, the count head's
    sample counts and a 50-step proposal cycle (one uniform TRAIN step, then
    SAMPLE steps)."""
    from neat_b200.trainer import FusedTrainer
    kw = dict(decoder_path=decoder_path(decoder), device=dev)
    if proposal:
        kw.update(proposal=True, proposal_budget=cfg.get("proposal_budget", 12), proposal_every=50,
                  grid_bf16=decoder == "bf16", proposal_count_eps=cfg.get("count_eps", COUNT_EPS),
                  proposal_count_min=2, proposal_mix=cfg.get("proposal_mix", PROPOSAL_MIX))
    elif decoder == "bf16":
        kw.update(grid_bf16=True)
    tr = FusedTrainer(tree, cam, cfg["C"], cfg["G"], cfg["M"], lr_grid=1e-2, lr_decoder=5e-5, seed=seed, **kw)
    tr.reserve(cfg["R"])
    return tr


def time_steps(tr, batches, phase_events=True):
    """CUDA-event time of tr.step over the batches (one stream), the mean
    per-phase times and the total samples of the steps (copied to pinned host
    memory after each step, no synchronisation inside)."""
    from neat_b200 import _lib
    K = len(batches)
    ev = None
    if phase_events:
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(_lib.NEAT_STEP_PHASES)] for _ in range(K)]
        for row in ev:  # torch creates the CUDA event on first record; the step records it again
            for e in row:
                e.record()
    counts = torch.zeros((K, 4), dtype=torch.int64).pin_memory()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for i, b in enumerate(batches):
        # the next batch's segment lists build under this step's Adam update
        nxt = batches[i + 1] if PREFETCH and i + 1 < K else None
        tr.step(*b, phase_events=ev[i] if ev else None, next=nxt)
        counts[i].copy_(tr.counters, non_blocking=True)
    t1.record()
    torch.cuda.synchronize()
    tr.check_status()
    ms = t0.elapsed_time(t1)
    phase_ms = None
    if ev:
        phase_ms = {p: sum(ev[i][j].elapsed_time(ev[i][j + 1]) for i in range(K)) / K for j, p in enumerate(PHASES)}
    return ms, phase_ms, counts


def step_variants(cfg, scene, tree, cam, dev, ref_rays_per_s, steps=50):
    """rays/s of the plain FP32 SIMT step, the BF16 step (BF16 grid copy and
    decoder operands, FP32 accumulation) and the BF16 step with the learned
    proposal (budget 12 samples per segment, fewer where the count head
    predicts little variation; one full 50-step cycle, its uniform TRAIN step
    included, after 20 cycles that train the proposal and its count head to
    their steady state; the race below covers training from the start), CUDA
    events around
    each timed loop; the BF16 + proposal step against both FP32 steps
    (ref_rays_per_s: the FP32-accurate tensor-core step of the main line)."""
    R = cfg["R"]
    gen = torch.Generator(device=dev)
    gen.manual_seed(4242)
    batches = [scene.sample_batch(R, gen) for _ in range(steps)]
    out = {}
    for name, dec, prop in (("fp32_simt", "simt", False), ("bf16", "bf16", False), ("bf16_proposal12", "bf16", True)):
        tr = make_trainer(cfg, tree, cam, dev, dec, prop, cfg["seed"])
        k = steps if prop else 10
        for i in range(3 if not prop else PROPOSAL_WARM_CYCLES * steps):
            tr.step(*batches[i % steps])
        ms, phase_ms, counts = time_steps(tr, batches[:k])
        out[name] = {"rays_per_s": R * k / (ms / 1000.0), "ms_per_step": ms / k, "steps": k,
                     "samples_per_step": float(counts[:, 1].double().mean()), "phase_ms": phase_ms}
        del tr
        torch.cuda.empty_cache()
    out["bf16_proposal12_vs_fp32_simt"] = out["bf16_proposal12"]["rays_per_s"] / out["fp32_simt"]["rays_per_s"]
    out["bf16_proposal12_vs_fp32_accurate_tcgen05"] = out["bf16_proposal12"]["rays_per_s"] / ref_rays_per_s
    out["note"] = ("ratios of rays/s on the same workload: against the FP32 SIMT step (FP32 FFMA on CUDA cores) and "
                   "against the FP32-accurate tcgen05 step of the main line (3-piece BF16 operands)")
    return out


def volume_psnr_race(cfg, scene, tree, cam, dev, steps, every=100, vol_n=256):
    """Time to the plain method's volume PSNR.  The plain method (FP32-accurate
    decoder, uniform 32 samples) trains `steps` steps; its final volume PSNR is
    the target.  Then BF16 + learned proposal (budget 12 samples per segment,
    fewer where the count head predicts little variation) trains until it
    reaches the target within 0.1 dB (at most `steps` steps), and so do two
    ablations of the learned part, BF16 with uniform samples and no network:
    12 per segment (the same budget) and the uniform budget whose samples per
    step come closest to the proposal run's mean (the same number of samples,
    spread evenly).  All runs see the same batches from the same initial state
    and are evaluated every `every` steps; each run's time to the target -
    0.1 dB is the CUDA-event time of its training steps up to the first
    evaluation at or above it (evaluations excluded).  Volume PSNR =
    10 log10(peak^2 / MSE) over the vol_n^3 voxel-corner lattice
    (UniformSampledVolume) against the f64 phantom density, peak = the
    phantom's maximum, MSE in f64."""
    gt = scene.density_volume(vol_n)
    peak2 = float(gt.max()) ** 2
    R = cfg["R"]

    def vpsnr(tr):
        vol, _, _ = tr.UniformSampledVolume((vol_n, vol_n, vol_n))
        mse = float(((vol[0].double() - gt) ** 2).mean())
        return 10.0 * np.log10(peak2 / mse)

    res = {}
    target = [None]

    def run(name, dec, prop, M):
        tr = make_trainer(dict(cfg, M=M), tree, cam, dev, dec, prop, cfg["seed"])
        gen = torch.Generator(device=dev)
        gen.manual_seed(777)
        ms, curve, k, samples = 0.0, [], 0, 0.0
        while k < steps:
            n = min(every, steps - k)
            bs = [scene.sample_batch(R, gen) for _ in range(n)]
            t, _, cnt = time_steps(tr, bs, phase_events=False)
            k += n
            ms += t
            samples += float(cnt[:, 1].double().sum())
            p = vpsnr(tr)
            curve.append([k, round(ms, 1), round(p, 3)])
            if target[0] is not None and p >= target[0] - 0.1:
                break
        res[name] = {"steps": k, "train_ms": ms, "ms_per_step": ms / k, "samples_per_step": samples / k,
                     "samples_per_segment_budget": M if not prop else cfg.get("proposal_budget", 12),
                     "volume_psnr_db": curve[-1][2], "curve": curve}
        if target[0] is None:
            target[0] = curve[-1][2]
        del tr
        torch.cuda.empty_cache()

    run("plain_fp32", "bf16x3", False, cfg["M"])
    run("bf16_proposal12", "bf16", True, cfg["M"])
    run("bf16_uniform12", "bf16", False, 12)
    # the uniform budget with the proposal run's samples per step: one step's
    # sample count per candidate budget (the counts depend on the rays only)
    gen = torch.Generator(device=dev)
    gen.manual_seed(777)
    b = scene.sample_batch(R, gen)
    best = None
    for M in range(1, 13):
        tr = make_trainer(dict(cfg, M=M), tree, cam, dev, "bf16", False, cfg["seed"])
        tr.step(*b)
        n = float(tr.counters[1].item())
        del tr
        if best is None or abs(n - res["bf16_proposal12"]["samples_per_step"]) < best[1]:
            best = (M, abs(n - res["bf16_proposal12"]["samples_per_step"]))
    torch.cuda.empty_cache()
    run("bf16_uniform_matched", "bf16", False, best[0])
    tgt = target[0]
    for name in ("plain_fp32", "bf16_proposal12", "bf16_uniform12", "bf16_uniform_matched"):
        hit = [c for c in res[name]["curve"] if c[2] >= tgt - 0.1]
        res[name]["ms_to_target"] = hit[0][1] if hit else None
        res[name]["steps_to_target"] = hit[0][0] if hit else None
    a, b = res["plain_fp32"]["ms_to_target"], res["bf16_proposal12"]["ms_to_target"]
    res["target_db"] = tgt - 0.1
    res["plain_final_db"] = tgt
    res["speedup_to_target"] = (a / b) if (a and b) else None
    for name in ("bf16_uniform12", "bf16_uniform_matched"):
        u = res[name]["ms_to_target"]
        res["proposal_vs_" + name[5:] + "_to_target"] = (u / b) if (u and b) else None
    res["definition"] = ("target = plain method's final volume PSNR - 0.1 dB; volume PSNR = 10 log10(peak^2 / MSE), "
                         "%d^3 voxel-corner lattice vs the phantom density, f64; time = CUDA events around the "
                         "training steps; proposal_vs_X = X's time to the target / the proposal's" % vol_n)
    return res


def reference_gpu_igs(cfg, scene, tree, cam, dev, reps=5):
    """The reference's own GPU grid sampler (IndirectGridSample3DForward/
    BackwardCUDAKernel, src/modules/IndirectGridSample3D.cu:432-801, compiled
    unmodified for sm_100a into oracle/_ref by `make -C oracle ref-cuda`)
    against this library's standalone neat_igs_forward/backward, on the same
    inputs: the SampleList of one batch of the workload (CreateSamplesForRays,
    ray-major as the reference produces it; the local coordinates and grid
    rows of ComputeLocalSamples), a random [A, C, G, G, G] grid and output
    gradient.  Median CUDA-event time of `reps` launches per kernel on the
    legacy default stream the reference launches on; the backward's zeroed
    gradients are reset outside the timed region.  Also the forward on the
    node-sorted sample order the fused step uses."""
    import ctypes
    path = os.path.join(ROOT, "oracle", "_ref", "libneat_ref_cuda.so")
    if not os.path.exists(path):
        return {"unavailable": "oracle/_ref/libneat_ref_cuda.so is not built (make -C oracle ref-cuda)"}
    from neat_b200 import _lib
    from neat_b200.api import ComputeLocalSamples, CreateSamplesForRays, GetRays
    ref = ctypes.CDLL(path)
    P, L, I = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
    ref.ref_igs_forward_cuda.argtypes = [P, L, I, I, I, I, P, P, L, P]
    ref.ref_igs_backward_cuda.argtypes = [P, L, I, I, I, I, P, P, L, P, P, P]
    lib = _lib.load()
    gen = torch.Generator(device=dev)
    gen.manual_seed(31)
    uv, img, _ = scene.sample_batch(cfg["R"], gen)
    s = CreateSamplesForRays(tree, GetRays(cam, uv, img), cfg["M"], True, seed=1, step=1)
    local = ComputeLocalSamples(tree, s.global_coordinate, s.node_id).contiguous()
    index = tree.GlobalNodeIdToLocalActiveId(s.node_id).contiguous()
    A, C, G = tree.NumActiveNodes(), cfg["C"], cfg["G"]
    S = int(index.numel())
    g = torch.Generator(device=dev)
    g.manual_seed(32)
    grid = torch.rand((A, C, G, G, G), generator=g, device=dev) * 2 - 1
    go = torch.randn((S, C), generator=g, device=dev)
    out_r = torch.empty((S, C), device=dev)
    out_n = torch.empty((S, C), device=dev)
    gg = torch.zeros_like(grid)
    gu = torch.zeros((S, 3), device=dev)
    st = torch.cuda.current_stream(dev).cuda_stream

    def timed(fn, reset=None):
        fn()  # warm-up
        ts = []
        for _ in range(reps):
            if reset is not None:
                reset()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            rc = fn()
            e1.record()
            torch.cuda.synchronize()
            if rc:
                raise RuntimeError(f"IGS launch failed ({rc})")
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    def reset():
        gg.zero_()
        gu.zero_()

    def fwd_ref(ix=index, lc=local, out=out_r):
        return ref.ref_igs_forward_cuda(grid.data_ptr(), A, C, G, G, G, ix.data_ptr(), lc.data_ptr(), S,
                                        out.data_ptr())

    def fwd_neat(ix=index, lc=local, out=out_n):
        return lib.neat_igs_forward(grid.data_ptr(), A, C, G, G, G, ix.data_ptr(), lc.data_ptr(), S, out.data_ptr(), st)

    def bwd_ref():
        return ref.ref_igs_backward_cuda(grid.data_ptr(), A, C, G, G, G, index.data_ptr(), local.data_ptr(), S,
                                         go.data_ptr(), gg.data_ptr(), gu.data_ptr())

    def bwd_neat():
        return lib.neat_igs_backward(grid.data_ptr(), A, C, G, G, G, index.data_ptr(), local.data_ptr(), S,
                                     go.data_ptr(), gg.data_ptr(), gu.data_ptr(), st)

    res = {"samples": S, "C": C, "G": G, "grid_rows": A,
           "ref_forward_ms": timed(fwd_ref), "neat_forward_ms": timed(fwd_neat)}
    res["forward_max_abs_diff"] = float((out_r - out_n).abs().max())
    res["ref_backward_ms"] = timed(bwd_ref, reset)
    res["neat_backward_ms"] = timed(bwd_neat, reset)
    order = torch.sort(index, stable=True).indices
    ix_s, lc_s = index[order].contiguous(), local[order].contiguous()
    res["ref_forward_node_sorted_ms"] = timed(lambda: fwd_ref(ix_s, lc_s))
    res["neat_forward_node_sorted_ms"] = timed(lambda: fwd_neat(ix_s, lc_s))
    res["note"] = ("reference kernels built unmodified for sm_100a (nvcc defaults, FMA contraction on); "
                   "forward_max_abs_diff is that contraction's rounding.  The fused step does not call these: its "
                   "gather and scatter run inside the tile kernels on a channel-last grid (phase_ms)")
    del grid, go, out_r, out_n, gg, gu
    torch.cuda.empty_cache()
    return res


def large_workload(dev, steps=50, warmup=3):
    """The large porous configuration, BF16 + learned proposal: rays/s over one
    full 50-step proposal cycle (its uniform 32-sample TRAIN step included)
    after 20 cycles that train the proposal and its count head, device-resident
    batches, CUDA events; per-phase times and samples per step."""
    cfg = dict(WORKLOADS["large"])
    scene, tree, cam = build_workload(cfg, dev)
    tr = make_trainer(cfg, tree, cam, dev, "bf16", True, cfg["seed"])
    R = cfg["R"]
    gen = torch.Generator(device=dev)
    gen.manual_seed(99)
    batches = [scene.sample_batch(R, gen) for _ in range(warmup + steps)]
    for i in range(warmup):  # the warm-up includes the first TRAIN step; the timed cycle has its own
        tr.step(*batches[i])
    while tr.step_id < 50 * PROPOSAL_WARM_CYCLES or (tr.step_id % 50) != 0:  # the timed region starts at a boundary
        tr.step(*batches[tr.step_id % len(batches)])
    ms, phase_ms, counts = time_steps(tr, batches[warmup:])
    S = counts[:, 1].double()
    out = {"workload": cfg["desc"], "rays_per_s": R * steps / (ms / 1000.0), "ms_per_step": ms / steps,
           "steps": steps, "timed": "one 50-step proposal cycle: 1 uniform TRAIN step (32 samples per segment) + "
                                    "49 SAMPLE steps (at most 12 per segment: the count head's counts)",
           "samples_per_step_mean": float(S.mean()), "samples_train_step": float(S.max()),
           "samples_sample_step": float(S.min()), "active_nodes": tree.NumActiveNodes(),
           "node_depths": {int(k): int(v) for k, v in zip(*np.unique(tree.node_depth[tree.active_node_ids],
                                                                    return_counts=True))},
           "grid_params": int(tr.grid.numel()), "phase_ms": phase_ms}
    del tr
    torch.cuda.empty_cache()
    return out


# --------------------------------------------------------------------------
# main
# --------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="neat", choices=["neat", "reference"])
    ap.add_argument("--workload", default="full", choices=list(WORKLOADS))
    ap.add_argument("--proposal", action="store_true",
                    help="main line with the learned proposal (BF16 decoder unless --decoder; on by itself for "
                         "the large workload), timed from a cycle boundary after %d proposal cycles"
                         % PROPOSAL_WARM_CYCLES)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-psnr", action="store_true", help="skip the small workload's time-to-PSNR leg")
    ap.add_argument("--no-variants", action="store_true", help="skip the FP32 / BF16 / BF16+proposal step variants")
    ap.add_argument("--no-large", action="store_true", help="skip the large porous workload's sub-line")
    ap.add_argument("--no-prefetch", action="store_true",
                    help="build every step's segment lists inside the step (no look-ahead under Adam)")
    ap.add_argument("--no-ref-igs", action="store_true",
                    help="skip timing the reference's GPU IGS kernels beside this library's")
    ap.add_argument("--volume-psnr", type=int, default=5000,
                    help="race plain vs BF16+proposal to the plain method's volume PSNR over this many steps "
                         "(full workload; 0 skips)")
    ap.add_argument("--rays", type=int, default=0, help="override rays per batch (profiling runs only)")
    ap.add_argument("--decoder", default=None, choices=list(PATH_NAMES),
                    help="decoder GEMM path: FP32 SIMT, tcgen05 FP32-accurate 3-piece BF16 split, tcgen05 BF16 "
                         "(default: bf16x3; bf16 for the large workload)")
    args = ap.parse_args()
    global PREFETCH
    PREFETCH = not args.no_prefetch
    if args.warmup < 3:
        args.warmup = 3
    cfg = dict(WORKLOADS[args.workload])
    if args.rays:
        cfg["R"] = args.rays
    large = args.workload == "large"
    proposal = large or args.proposal
    decoder = args.decoder or ("bf16" if proposal else "bf16x3")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        # the reference arm: rank 0 alone runs the CPU path
        if rank != 0:
            return
        v, info = cpu_reference_rays_per_s(cfg, args.steps, args.warmup, budget_s=120.0)
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "rays/s", "n_gpus": args.gpus,
                "steps": info["steps"], "warmup": args.warmup, "ms_per_step": 1000.0 * info["seconds"] / info["steps"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": {"workload": cfg["desc"], "rays_per_step": info["rays"]},
                "cpu_baseline": {"value": v, "unit": "rays/s", "cores": info["cores"], "kind": info["kind"],
                                 "sample": f"{info['rays']} rays/step of the same workload, {info['steps']} steps; "
                                           + CPU_PATH_DESC},
                "e2e": {"value": v, "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device (the neat arm has no CPU fallback)")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    from neat_b200 import _lib
    from neat_b200.csrc import build
    build.build()
    scene, tree, cam = build_workload(cfg, dev)
    n_active = tree.NumActiveNodes()
    R, K, W = cfg["R"], args.steps, args.warmup
    tr = make_trainer(cfg, tree, cam, dev, decoder, proposal, cfg["seed"] + rank)
    gen = torch.Generator(device=dev)
    gen.manual_seed(1000 + rank)
    batches = [scene.sample_batch(R, gen) for _ in range(W + K)]

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- warm-up (device-resident batches; with the proposal it includes the first TRAIN step).
    # It exercises the look-ahead between warm-up batches (the process's first
    # side-stream build carries a one-time start-up cost); the last warm-up step
    # does not build the first timed batch's lists, which stay inside the timed region.
    for i in range(W):
        tr.step(*batches[i], next=batches[i + 1] if PREFETCH and i + 1 < W else None)
    # with the proposal: train it and its count head to their steady state, and
    # start the timed region at a cycle boundary (a uniform TRAIN step first)
    while proposal and (tr.step_id < 50 * PROPOSAL_WARM_CYCLES or tr.step_id % 50 != 0):
        tr.step(*batches[tr.step_id % W])
    torch.cuda.synchronize()
    tr.check_status()

    # ---- timed: device-resident inputs (value)
    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    clocks.begin()
    ms, phase_ms, counts = time_steps(tr, batches[W:])
    clocks.end()
    clock_info = clocks.stop()
    barrier()
    ms = max_over_ranks(ms)
    value = R * K * world / (ms / 1000.0)
    S_steps = counts[:, 1].double()
    S = float(S_steps.mean())
    counters = counts[-1].tolist()

    # ---- timed: end to end through the public API with host buffers (e2e)
    # (FusedTrainer.step stages pinned host batches through its copy stream,
    # double-buffered: the copy of step i + 1 overlaps step i; every copy and
    # every step lies between e0 and e1)
    hb = []
    for i in range(K + 1):
        uv, img, tgt = scene.sample_batch(R, gen)
        hb.append((uv.cpu().pin_memory(), img.cpu().pin_memory(), tgt.cpu().pin_memory()))
    loss_host = torch.empty(K, dtype=torch.float32).pin_memory()
    tr.step(*hb[K])  # untimed: creates the staging buffers and the copy stream
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    tr.host_copy_stream().wait_event(e0)
    for i in range(K):
        loss = tr.step(*hb[i], next=hb[i + 1] if PREFETCH and i + 1 < K else None)
        loss_host[i:i + 1].copy_(loss, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    tr.check_status()
    e2e = R * K * world / (e2e_ms / 1000.0)
    h2d = R * (8 + 4 + 4)
    grid_numel = tr.grid.numel()
    del tr
    torch.cuda.empty_cache()

    # ---- roofline of the dominant kernel (backward tiles)
    H = 64
    flops_bwd = 4.0 * hidden_flops(cfg["C"], H) * S  # dX + dW products of the decoder backward
    t_bwd = phase_ms["backward_tiles"] / 1000.0
    peaks, peak_kind = measured_peaks()
    achieved = flops_bwd / t_bwd / 1e12
    peak = peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops"))
    sm_mhz = clock_info.get("sm_mhz") or 1965.0
    simt_peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12

    # single-GPU characterisation legs (N = 1 only, like the CPU baseline): the
    # step variants, the races, the large workload and the reference kernels
    single = world == 1
    ttp = None
    if not args.no_psnr and single:
        ttp = time_to_psnr(dev, ["simt", "bf16x3", "bf16"])
    variants = None
    if not args.no_variants and not large and single:
        variants = step_variants(cfg, scene, tree, cam, dev, value / world)
    vrace = None
    if args.volume_psnr and not large and single:
        vrace = volume_psnr_race(cfg, scene, tree, cam, dev, args.volume_psnr)
    ref_igs = None
    if not args.no_ref_igs and not large and single:
        ref_igs = reference_gpu_igs(cfg, scene, tree, cam, dev)
    large_line = None
    if not args.no_large and not large and single:
        del scene, tree, cam, batches
        torch.cuda.empty_cache()
        large_line = large_workload(dev)
    cpu_base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cv, ci = cpu_reference_rays_per_s(cfg, 5, 1, budget_s=30.0, min_s=12.0)
        cpu_base = {"value": cv, "unit": "rays/s", "cores": ci["cores"], "kind": ci["kind"],
                    "sample": f"{ci['rays']} rays/step of the same workload x {ci['steps']} steps "
                              f"({ci['seconds']:.1f} s); " + CPU_PATH_DESC}
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return
    launches = sum(step_launches(decoder, cfg["C"], proposal, proposal and i % 50 == 0) for i in range(K))
    traffic_key = (args.workload, decoder)
    line = {
        "metric": METRIC, "value": value, "unit": "rays/s", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16" if decoder == "bf16" else "f32",
        "data": "synthetic",
        "config": {"workload": cfg["desc"], "decoder": DECODER_DESC[decoder],
                   "proposal": ("learned, budget %d samples per segment, the count head's counts (count_eps %g), "
                                "uniform share %g, 50-step cycle, timed after %d cycles from a cycle boundary; %d of "
                                "the timed steps are uniform TRAIN steps"
                                % (cfg.get("proposal_budget", 12), cfg.get("count_eps", COUNT_EPS),
                                   cfg.get("proposal_mix", PROPOSAL_MIX), PROPOSAL_WARM_CYCLES,
                                   sum(i % 50 == 0 for i in range(K))))
                   if proposal else None,
                   "rays_per_step": R, "samples_per_step": S, "segments_per_step": counters[0],
                   "active_nodes": n_active, "parallelism": f"replicas x{world}",
                   "l2": "working set > L2: grid + Adam state %.2f GB per replica" % (4 * 4 * grid_numel / 1e9)},
        "phase_ms": phase_ms,
        "roofline": {"kernel": KERNEL_NAME[decoder] % cfg["C"], "bound": "tensor", "achieved": achieved,
                     "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": (TRAFFIC_BYTES_PER_SAMPLE[traffic_key][0] * S
                                 if traffic_key in TRAFFIC_BYTES_PER_SAMPLE else None),
                     "traffic_source": (TRAFFIC_BYTES_PER_SAMPLE[traffic_key][1]
                                        if traffic_key in TRAFFIC_BYTES_PER_SAMPLE else None),
                     "peak_source": f"bf16_tflops_sustained ({peak_kind})",
                     "fp32_simt_peak_tflops": simt_peak,
                     "frac_of_fp32_simt": achieved / simt_peak},
        "step_roofline": step_roofline(S, R, grid_numel, cfg["C"], ms / K, peaks, simt_peak),
        "e2e": {"value": e2e, "unit": "rays/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 4,
                "path": "FusedTrainer.step on pinned host batches: copied in on the trainer's copy stream into "
                        "two alternating device buffer sets (the copy of step i + 1 overlaps step i), each step's "
                        "loss copied back to pinned host memory; all copies and steps inside the timed region"},
        "gpu_launches": launches,
        "clocks": clock_info,
        "cpu_baseline": cpu_base,
        "time_to_psnr": ttp,
        "variants": variants,
        "volume_psnr_race": vrace,
        "large_workload": large_line,
        "reference_gpu_igs": ref_igs,
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
