"""MAP E-step throughput benchmark (particles/s) on B200.

Workload: BASELINE config 2, "MAP2D at scale": 20,000 synthetic particles of
128 x 128 from K = 50 random-blob class templates, 72 in-plane angles (5 deg)
x 29 translations (+-6 px, step 2), CTF per particle, white noise at SNR
0.03, current_size = ori_size = 128 (8,320 Fourier coefficients per image).
A step is one E-step pass (expectationSomeParticles: diff2, posterior,
significance, weighted sums, backprojection) over all particles, in pools
of --pool particles.

Arms:
  default            this library (librome_b200, CUDA, sm_100a)
  --impl reference   the reference's CPU implementation on the host cores
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "E-step particles/s: learned-proposal+BF16 vs plain FP32 GPU at >=99% pose agree"
UNIT = "particles/s"



def tuned_shapes():
    """The tensor-core autotuner's choices: kind/planes N x Kp (128-row tiles) -> tile, with candidate times."""
    from rome_b200 import abi
    out = {}
    for r in abi.tuning_report():
        key = f"{r['kind']}/{r['planes']}p N={r['N']} Kp={r['Kp']} mtiles={r['mtiles']}"
        out[key] = {"choice": r["choice"], "ms": {k: float(v[:-2]) for k, v in r.items() if v.endswith("ms")}}
    return out

def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="map2d_cfg2")
    ap.add_argument("--precision", default="bf16", choices=["fp32", "bf16", "bf16x3"])
    ap.add_argument("--pool", type=int, default=2000)
    ap.add_argument("--particles", type=int, default=0, help="override the particle count (debug)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mode", default="learned", choices=["learned", "exhaustive", "prep", "reconstruct"],
                    help="prep: the image preparation (setFourierTransforms) alone, from float32 images")
    ap.add_argument("--topk", type=int, default=16, help="network outputs proposed per particle (x2 orientations)")
    ap.add_argument("--train-particles", type=int, default=20000)
    ap.add_argument("--train-epochs", type=int, default=15)
    ap.add_argument("--workers", type=int, default=2,
                    help="host threads, each with its own context, working on alternate pools (learned mode)")
    ap.add_argument("--snr-scale", type=float, default=1.0,
                    help="3D workloads: multiply the configured signal-to-noise ratios (calibration runs)")
    ap.add_argument("--min-mass", type=float, default=0.995,
                    help="particles whose top-k proposals hold less network probability are searched exhaustively")
    ap.add_argument("--proposals3d", default="none", choices=["none", "lowres"],
                    help="3D workloads: lowres restricts each particle's coarse pass to the --topk orientations "
                         "of a low-resolution exhaustive coarse pass at --lowres-size (fallback below --min-mass)")
    ap.add_argument("--lowres-size", type=int, default=12, help="coarse size of the low-resolution pass")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.device}", f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                vals = [v.strip() for v in out.stdout.strip().split(",")]
                if len(vals) == 6:
                    self.samples.append(vals)
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[2 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons}


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


def train_proposals(args, ctx, prep_ctx, w, rank):
    """The proposal network of this rank, trained before the timed region on
    its own training particles (same class templates, other noise, poses and
    CTFs: the particles of an earlier EM iteration stand in for them) against
    the exhaustive E-step's posterior (class, psi) marginals."""
    import dataclasses

    import torch
    from rome_b200.proposal import ProposalNet, posterior_targets
    from rome_b200.particles import prepared_pool
    from rome_b200.workload import build_map2d, image_template, prep_options, raw_particles, slice_particles, subset
    wt = dataclasses.replace(w, n_particles=args.train_particles, particle_seed=w.seed + 5000 + 1000 * rank)
    tp, _, _, ttruth = build_map2d(wt)
    K, npsi, cur = tp.nr_classes, tp.nr_psi, tp.current_size
    net = ProposalNet(ctx, K, npsi // 2, 16, (16, 16), 2.0, min(24.0, cur / 2 - 2), seed=3)
    raw = raw_particles(tp, ttruth)
    tmpl = image_template(tp)
    del tp
    t0 = time.perf_counter()
    # the training particles as read (raw images), prepared on the device like the E-step's
    d_raw = torch.from_numpy(raw.images).to(f"cuda:{ctx.device}")
    dr = dataclasses.replace(raw, images=d_raw)
    staged = [prepared_pool(prep_ctx, subset(tmpl, lo, min(tmpl.nr_images, lo + args.pool)),
                            slice_particles(dr, lo, min(tmpl.nr_images, lo + args.pool)), prep_options(w))
              for lo in range(0, tmpl.nr_images, args.pool)]
    del d_raw, dr
    t_stage = time.perf_counter() - t0
    t0 = time.perf_counter()
    xs, ts = [], []
    for q in staged:
        r = ctx.map2d_estep_pool(q, marginals=True)
        ts.append(posterior_targets(r["post_class_psi"], K, npsi))
        xs.append(net.features(q))
    torch.cuda.synchronize()
    t_label = time.perf_counter() - t0
    del staged
    t0 = time.perf_counter()
    losses = net.train(np.concatenate(xs), np.concatenate(ts), epochs=args.train_epochs, batch=256, lr=3e-3)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    info = {"train_particles": int(tmpl.nr_images), "epochs": args.train_epochs, "stage_s": round(t_stage, 2),
            "label_s": round(t_label, 2),
            "train_s": round(t_train, 2), "loss_first": round(float(losses[0]), 4),
            "loss_last": round(float(losses[-1]), 4), "params": int(net.nparam),
            "net": "polar |F| and |CTF| input 16 radii x %d angles, 2 circular 3x3 convs (16, 16), "
                   "circular-correlation head" % (npsi // 2)}
    return net, info


def merge_timings(ts):
    """Phase timings of several contexts added up (device ms, launches, work)."""
    out = {}
    for t in ts:
        for k, v in t.items():
            if isinstance(v, dict):
                d = out.setdefault(k, {"ms": 0.0, "launches": 0, "flops": 0.0, "bytes": 0.0})
                for f in d:
                    d[f] += v[f]
            else:
                out[k] = out.get(k, 0) + v
    return out


def _same_pose(a, b):
    return (a["cls"] == b["cls"]) & (a["psi"] == b["psi"]) & (a["xoff"] == b["xoff"]) & (a["yoff"] == b["yoff"])


def _timed(torch, fn, steps):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    out = None
    for _ in range(steps):
        out = fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), out


def run_ours(args):
    import dataclasses

    import torch
    import torch.distributed as dist

    from rome_b200.distributed import MODEL_SUM_KEYS, allreduce_backprojectors, allreduce_model_sums
    from rome_b200.map2d import GpuContext
    from rome_b200.particles import h2d_bytes as prep_h2d_bytes
    from rome_b200.particles import pin_particles, prepared_pool, prepared_stream
    from rome_b200.proposal import learned_estep_pools
    from rome_b200.workload import (CONFIGS, build_map2d, image_template, prep_options, raw_particles,
                                    slice_particles, subset)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    w = CONFIGS[args.config]
    if args.particles:
        w = dataclasses.replace(w, n_particles=args.particles)
    # every rank processes its own particles (weak scaling, no data-path collective)
    w = dataclasses.replace(w, particle_seed=w.seed + 1 + 1000 * rank)
    pool, proj, r_max, truth = build_map2d(w)
    # the particles as read (float32 images + metadata); everything below starts from them
    raw = raw_particles(pool, truth)
    pool = image_template(pool)
    opts = prep_options(w)
    N = pool.nr_images
    learned = args.mode == "learned"
    ctx = GpuContext(local, args.precision, profile=True)
    ctx.set_projectors(proj, pool.ori_size, r_max)
    prep_ctx = GpuContext(local, "fp32", profile=True)  # image preparation (setFourierTransforms)
    net, train_info = train_proposals(args, ctx, prep_ctx, w, rank) if learned else (None, None)
    # further contexts + networks (same model, same weights), one host thread each
    workers = []
    if learned:
        from rome_b200.proposal import ProposalNet
        for _ in range(max(0, args.workers - 1)):
            c = GpuContext(local, args.precision, profile=True)
            c.set_projectors(proj, pool.ori_size, r_max)
            n2 = ProposalNet(c, net.n_classes, net.n_theta, net.n_r, net.channels, net.r_lo, net.r_hi)
            n2.set_params(net.get_params())
            workers.append((c, n2))
    lane_ctxs = [ctx] + [c for c, _ in workers]
    bounds = [(lo, min(N, lo + args.pool)) for lo in range(0, N, args.pool)]
    tmpls = [subset(pool, lo, hi) for lo, hi in bounds]
    # value: pools prepared once from images resident in HBM, then E-steps over the prepared pools
    d_raw = torch.from_numpy(raw.images).to(f"cuda:{local}")
    dr = dataclasses.replace(raw, images=d_raw)

    def prepare_all():
        return [prepared_pool(prep_ctx, t, slice_particles(dr, lo, hi), opts) for t, (lo, hi) in zip(tmpls, bounds)]

    dev = prepare_all()
    prepare_all()
    prep_ms, _ = _timed(torch, prepare_all, 1)
    del d_raw, dr
    # e2e: page-locked host images, copied in and prepared while earlier pools compute
    host_raw = [pin_particles(slice_particles(raw, lo, hi)) for lo, hi in bounds]
    items = list(zip(tmpls, host_raw))

    exchange_bytes = [0]

    def exchange(res):
        """The iteration's one exchange step over ranks (MLModel::reduceData and
        MAPModel::reduceData): the pools' weighted sums and every class's
        back-projector summed over all ranks, the latter device-resident (NCCL)."""
        if world == 1:
            return
        sums = {}
        for r in res:
            o = r[0] if isinstance(r, tuple) else r
            for k in MODEL_SUM_KEYS:
                if k in o:
                    sums[k] = sums.get(k, 0) + np.asarray(o[k], np.float64)
        red = allreduce_model_sums(sums, device=f"cuda:{local}")
        exchange_bytes[0] = allreduce_backprojectors(ctx) + sum(int(np.asarray(v).nbytes) for v in red.values())

    def step_dev():
        # one EM iteration: the model's projections are computed once per step, not carried over
        for c in lane_ctxs:
            c.invalidate_projections()
        if learned:
            res = learned_estep_pools(ctx, net, dev, args.topk, args.min_mass, workers=workers)
        else:
            res = [(ctx.map2d_estep_pool(q), None, None, None) for q in dev]
        exchange(res)
        return res

    def step_e2e():
        # host (pinned) raw images copied in and prepared on the device (pool k + 1 while pool k computes),
        # E-step, results copied out
        for c in lane_ctxs:
            c.invalidate_projections()
        stream = prepared_stream(prep_ctx, items, opts)
        if learned:
            res = learned_estep_pools(ctx, net, stream, args.topk, args.min_mass, workers=workers)
        else:
            res = [ctx.map2d_estep_pool(q) for q in stream]
        exchange(res)
        return res

    for _ in range(args.warmup):
        step_dev()
    if world > 1:
        dist.barrier()
    for c in lane_ctxs:
        c.reset_timings()
    with ClockSampler(local) as clk:
        torch.cuda.nvtx.range_push("bench_timed")  # lets an ncu launch list select the timed region
        ms, last = _timed(torch, step_dev, args.steps)
        torch.cuda.nvtx.range_pop()
    timings = merge_timings([c.get_timings() for c in lane_ctxs])
    # the network alone (features, forward, top-k, expansion) over the same pools
    prop_ms = _timed(torch, lambda: [net.propose(q, args.topk) for q in dev], 1)[0] if learned else 0.0
    step_e2e()  # warm-up: the staging buffers' first allocation
    if world > 1:
        dist.barrier()
    e_ms, _ = _timed(torch, step_e2e, max(1, args.steps))
    ms_t = torch.tensor([ms, e_ms], device="cuda")
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms, e_ms = ms_t.tolist()
    ms_step = ms / args.steps
    value = N * world / (ms_step / 1e3)
    e2e_value = N * world / (e_ms / max(1, args.steps) / 1e3)

    # ---- comparison arms and judges (outside the timed regions) ----
    def exhaustive_all(c):
        return [c.map2d_estep_pool(q) for q in dev]

    ex_ms, ex_res = _timed(torch, lambda: exhaustive_all(ctx), 1)
    judge = {}
    fp32_line = None
    if args.precision != "fp32" or learned:
        with GpuContext(local, "fp32") as c32:
            c32.set_projectors(proj, pool.ori_size, r_max)
            c32.map2d_estep_pool(dev[0])
            f_ms, f_res = _timed(torch, lambda: exhaustive_all(c32), 1)
        fp32_line = {"value": round(N / (f_ms / 1e3), 2), "unit": UNIT, "particles": N,
                     "search": "exhaustive", "precision": "fp32"}
    else:
        f_ms, f_res = ex_ms, ex_res
    cat = lambda rs, k: np.concatenate([r[k] for r in rs])  # noqa: E731
    keys = ("cls", "psi", "xoff", "yoff")
    ref = {k: cat(f_res, k) for k in keys}
    mine = {k: cat([r[0] for r in last], k) for k in keys}
    exb = {k: cat(ex_res, k) for k in keys}
    judge["pose_agreement_vs_plain_fp32"] = round(float(np.mean(_same_pose(mine, ref))), 5)
    judge["exhaustive_%s_pose_agreement_vs_plain_fp32" % args.precision] = round(
        float(np.mean(_same_pose(exb, ref))), 5)
    judge["class_agreement_vs_truth"] = round(float(np.mean(mine["cls"] - 1 == truth["cls"])), 4)
    if learned:
        props = np.concatenate([r[1] for r in last])
        mass = np.concatenate([r[2] for r in last])
        nlow = sum(len(r[3]) for r in last)
        # reported psi: the table angle folded into (-180, 180]
        tab = np.asarray(pool.over_psi[-1])[:, 0]
        ipsi = {(float(v) - 360.0 if v > 180 else float(v)): k for k, v in enumerate(tab)}
        jbest = (ref["cls"] - 1) * pool.nr_psi + np.array([ipsi[float(v)] for v in ref["psi"]])
        covered = (props == jbest[:, None]).any(axis=1)
        judge["proposal_coverage_of_fp32_mode"] = round(float(np.mean(covered)), 5)
        judge["mean_proposal_mass"] = round(float(mass.mean()), 4)
        nsig = np.concatenate([r[0]["nr_sign"] for r in last])
        judge["significant_hypotheses_per_particle"] = {"mean": round(float(nsig.mean()), 2),
                                                        "p90": float(np.percentile(nsig, 90))}
        judge["orientations_searched"] = f"{props.shape[1]} of {pool.nr_classes * pool.nr_psi}"
        judge["exhaustive_fallback_fraction"] = round(nlow / N, 5)
        # what other fallback thresholds would give: (fraction searched exhaustively, pose agreement)
        agree_l, agree_x = _same_pose(mine, ref), _same_pose(exb, ref)
        judge["fallback_sweep"] = {
            str(tau): [round(float(np.mean(mass < tau)), 4),
                       round(float(np.mean(np.where(mass < tau, agree_x, agree_l))), 5)]
            for tau in (0.99, 0.995, 0.999, 0.9995, 0.9999)} if nlow == 0 else "run with --min-mass 0"
    hbm, bf16, peak_kind = load_peaks()
    phases = {k: round(v["ms"] / args.steps, 3) for k, v in timings.items() if isinstance(v, dict)}
    if learned:
        phases["propose"] = round(prop_ms, 3)
    # dominant kernel: the restricted contraction (learned mode) or the cross-term GEMM (exhaustive mode),
    # algorithmic flops 4 * active pixels per (particle, hypothesis), timed by the phase's CUDA events
    gem = timings["restricted" if learned else "cross_gemm"]
    per_launch_ms = gem["ms"] / max(gem["launches"], 1)
    flops_per_launch = gem["flops"] / max(gem["launches"], 1)
    achieved = flops_per_launch / (per_launch_ms / 1e3) / 1e12 if gem["ms"] > 0 else 0.0
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_step, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": {"fp32": "f32", "bf16": "bf16", "bf16x3": "bf16x3"}[args.precision],
        "data": "synthetic (seeded random-blob templates, CTF, white noise)",
        "config": {"workload": args.config, "particles_per_gpu": N, "image": w.ori_size, "classes": w.n_classes,
                   "psi": int(pool.nr_psi), "translations": int(pool.nr_trans), "pool": args.pool,
                   "precision": args.precision,
                   "search": (f"learned proposals, top-{args.topk} network outputs -> {2 * args.topk} orientations; "
                              f"exhaustive where their probability mass < {args.min_mass}" if learned else "exhaustive"),
                   "inputs": "larger than L2 (no flush)",
                   "host_threads": args.workers if learned else 1,
                   "exchange": ("per step: wsums and every class's back-projector all-reduced over the ranks on "
                                f"the device (NCCL), {exchange_bytes[0]} bytes per rank" if world > 1 else
                                "none (one rank)")},
        "e2e": {"value": round(e2e_value, 2), "unit": UNIT,
                "from": "float32 images + metadata in page-locked host memory: copy, image preparation "
                        "(setFourierTransforms), E-step, results back",
                "h2d_bytes_per_step": int(sum(prep_h2d_bytes(r) + r.nr_images * (3 * 8 + 4)
                                              + (r.nr_images * 8 * args.topk if learned else 0) for r in host_raw)),
                "d2h_bytes_per_step": int(sum(ctx.d2h_bytes(q) + q.nr_images * 3 * 8
                                              + (q.nr_images * (8 * args.topk + 4) if learned else 0)
                                              for q in tmpls))},
        "image_preparation": {"value": round(N * world / (prep_ms / 1e3), 2), "unit": UNIT,
                              "ms_per_step": round(prep_ms, 3),
                              "what": "setFourierTransforms of every pool from float32 images resident in HBM",
                              "options": dataclasses.asdict(opts)},
        "gpu_launches": int(timings["total_launches"]),
        "roofline": None,
        "roofline_contraction": {
            "bound": "tensor", "achieved": round(achieved, 2), "peak": bf16, "unit": "TFLOP/s",
            "frac": round(achieved / bf16, 4), "traffic": kernel_traffic(args, learned, gem),
            "peak_kind": peak_kind, "launches": int(gem["launches"]), "ms_per_launch": round(per_launch_ms, 4),
            "kernel": ("restricted_tc_kernel (tcgen05, w formed in shared memory)" if learned else
                       "tc_gemm_kernel (cross term, diff2 epilogue)")},
        "phases_ms_per_step": phases,
        "judge": judge,
        "exhaustive_%s" % args.precision: {"value": round(N / (ex_ms / 1e3), 2), "unit": UNIT},
        "clocks": clk.summary(),
    }
    # the roofline names the phase with the most device time: the back-projection when it outweighs the
    # contraction (learned mode), with the algorithmic bytes the library counts for it
    bpt = timings["backproject"]
    if bpt["ms"] > gem["ms"] and bpt["bytes"] > 0:
        bp_ms = bpt["ms"] / max(bpt["launches"], 1)
        bp_ach = bpt["bytes"] / (bpt["ms"] / 1e3) / 1e9
        line["roofline"] = {
            "bound": "hbm", "achieved": round(bp_ach, 1), "peak": hbm, "unit": "GB/s", "frac": round(bp_ach / hbm, 4),
            "traffic": None, "peak_kind": peak_kind, "launches": int(bpt["launches"]),
            "ms_per_launch": round(bp_ms, 4),
            "kernel": "back-projection phase (bp_prep_kernel, list sort, bp_list_kernel): algorithmic bytes = 24 B "
                      "per active pixel of every significant hypothesis + 96 B (12 FP64 updates) per active pixel "
                      "of every back-projected slice; bound in practice by L2 FP64 atomics (the class "
                      "back-projectors stay in L2)"}
    else:
        line["roofline"] = line["roofline_contraction"]
    line["autotune"] = tuned_shapes()
    if fp32_line is not None:
        line["plain_fp32"] = fp32_line
    if train_info is not None:
        # the one-time cost of the learned path (staging, labels from the exhaustive E-step, training),
        # spread over EM iterations of this many particles, against the exhaustive BF16 E-step
        once = train_info["stage_s"] + train_info["label_s"] + train_info["train_s"]
        step_s, ex_s = ms_step / 1e3, ex_ms / 1e3
        train_info["one_time_s"] = round(once, 2)
        train_info["amortised"] = {
            f"{n}_iterations": round(n * N * world / (n * step_s + once), 2) for n in (10, 25, 100)}
        train_info["break_even_iterations_vs_exhaustive_%s" % args.precision] = (
            round(once / (ex_s - step_s), 1) if ex_s > step_s else None)
        line["learned"] = train_info
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args, w)
    for c, n2 in workers:
        n2.close()
        c.close()
    prep_ctx.close()
    if net is not None:
        net.close()
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def kernel_traffic(args, learned, gem):
    """DRAM bytes per launch of the reported kernel from its committed ncu
    capture (profiles/*_traffic.json), scaled to this launch size by the
    algorithmic work (rows processed), or None without a capture."""
    name = "restricted_tc_traffic.json" if learned else "cross_gemm_traffic.json"
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    if d.get("workload") != args.config or d.get("precision") != args.precision:
        return None
    flops = gem["flops"] / max(gem["launches"], 1)
    if "flops_per_launch" in d:
        return int(d["dram_bytes_per_launch"] * flops / d["flops_per_launch"])
    return int(d["dram_bytes_per_launch"] * args.pool / d["pool"])


def cross_gemm_traffic(args, pool_particles):
    """DRAM bytes per launch of the cross-term GEMM from the committed ncu
    capture (profiles/cross_gemm_traffic.json), scaled to this pool size by
    the number of rows (particles x translations) the launch processes."""
    path = os.path.join(ROOT, "profiles", "cross_gemm_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    if d.get("workload") != args.config or d.get("precision") != args.precision:
        return None
    return int(d["dram_bytes_per_launch"] * pool_particles / d["pool"])


_W = {}


def _oracle_init(proj, r_max):
    _W["proj"], _W["r_max"] = proj, r_max


def _oracle_worker(pool):
    """One process of the CPU baseline: the oracle E-step on a sub-pool."""
    from oracle import oracle_py
    t = time.perf_counter()
    oracle_py.map2d_estep_pool(pool, _W["proj"], _W["r_max"])
    return time.perf_counter() - t


def oracle_rate(w, target_seconds: float = 15.0, cores: int = 0):
    """Particles/s of the C oracle (FP64, the reference's operation order and
    loop structure) on a bounded sample of the same workload: one particle
    per process, all host cores, sample sized to about `target_seconds`."""
    import dataclasses
    import multiprocessing as mp
    import pickle

    from rome_b200.workload import build_map2d, subset
    cores = cores or os.cpu_count() or 1
    probe = dataclasses.replace(w, n_particles=max(cores, 1), seed=w.seed + 7)
    pool, proj, r_max, _ = build_map2d(probe)
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores, initializer=_oracle_init, initargs=(proj, r_max)) as pp:
        # one particle to size the sample
        t1 = pp.map(_oracle_worker, [subset(pool, 0, 1)])[0]
        rounds = max(1, int(target_seconds / max(t1, 1e-3)))
        n = min(pool.nr_images, cores)
        jobs = [subset(pool, i, i + 1) for i in range(n)] * rounds
        t0 = time.perf_counter()
        pp.map(_oracle_worker, jobs)
        dt = time.perf_counter() - t0
    return {"value": round(len(jobs) / dt, 4), "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{len(jobs)} particles of {w.ori_size}x{w.ori_size}, K={w.n_classes}, "
                      f"{pool.nr_psi} psi x {pool.nr_trans} translations, one particle per process, "
                      f"{dt:.1f} s wall"}


REF_BENCH = os.path.join(ROOT, "oracle", "_ref", "map2d_bench")


# one CPU-baseline sample for both the GPU arm's cpu_baseline and the reference arm: pools of 16 particles,
# the first REF_WARM_POOLS run and not counted
REF_POOL, REF_WARM_POOLS, REF_TIMED_POOLS = 16, 2, 8


def reference_rate(w, pool: int, warm_pools: int, timed_pools: int, tmpdir: str):
    """Particles/s of the reference's own MAP2D E-step (oracle/_ref/map2d_bench:
    the reference sources compiled unchanged, every OpenMP thread of the host)
    on a dataset of the same workload, searched against the templates the
    particles were made from (as the GPU benchmark does) at the full image
    size with every class: expectationSomeParticles() timed per pool, the
    first `warm_pools` pools not counted.  Returns (baseline dict, seconds per
    timed pool)."""
    from rome_b200.synthetic import Map2dSpec, _render_blobs_2d, make_templates_2d, write_dataset_2d
    npools = warm_pools + timed_pools
    spec = Map2dSpec(n_particles=pool * npools, size=w.ori_size, n_classes=w.n_classes, n_blobs=w.n_blobs,
                     blob_sigma=w.blob_sigma, max_shift=w.max_shift, defocus=w.defocus, pixel=w.pixel, snr=w.snr,
                     seed=w.seed + 101)
    star = write_dataset_2d(os.path.join(tmpdir, "data"), spec)
    tmpl = make_templates_2d(np.random.default_rng(spec.seed), spec)  # the generator's own first draws
    raw = os.path.join(tmpdir, "refs.f64")
    np.stack([_render_blobs_2d(spec.size, t["centers"], t["sigmas"], t["amps"]) for t in tmpl]).astype(
        np.float64).tofile(raw)
    cmd = [REF_BENCH, "-i", star, "-K", str(w.n_classes), "-angpix", str(w.pixel), "-psi_step",
           str(int(round(w.psi_step))), "-offset_range", str(w.offset_range), "-offset_step", str(w.offset_step),
           "-oversampling", "0", "-ctf", "1", "-pool", str(pool), "-warm_pools", str(warm_pools),
           "-time_pools", str(timed_pools), "-refs_raw", raw]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=1800, cwd=tmpdir)
    if out.returncode != 0:
        raise RuntimeError(f"map2d_bench exited {out.returncode}: {out.stderr[-300:]}")
    pools, threads, cur = [], 0, 0
    for ln in out.stdout.splitlines():
        kv = dict(x.split("=") for x in ln.split()[1:] if "=" in x)
        if ln.startswith("map2d_bench_pool"):
            pools.append((int(kv["particles"]), float(kv["estep_s"])))
        elif ln.startswith("map2d_bench "):
            threads, cur = int(kv["threads"]), int(kv["current_size"])
    n = sum(p for p, _ in pools)
    t = sum(x for _, x in pools)
    per = sorted(x / p for p, x in pools)
    return {"value": round(n / t, 4), "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"{n} particles ({len(pools)} pools of {pool}) of {w.ori_size}x{w.ori_size}, K={w.n_classes}, "
                      f"{int(round(360 / w.psi_step))} psi x translations +-{w.offset_range} step {w.offset_step}, "
                      f"current_size {cur}, searched against the generating templates; reference "
                      f"expectationSomeParticles() timed with dtime(), {t:.1f} s; {warm_pools} warm-up pools "
                      f"not counted",
            "s_per_particle": {"min": round(per[0], 4), "median": round(per[len(per) // 2], 4),
                               "max": round(per[-1], 4)}}, t / max(len(pools), 1)


REF_BENCH3D = os.path.join(ROOT, "oracle", "_ref", "map3d_bench")
REF_RECON = os.path.join(ROOT, "oracle", "_ref", "recon_bench")


def reference_rate_3d(w, pool: int, warm_pools: int, timed_pools: int, tmpdir: str):
    """Particles/s of the reference's own MAP3D E-step (oracle/_ref/map3d_bench:
    the reference sources compiled unchanged, every OpenMP thread of the host)
    on a dataset of the same workload (128^2 particles projected from K
    random-blob volumes, CTF, white noise at the workload's SNR), searched
    against those K volumes at the full image size with every class: one
    pool after another as expectation() runs them, the first `warm_pools`
    not counted.  Returns (baseline dict, seconds per timed pool)."""
    from rome_b200.synthetic import Map3dSpec, make_volumes_3d, render_volume, write_dataset_3d
    npools = warm_pools + timed_pools
    spec = Map3dSpec(n_particles=pool * npools, size=w.ori_size, n_classes=w.n_classes, n_blobs=w.n_blobs,
                     blob_sigma=w.blob_sigma, max_shift=w.max_shift, defocus=w.defocus, pixel=w.pixel, snr=w.snr,
                     seed=w.seed + 101)
    star, ref = write_dataset_3d(os.path.join(tmpdir, "data"), spec)
    vols = make_volumes_3d(np.random.default_rng(spec.seed), spec)  # the generator's own first draws
    raw = os.path.join(tmpdir, "refs.f64")
    np.stack([render_volume(spec.size, v) for v in vols]).astype(np.float64).tofile(raw)
    cmd = [REF_BENCH3D, "-i", star, "-ref", ref, "-refs_raw", raw, "-K", str(w.n_classes), "-angpix", str(w.pixel),
           "-healpix_order", str(w.healpix_order), "-oversampling", "1", "-offset_range", str(w.offset_range),
           "-offset_step", str(w.offset_step), "-ctf", "1", "-pool", str(pool), "-warm_pools", str(warm_pools),
           "-time_pools", str(timed_pools)]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=1800, cwd=tmpdir)
    if out.returncode != 0:
        raise RuntimeError(f"map3d_bench exited {out.returncode}: {out.stderr[-300:]}")
    pools, threads, cur, coarse = [], 0, 0, 0
    for ln in out.stdout.splitlines():
        kv = dict(x.split("=") for x in ln.split()[1:] if "=" in x)
        if ln.startswith("map3d_bench_pool"):
            pools.append((int(kv["particles"]), float(kv["estep_s"])))
        elif ln.startswith("map3d_bench "):
            threads, cur, coarse = int(kv["threads"]), int(kv["current_size"]), int(kv["coarse_size"])
    n = sum(p for p, _ in pools)
    t = sum(x for _, x in pools)
    per = sorted(x / p for p, x in pools)
    return {"value": round(n / t, 4), "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"{n} particles ({len(pools)} pools of {pool}) of {w.ori_size}x{w.ori_size}, K={w.n_classes}, "
                      f"HEALPix order {w.healpix_order}, oversampling 1, translations +-{w.offset_range} step "
                      f"{w.offset_step}, coarse size {coarse}, current size {cur}, searched against the generating "
                      f"volumes; reference expectationSomeParticles() timed with dtime(), {t:.1f} s; "
                      f"{warm_pools} warm-up pools not counted",
            "s_per_particle": {"min": round(per[0], 4), "median": round(per[len(per) // 2], 4),
                               "max": round(per[-1], 4)}}, t / max(len(pools), 1)


def cpu_baseline(args, w):
    """The reported CPU baseline: the reference itself when oracle/_ref was
    built, else the oracle port."""
    import tempfile
    try:
        rate = reference_rate_3d if args.config.startswith("map3d") else reference_rate
        if os.path.exists(REF_BENCH3D if args.config.startswith("map3d") else REF_BENCH):
            with tempfile.TemporaryDirectory(prefix="rome_refbench_") as tmp:
                return rate(w, pool=REF_POOL, warm_pools=REF_WARM_POOLS, timed_pools=REF_TIMED_POOLS, tmpdir=tmp)[0]
        return oracle_rate(w, target_seconds=15.0)
    except Exception as e:  # the baseline is reported, never required
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"failed: {e}"}


def reference_rate_recon(n: int = 60000):
    """The reference's per-image reconstruction work (rome_reconstruct's
    image loop on transformed spectra: shift, CTF image and products,
    MyBackProjector::backproject into the padded grid) timed by
    oracle/_ref/recon_bench on every host core, one back-projector per
    thread as one per MPI rank."""
    import subprocess
    cores = os.cpu_count() or 1
    env = dict(os.environ, OMP_NUM_THREADS=str(cores))
    r = subprocess.run([REF_RECON, "-n", str(n), "-size", "128", "-angpix", "1.5"], env=env, capture_output=True,
                       text=True, timeout=1800)
    line = [x for x in r.stdout.splitlines() if x.startswith("RECON_BENCH")]
    if r.returncode != 0 or not line:
        raise RuntimeError(f"recon_bench failed ({r.returncode}): {r.stderr[-500:]}")
    v = dict(kv.split("=") for kv in line[-1].split()[1:])
    secs = float(v["seconds"])
    return {"value": round(n / secs, 2), "unit": "particles/s", "cores": int(v["threads"]), "kind": "reference",
            "sample": f"{n} images of 128x128 back-projected at known poses into the pad-2 grid (259^3) by the "
                      f"reference's own shiftImageInFourierTransform, CTF::getFftwImage and "
                      f"MyBackProjector::backproject (rome_reconstruct's image loop without reading and "
                      f"transforming the images), one back-projector per thread as one per MPI rank, "
                      f"{secs:.1f} s",
            "s_per_image_per_thread": {"min": float(v["per_image_min"]), "median": float(v["per_image_median"]),
                                       "max": float(v["per_image_max"])}}


def run_reference(args):
    """The reference arm: the reference's own CPU E-step (oracle/_ref, or the
    oracle port where the reference could not be built) on every host core,
    same workload and metric; rank 0 only, the other ranks exit at once."""
    import tempfile
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if args.mode == "reconstruct":
        if not os.path.exists(REF_RECON):
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/recon_bench was not built (the "
                              "reference tree was absent at build time)"}))
            return
        best = reference_rate_recon()
        print(json.dumps({"metric": "reconstruction at known poses: back-projection particles/s (rome_reconstruct)",
                          "value": best["value"], "unit": UNIT, "n_gpus": int(os.environ.get("WORLD_SIZE", 1)),
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                          "impl": "reference", "config": {"workload": "map3d_cfg3 M-step shapes: reconstruction at "
                                                                      "known poses", "image": 128, "pad": 259},
                          "cpu_baseline": best,
                          "e2e": {"value": best["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return
    from rome_b200.workload import CONFIGS
    w = CONFIGS[args.config]
    is3d = args.config.startswith("map3d")
    if os.path.exists(REF_BENCH3D if is3d else REF_BENCH):
        # the cpu_baseline sample (one pool of 16 particles per step), so that both arms report one number
        with tempfile.TemporaryDirectory(prefix="rome_refbench_") as tmp:
            best, s_per_step = (reference_rate_3d if is3d else reference_rate)(
                w, pool=REF_POOL, warm_pools=REF_WARM_POOLS, timed_pools=REF_TIMED_POOLS, tmpdir=tmp)
    elif is3d:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/map3d_bench was not built (the "
                          "reference tree was absent at build time); the 3D oracle port is not a timing harness"}))
        return
    else:
        best = oracle_rate(w, target_seconds=20.0)
        s_per_step = None
    line = {"value": best["value"], "unit": UNIT, "n_gpus": int(os.environ.get("WORLD_SIZE", 1)),
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(s_per_step * 1e3, 3) if s_per_step else None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "metric": "MAP3D E-step particles/s (exhaustive search)" if is3d else METRIC,
            "config": {"workload": args.config, "image": w.ori_size, "classes": w.n_classes,
                       "step": f"one pool of {REF_POOL} particles ({REF_TIMED_POOLS} timed, {REF_WARM_POOLS} "
                               f"warm-up)"},
            "cpu_baseline": best,
            "e2e": {"value": best["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours_3d(args):
    """The MAP3D E-step (coarse pass over every class x direction x psi x
    translation on the tensor cores, fine pass over the coarse-significant
    points, posterior and significance in FP64, wsums, back-projection) on
    the 3D configuration's synthetic workload, one JSON line.  value: images
    prepared once and resident in HBM; e2e: float32 images and metadata in
    page-locked host memory, copied in (pool k + 1 while pool k computes),
    prepared on the device (setFourierTransforms), E-step, results back."""
    import dataclasses

    import torch

    from rome_b200.map2d import GpuContext
    from rome_b200.map3d import map3d_estep_pools_adaptive
    from rome_b200.particles import h2d_bytes as prep_h2d_bytes
    from rome_b200.particles import pin_particles, prepared_pool, prepared_stream
    from rome_b200.workload import CONFIGS, build_map3d, prep_options, raw_particles, slice_particles, subset3d
    w = CONFIGS[args.config]
    if args.particles:
        w = dataclasses.replace(w, n_particles=args.particles)
    if args.snr_scale != 1.0:
        w = dataclasses.replace(w, snr=w.snr * args.snr_scale, snr_range=None if w.snr_range is None else
                                tuple(v * args.snr_scale for v in w.snr_range))
    t0 = time.perf_counter()
    pool, proj, r_max, truth = build_map3d(w)
    t_build = time.perf_counter() - t0
    N = pool.nr_images
    raw = raw_particles(pool, truth)
    bounds = [(lo, min(N, lo + args.pool)) for lo in range(0, N, args.pool)]
    tmpls = [subset3d(pool, lo, hi) for lo, hi in bounds]
    opts = prep_options(w)
    ctx = GpuContext(0, args.precision, profile=True)
    ctx.set_projectors(proj, pool.ori_size, r_max)
    # one context per host thread: pools are dealt round-robin, so one context's host-side work (list sizes,
    # result copies) overlaps the other's kernels; their back-projectors are added into ctx's after each step
    lanes = [ctx]
    for _ in range(max(0, args.workers - 1)):
        c = GpuContext(0, args.precision, profile=True)
        c.set_projectors(proj, pool.ori_size, r_max)
        lanes.append(c)
    from concurrent.futures import ThreadPoolExecutor
    execs = [ThreadPoolExecutor(max_workers=1) for _ in lanes]
    # low-resolution proposals: one auxiliary context per lane runs the small exhaustive coarse pass (its
    # sums and back-projectors are discarded); its device time is counted with the lanes'
    lowres = args.proposals3d == "lowres"
    auxes = []
    for _ in (lanes if lowres else []):
        a = GpuContext(0, args.precision, profile=True)
        a.set_projectors(proj, pool.ori_size, r_max)
        auxes.append(a)
    fallback = []
    prep_ctx = GpuContext(0, "fp32", profile=True)
    d_raw = torch.from_numpy(raw.images).cuda()
    dr = dataclasses.replace(raw, images=d_raw)
    staged = [prepared_pool(prep_ctx, t, slice_particles(dr, lo, hi), opts) for t, (lo, hi) in zip(tmpls, bounds)]
    del d_raw, dr
    host_raw = [pin_particles(slice_particles(raw, lo, hi)) for lo, hi in bounds]

    def lowres_pool(c, a, sp):
        from rome_b200.proposal import lowres_estep3d
        out, _, _, low = lowres_estep3d(c, a, sp.pool, args.topk, args.lowres_size, args.min_mass, dev=sp.dev)
        fallback.append((int(low.size), sp.pool.nr_images))
        return out

    def run_lanes(pools):
        if lowres:
            futs = [execs[q % len(lanes)].submit(lowres_pool, lanes[q % len(lanes)], auxes[q % len(lanes)], sp)
                    for q, sp in enumerate(pools)]
        else:
            futs = [execs[q % len(lanes)].submit(map3d_estep_pools_adaptive, lanes[q % len(lanes)], sp.pool, sp.dev)
                    for q, sp in enumerate(pools)]
        res = [f.result() for f in futs]
        for c in lanes[1:]:
            ctx.add_backprojectors(c, clear=True)
        return res

    def step():
        return run_lanes(staged)

    def step_e2e():
        return run_lanes(prepared_stream(prep_ctx, list(zip(tmpls, host_raw)), opts))

    for _ in range(args.warmup):
        step()
    for c in lanes + auxes:
        c.reset_timings()
    fallback.clear()
    with ClockSampler(0) as clk:
        ms, last = _timed(torch, step, args.steps)
    timings = merge_timings([c.get_timings() for c in lanes + auxes])
    timed_fallback = list(fallback)
    step_e2e()
    e_ms, _ = _timed(torch, step_e2e, max(1, args.steps))
    cls = np.concatenate([r["cls"] for r in last]) - 1
    # the timed contexts' device memory is released before the comparison arm runs
    for e in execs:
        e.shutdown(wait=True)
    for c in lanes + auxes:
        c.close()
    # the plain FP32 E-step on the same prepared particles: the comparison arm and the pose judge
    judge = {}
    if args.precision != "fp32":
        with GpuContext(0, "fp32") as c32:
            c32.set_projectors(proj, pool.ori_size, r_max)
            map3d_estep_pools_adaptive(c32, staged[0].pool, staged[0].dev)
            f_ms, f_res = _timed(torch, lambda: [map3d_estep_pools_adaptive(c32, sp.pool, sp.dev) for sp in staged], 1)
        cat = lambda rs, k: np.concatenate([r[k] for r in rs])  # noqa: E731
        same = np.ones(N, bool)
        for k in ("cls", "rot", "tilt", "psi", "xoff", "yoff"):
            same &= cat(last, k) == cat(f_res, k)
        judge = {"pose_agreement_vs_plain_fp32": round(float(same.mean()), 5),
                 "plain_fp32": {"value": round(N / (f_ms / 1e3), 2), "unit": UNIT}}
    hbm, bf16, peak_kind = load_peaks()
    phases = {k: round(v["ms"] / args.steps, 3) for k, v in timings.items() if isinstance(v, dict)}
    # the phase with the most device time names the roofline: the posterior (HBM: diff2 read once, 4 B per
    # hypothesis), the projections or the back-projection (HBM, the algorithmic bytes the library counts),
    # or the contraction (tensor: 4 * active pixels flops per hypothesis, coarse and fine)
    post, gem = timings["posterior"], timings["cross_gemm"]
    hbm_phases = {
        "posterior": "posterior + significance (post_select2_kernel and fallbacks): algorithmic bytes = the diff2 "
                     "rows read once, 4 B per hypothesis",
        "project": "projections (project3d_kernel, coarse and fine): algorithmic bytes = the class volumes read "
                   "once + the projections and operands written",
        "backproject": "back-projection (bp_prep_kernel, list sort, bp3d_list_kernel): algorithmic bytes = 24 B per "
                       "active pixel of every significant hypothesis + 192 B (24 FP64 updates) per active pixel of "
                       "every back-projected slice; bound in practice by L2 FP64 atomics"}
    top = max(hbm_phases, key=lambda k: timings[k]["ms"] if timings[k]["bytes"] > 0 else -1.0)
    if timings[top]["ms"] >= gem["ms"]:
        ph = timings[top]
        ach = ph["bytes"] / (ph["ms"] / 1e3) / 1e9
        roof = {"bound": "hbm", "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s", "frac": round(ach / hbm, 4),
                "traffic": None, "peak_kind": peak_kind, "launches": int(ph["launches"]),
                "ms_per_step": round(ph["ms"] / args.steps, 3), "kernel": hbm_phases[top]}
    else:
        ach = gem["flops"] / (gem["ms"] / 1e3) / 1e12
        roof = {"bound": "tensor", "achieved": round(ach, 2), "peak": bf16, "unit": "TFLOP/s",
                "frac": round(ach / bf16, 4), "traffic": None, "peak_kind": peak_kind,
                "launches": int(gem["launches"]), "ms_per_step": round(gem["ms"] / args.steps, 3),
                "kernel": "cross-term contraction (coarse tc_gemm_kernel + fine pass): 4 * active pixels flops "
                          "per hypothesis"}
    line = {
        "metric": "MAP3D E-step particles/s (" + ("coarse pass restricted to low-resolution proposals" if lowres
                                                  else "exhaustive search") + ")",
        "value": round(N / (ms / args.steps / 1e3), 2),
        "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {"fp32": "f32", "bf16": "bf16", "bf16x3": "bf16x3"}[args.precision],
        "data": "synthetic (seeded random-blob volumes, Fourier-slice particles, CTF, white noise)",
        "config": {"workload": args.config, "particles": N, "image": w.ori_size, "coarse_size": pool.coarse_size,
                   "classes": w.n_classes, "directions": pool.nr_dir, "psi": pool.nr_psi,
                   "translations": pool.nr_trans, "oversampling": 1, "pool": args.pool, "precision": args.precision,
                   "inputs": "larger than L2 (no flush)", "host_threads": len(lanes),
                   "snr": w.snr, "snr_range": w.snr_range, "noisy_fraction": w.noisy_fraction,
                   "build_s": round(t_build, 1)},
        "e2e": {"value": round(N / (e_ms / max(1, args.steps) / 1e3), 2), "unit": UNIT,
                "from": "float32 images + metadata in page-locked host memory: copy, image preparation "
                        "(setFourierTransforms), E-step, results back",
                "h2d_bytes_per_step": int(sum(prep_h2d_bytes(r) for r in host_raw)),
                "d2h_bytes_per_step": int(N * (11 * 8 + 4))},
        "class_agreement_vs_truth": round(float(np.mean(cls == truth["cls"])), 4),
        "nr_sign_mean": round(float(np.mean(np.concatenate([r["nr_sign"] for r in last]))), 1),
        # the per-particle spread of the coarse significance (what the reference's
        # Exp_Mweight_old::analysis records per pool, src/exp_mweight.cpp:95-160): coarse-significant
        # points per particle, each refined by 32 fine hypotheses
        "coarse_significant_per_particle": dict(zip(
            ("min", "p10", "p50", "p90", "p99", "max"),
            (float(v) for v in np.percentile(np.concatenate([r["nr_sign"] for r in last]), [0, 10, 50, 90, 99, 100])))),
        "judge": judge,
        "phases_ms_per_step": phases,
        "gpu_launches": int(timings["total_launches"]),
        "roofline": roof,
        "clocks": clk.summary(),
    }
    if lowres:
        line["proposals3d"] = {"kind": "lowres", "k": args.topk, "coarse_size": args.lowres_size,
                               "min_mass": args.min_mass,
                               "fallback_fraction": round(sum(a for a, _ in timed_fallback)
                                                          / max(1, sum(b for _, b in timed_fallback)), 5)}
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args, w)
    prep_ctx.close()
    print(json.dumps(line), flush=True)


def run_prep(args):
    """Secondary mode: the image preparation (ParticleModel::setFourierTransforms)
    of the configuration's particles from float32 images, pool by pool.  value:
    images resident in HBM; e2e: page-locked host images copied in (next pool
    while this one is prepared), prepared arrays left on the device for the
    E-step, per-particle outputs read back.  One JSON line."""
    import dataclasses

    import torch

    from rome_b200.map2d import GpuContext
    from rome_b200.particles import h2d_bytes, pin_particles, prepare_particles, prepared_stream
    from rome_b200.workload import CONFIGS, build_map2d, image_template, prep_options, raw_particles, slice_particles, subset
    w = CONFIGS[args.config]
    if args.particles:
        w = dataclasses.replace(w, n_particles=args.particles)
    pool, _, _, truth = build_map2d(w)
    raw = raw_particles(pool, truth)
    tmpl = image_template(pool)
    del pool
    opts = prep_options(w)
    N = tmpl.nr_images
    bounds = [(lo, min(N, lo + args.pool)) for lo in range(0, N, args.pool)]
    ctx = GpuContext(0, "fp32", profile=True)
    d_raw = torch.from_numpy(raw.images).to("cuda:0")
    dr = dataclasses.replace(raw, images=d_raw)

    def step():
        # each pool's outputs are released before the next pool (an E-step would consume them)
        for lo, hi in bounds:
            prepare_particles(ctx, slice_particles(dr, lo, hi), opts, tmpl.sigma2_noise, tmpl.current_size,
                              on_device=True, power=False)

    for _ in range(args.warmup):
        step()
    ctx.reset_timings()
    with ClockSampler(0) as clk:
        ms, _ = _timed(torch, step, args.steps)
    t = ctx.get_timings()
    host = [pin_particles(slice_particles(raw, lo, hi)) for lo, hi in bounds]
    items = [(subset(tmpl, lo, hi), h) for (lo, hi), h in zip(bounds, host)]
    e_step = lambda: [q.pool.highres_Xi2 for q in prepared_stream(ctx, items, opts)]  # noqa: E731
    e_step()
    e_ms, _ = _timed(torch, e_step, args.steps)
    hbm, _, peak_kind = load_peaks()
    ph = t["images"]
    # algorithmic bytes: the float32 image in, the five FP64 half-plane arrays out
    F = tmpl.current_size * (tmpl.current_size // 2 + 1)
    per = raw.images[0].nbytes + 5 * F * 8
    achieved = per * N * args.steps / (ph["ms"] / 1e3) / 1e9
    line = {
        "metric": "image preparation particles/s (setFourierTransforms)", "value": round(N / (ms / args.steps / 1e3), 2),
        "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (the configuration's particles as float32 real-space images)",
        "config": {"workload": args.config + " image preparation", "particles": N, "image": w.ori_size,
                   "pool": args.pool, "options": dataclasses.asdict(opts), "inputs": "larger than L2 (no flush)"},
        "e2e": {"value": round(N / (e_ms / args.steps / 1e3), 2), "unit": UNIT,
                "h2d_bytes_per_step": int(sum(h2d_bytes(h) for h in host)),
                "d2h_bytes_per_step": int(N * 3 * 8)},
        "gpu_launches": int(t["total_launches"]),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                     "frac": round(achieved / hbm, 4), "traffic": None, "peak_kind": peak_kind,
                     "kernel": "the preparation phase as a whole (own kernels and cuFFT), algorithmic bytes "
                               f"{per} per image", "launches": int(ph["launches"])},
        "clocks": clk.summary(),
    }
    ctx.close()
    print(json.dumps(line), flush=True)


def run_reconstruct(args):
    """Secondary mode: reconstruction at known poses (the reference's
    rome_reconstruct) of 10,000 particles of 128^2 into the padded 259^3
    grid of the 3D configuration's M-step.  value: back-projection of the
    prepared spectra resident in HBM (particles/s); reconstruct_ms: the
    gridding-corrected reconstruction of the volume (10 iterations); e2e:
    STAR + MRCS on disk -> loader -> device preparation -> back-projection ->
    reconstruction -> volume in host memory.  Images are seeded noise with
    random poses and CTFs (the work does not depend on their content).  One
    JSON line."""
    import tempfile

    import torch

    from rome_b200.map2d import GpuContext
    from rome_b200.particles import PrepOptions, prepare_particles
    from rome_b200.reconstruct_poses import POSE_LABELS, reconstruct_from_star
    from rome_b200.star_mrcs import ParticleStack
    from rome_b200.synthetic import write_mrcs
    N = args.particles or 10000
    S, angpix = 128, 1.5
    rng = np.random.default_rng(5)
    tmp = tempfile.mkdtemp(prefix="rome_recon_bench_")
    mrcs = os.path.join(tmp, "p.mrcs")
    write_mrcs(mrcs, rng.standard_normal((N, S, S), dtype=np.float32), angpix)
    star = os.path.join(tmp, "p.star")
    rot, psi = rng.uniform(0, 360, N), rng.uniform(0, 360, N)
    tilt = np.rad2deg(np.arccos(rng.uniform(-1, 1, N)))
    ox, oy = rng.uniform(-4, 4, N), rng.uniform(-4, 4, N)
    du, dv, da = rng.uniform(1e4, 3e4, N), rng.uniform(1e4, 3e4, N), rng.uniform(0, 180, N)
    labels = ["rlnImageName", "rlnMicrographName", "rlnDefocusU", "rlnDefocusV", "rlnDefocusAngle", "rlnVoltage",
              "rlnSphericalAberration", "rlnAmplitudeContrast", *POSE_LABELS]
    with open(star, "w") as f:
        f.write("data_\nloop_\n" + "".join(f"_{lab} #{i + 1}\n" for i, lab in enumerate(labels)))
        for i in range(N):
            f.write(f"{i + 1:06d}@{mrcs} mic{i % 50:03d} {du[i]:.3f} {dv[i]:.3f} {da[i]:.3f} 300 2.7 0.1 "
                    f"{rot[i]:.4f} {tilt[i]:.4f} {psi[i]:.4f} {ox[i]:.4f} {oy[i]:.4f}\n")
    poses = np.stack([rot, tilt, psi, ox, oy], axis=1)
    st = ParticleStack(star)
    order = np.argsort(np.asarray([int(x.split("@")[0]) for x in st.columns["rlnImageName"]]))  # file order
    r_max, F = S // 2, S * (S // 2 + 1)
    pad = 2 * (2 * r_max + 1) + 1
    ctx = GpuContext(0, "fp32", profile=True)
    ctx.set_projectors(np.zeros((1, pad, pad, pad // 2 + 1, 2)), S, r_max)
    opts = PrepOptions(pixel_size=angpix, particle_diameter=S * angpix, do_ctf_correction=True)
    sig = np.ones((st.nr_groups, S // 2 + 1))
    spectra = []
    for imgs in st.device_pools(0, args.pool, order=order):
        imgs.xoff[:] = 0.0
        imgs.yoff[:] = 0.0
        o = prepare_particles(ctx, imgs, opts, sig, S, on_device=True, power=False)
        spectra.append((o["Fimg_nomask_real"], o["Fimg_nomask_imag"], o["Fctf"],
                        poses[imgs.first_image:imgs.first_image + imgs.nr_images]))

    def step():
        for re, im, c, ps in spectra:
            ctx.backproject_images(0, re, im, c, ps)

    for _ in range(args.warmup):
        step()
    ctx.reset_timings()
    with ClockSampler(0) as clk:
        ms, _ = _timed(torch, step, args.steps)
    t = ctx.get_timings()
    rec = lambda: ctx.reconstruct(0, S, 3, np.zeros(S // 2 + 1), 1.0, 1.0, 10, False)  # noqa: E731
    rec()  # warm-up: cuFFT plans and work buffers
    rec_ms, _ = _timed(torch, rec, 1)
    del spectra
    ctx.close()
    # the pool loader alone: STAR/MRCS (page cache) -> page-locked buffers -> device, one pool ahead
    def load_all():
        n = 0
        for q in st.device_pools(0, args.pool, order=order):
            n += q.nr_images
        return n

    load_all()
    load_runs = sorted(_timed(torch, load_all, 1)[0] for _ in range(5))
    load_ms = load_runs[len(load_runs) // 2]
    reconstruct_from_star(star, angpix, 10, True, pool=args.pool)  # warm-up (page cache, allocations)
    e_ms, _ = _timed(torch, lambda: reconstruct_from_star(star, angpix, 10, True, pool=args.pool), 1)
    hbm, _, peak_kind = load_peaks()
    bp = t["backproject"]
    achieved = bp["bytes"] / (bp["ms"] / 1e3) / 1e9
    line = {
        "metric": "reconstruction at known poses: back-projection particles/s (rome_reconstruct)",
        "value": round(N / (ms / args.steps / 1e3), 2), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded noise images, random poses and CTFs; the work does not depend on content)",
        "config": {"workload": "map3d_cfg3 M-step shapes: reconstruction at known poses", "particles": N, "image": S,
                   "pad": pad, "gridding_iterations": 10, "pool": args.pool, "ctf": True,
                   "inputs": "larger than L2 (no flush)"},
        "reconstruct_ms": round(rec_ms, 3),
        "loader": {"value": round(N / (load_ms / 1e3), 2), "unit": UNIT, "ms": round(load_ms, 2),
                   "ms_runs": [round(x, 2) for x in load_runs],
                   "GB_per_s": round(N * S * S * 4 / (load_ms / 1e3) / 1e9, 2),
                   "what": "STAR/MRCS pool loader: memory-mapped stack (page cache) -> page-locked buffer -> "
                           "device, next pool read while the current one is copied; median of 5 runs after "
                           "one warm-up, each run's page-locked buffers and side stream created inside its "
                           "timed region"},
        "e2e": {"value": round(N / (e_ms / 1e3), 2), "unit": UNIT,
                "from": "STAR + MRCS on disk (page cache): loader, copy, device preparation, back-projection, "
                        "reconstruction, volume back",
                "ms": round(e_ms, 2), "h2d_bytes_per_step": int(N * S * S * 4),
                "d2h_bytes_per_step": int(S ** 3 * 8)},
        "gpu_launches": int(t["total_launches"]),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                     "frac": round(achieved / hbm, 4), "traffic": None, "peak_kind": peak_kind,
                     "kernel": "bp_images_kernel: algorithmic bytes = spectra and CTF read once (24 B per "
                               "coefficient); the 12 FP64 atomics per active pixel land in L2",
                     "launches": int(bp["launches"])},
        "cpu_baseline": (reference_rate_recon() if not args.no_cpu_baseline and os.path.exists(REF_RECON)
                         else None),
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    a = parse()
    if a.mode == "prep" and a.impl != "reference":
        run_prep(a)
        sys.exit(0)
    if a.mode == "reconstruct" and a.impl != "reference":
        run_reconstruct(a)
        sys.exit(0)
    if a.config.startswith("map3d") and a.impl != "reference":
        run_ours_3d(a)
        sys.exit(0)
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)
