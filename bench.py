"""Benchmark: forward+backward Mrays/s of the differentiable Gaussian ray caster on the 1M-Gaussian
unbounded scene with 16 views of uneven resolution (the batched, BF16-storage form), next to the
plain FP32 single-view drop-in form on the same views, the reference algorithm on the host cores
and the HBM roofline of the dominant kernel.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--views V]

A step is one training iteration of the hot path over the batch: pre-pass + LBVH build + colour
pass + forward launch + MSE loss + backward launch + SH/SG backward and gradient assembly.  Inputs
(parameters 460 MB FP32 / 314 MB BF16-stored) are larger than the 126 MB L2, so no flush is needed
between timed steps.  Multi-GPU runs are independent replicas (one GPU renders the whole batch;
the path needs no exchange), timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+bwd Mrays/s @1M Gaussians: plain FP32 vs batched+BF16 at PSNR Δ≤0.05 dB"
WORKLOAD = "unbounded_1m"


def _dist():
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    return rank, world, local


def _clock_sampler(gpu_index):
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    try:
        return subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
    except OSError:
        return None


def _clock_summary(proc):
    if proc is None:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
    proc.terminate()
    try:
        out, _ = proc.communicate(timeout=5)
    except subprocess.TimeoutExpired:
        proc.kill()
        out, _ = proc.communicate()
    sm, mx, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in out.strip().splitlines():
        f = [x.strip() for x in line.split(",")]
        if len(f) < 9:
            continue
        try:
            sm.append(float(f[1]))
            mx = float(f[2])
        except ValueError:
            continue
        for nm, v in zip(names, f[5:9]):
            if v.lower() == "active":
                reasons.add(nm)
    return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
            "samples": len(sm)}


def max_over_ranks(value: float, device) -> float:
    """Max of a per-rank scalar over the process group (the step time of the slowest replica)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _profile_figures(name):
    """key = value figures of a committed ncu summary under profiles/ (empty when absent)."""
    out = {}
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            for line in f:
                if "=" in line and not line.lstrip().startswith("#"):
                    k, v = line.split("=", 1)
                    try:
                        out[k.strip()] = float(v.split()[0])
                    except (ValueError, IndexError):
                        pass
    except OSError:
        pass
    return out


TRAFFIC_PROFILE = "k_render_traffic_unbounded_1m_16view.txt"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def bytes_per_gaussian(nsg, sh_coeffs, bf16):
    """Storage bytes of one Gaussian's parameters (positions, scales, quaternion, density, SH, SG)."""
    amp = 2 if bf16 else 4
    return 12 + 12 + 16 + amp + 3 * sh_coeffs * amp + nsg * (3 * amp + 4 + 12)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--views", type=int, default=16)
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--no-plain", action="store_true", help="skip the plain single-view comparison")
    ap.add_argument("--no-cpu", action="store_true", help="skip the host-core baseline")
    ap.add_argument("--cpu-rays", type=int, default=4096, help="rays per view in the accuracy and host-core samples")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (engine defaults)")
    ap.add_argument("--no-graph", action="store_true", help="skip the CUDA-graph replay measurement")
    ap.add_argument("--plain-only", action="store_true",
                    help="run only the plain drop-in form (RenderOptixFunction per view, parity arithmetic) for "
                         "--steps steps and print its Mrays/s (a profiling case for its kernels)")
    ap.add_argument("--drift", type=int, default=0,
                    help="also measure refit-only LBVH drift over this many captured training iterations")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank, world, local = _dist()
    if args.impl == "reference":
        return reference_arm(args, rank, world)
    if args.plain_only:
        return plain_only(args, local)
    return our_arm(args, rank, world, local)


def plain_only(args, local):
    """The plain FP32 drop-in form alone: RenderOptixFunction forward + MSE + backward per view."""
    import torch
    from ray_gauss_b200.engine import Engine
    from ray_gauss_b200.optix_raycasting.render_optix import RenderOptixFunction, RenderOptixSettings
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    _, P32, cams, white = _setup(args, dev)
    P = {k: v.clone().requires_grad_(True) for k, v in P32.items()}
    nsg = P["sph_gauss_features"].shape[2]
    eng = Engine(local)
    targets = [torch.rand((c.image_width * c.image_height, 3), device=dev) for c in cams]

    def step():
        for v, cam in enumerate(cams):
            s = RenderOptixSettings(eng, False, None, None, None, None, None, cam, 1024, nsg, 0, 0, 0, (1, 1), white,
                                    None, mode="parity")
            img = RenderOptixFunction.apply(*(P[k] for k in GRAD_KEYS), s)
            torch.nn.functional.mse_loss(img, targets[v]).backward()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    R = sum(c.image_width * c.image_height for c in cams)
    print(json.dumps({"form": "plain FP32 drop-in (RenderOptixFunction per view, parity arithmetic)",
                      "gaussians": int(P32["positions"].shape[0]), "views": len(cams), "rays_per_step": R,
                      "ms_per_step": round(ms, 3), "value": round(R / (ms * 1e-3) / 1e6, 3), "unit": "Mrays/s"}))
    return 0


def _setup(args, device):
    import torch
    from ray_gauss_b200 import synthetic as S
    p, cams, white = S.workload(WORKLOAD, seed=0, device="cpu", n=args.n)
    cams = cams[: args.views]
    cams = [c.to(device) for c in cams]
    P32 = {k: v.to(device) for k, v in p.items()}
    return p, P32, cams, white


def _bf16(P32):
    import torch
    P = dict(P32)
    for k in ("densities", "color_features", "sph_gauss_features"):
        P[k] = P32[k].to(torch.bfloat16)
    return P


def our_arm(args, rank, world, local):
    import torch
    from ray_gauss_b200.batched import BatchedRenderFunction, BatchedViews
    from ray_gauss_b200.engine import Engine
    from ray_gauss_b200.optix_raycasting.render_optix import RenderOptixFunction, RenderOptixSettings

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    p_host, P32, cams, white = _setup(args, dev)
    n = P32["positions"].shape[0]
    eng = Engine(local)
    views = BatchedViews(cams, white_background=white, mode="fast", engine=eng)
    R = views.n_rays
    eng.reserve(n, len(cams), R)
    Pb = _bf16(P32)
    leaves = {k: v.clone().requires_grad_(True) for k, v in Pb.items()}
    g = torch.Generator(device=dev)
    g.manual_seed(1)
    target = torch.rand((R, 3), device=dev, generator=g)

    def step_batched(P):
        out = BatchedRenderFunction.apply(P["positions"], P["scales"], P["quaternions"], P["densities"],
                                          P["color_features"], P["sph_gauss_features"], P["bandwidth_sharpness"],
                                          P["lobe_axis"], views)
        loss = torch.nn.functional.mse_loss(out, target)
        loss.backward()
        return loss

    def zero(P):
        for v in P.values():
            v.grad = None

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    # ---- autotune the render kernels on this scene and these views (a few launches) ----
    tuning = eng.get_tuning()
    if not args.no_tune:
        from ray_gauss_b200.autotune import autotune
        tuning = autotune(Pb, views, target, repeats=1, chunks=(32, 64, 128), capacities=(64,), ctas=(0,))

    # ---- headline: batched BF16-storage form (device-resident inputs) ----
    for _ in range(args.warmup):
        zero(leaves)
        step_batched(leaves)
    torch.cuda.synchronize()
    eng.status(reset=True)
    eng.timers = {}
    launches0 = eng.kernel_launches()
    clocks = _clock_sampler(local) if rank == 0 else None
    barrier()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(args.steps):
        zero(leaves)
        step_batched(leaves)
    t1.record()
    torch.cuda.synchronize()
    barrier()
    clk = _clock_summary(clocks) if rank == 0 else None
    ms = t0.elapsed_time(t1) / args.steps
    launches = eng.kernel_launches() - launches0
    timers, eng.timers = eng.timers, None
    st = eng.status()
    # the fine-grained traversal counters come from one more, untimed step of the counting kernels
    eng.set_tuning(diagnostics=1)
    eng.status(reset=True)
    zero(leaves)
    step_batched(leaves)
    torch.cuda.synchronize()
    diag = eng.status(reset=True)
    eng.set_tuning(diagnostics=0)
    for k in ("node_visits", "leaf_tests", "list_entries", "slab_steps", "entry_slabs"):
        st[k] = diag[k] * args.steps          # counters_per_step divides by the step count
    ms_max = max_over_ranks(ms, dev)
    value = world * R / (ms_max * 1e-3) / 1e6

    # render launches (CUDA events on the launching stream, averaged over the timed steps)
    bwd_ms = statistics.mean(a.elapsed_time(b) for a, b in timers["launch_backward"])
    fwd_ms = statistics.mean(a.elapsed_time(b) for a, b in timers["launch_forward"])
    prep_ms = statistics.mean(a.elapsed_time(b) for a, b in timers["prepare"])
    shb_ms = statistics.mean(a.elapsed_time(b) for a, b in timers["backward_sh"])
    nsg = P32["sph_gauss_features"].shape[2]
    ncoef = P32["color_features"].shape[2]
    V = len(cams)
    p_store = bytes_per_gaussian(nsg, ncoef, True)
    g_bytes = bytes_per_gaussian(nsg, ncoef, False)
    # algorithmic bytes per launch (parameters counted once per launch, all views):
    #   forward  B_fwd = N P_store + 12 R (parameters read once, ray colours written)
    #   backward the leaf records (64 B) + scale/quaternion (32 B) + colour per view (16 B) read once per
    #            Gaussian, the gradient accumulators written once (48 B + 16 B per view), ray colour and
    #            dL/dcolour read once per ray (24 B), and the forward's hit-list record read once
    rec_bytes = 4 * st.get("record_words", 0)   # size of the last forward's record (not a running sum)
    alg_fwd = n * p_store + 12 * R
    alg_bwd = n * (64 + 32 + 16 * V) + n * (48 + 16 * V) + 24 * R + rec_bytes
    peak, peak_kind = _peaks()
    # DRAM traffic and SM issue utilisation from the committed ncu summary of the same workload (a
    # profiler number is never timed here)
    prof = _profile_figures(TRAFFIC_PROFILE)
    same = prof.get("gaussians") == n and prof.get("views") == V
    hit_pairs = st.get("hit_pairs", 0) / max(1, args.steps)   # forward + backward recompute, per step
    rl_launches = {}
    for name, ms_l, alg in (("forward", fwd_ms, alg_fwd), ("backward", bwd_ms, alg_bwd)):
        ach = alg / (ms_l * 1e-3) / 1e9
        traffic = int(prof[f"{name}_dram_bytes"]) if same and f"{name}_dram_bytes" in prof else None
        rl_launches[name] = {
            "kernel": f"k_render<{name}> (rg_launch_{name})", "ms_per_launch": round(ms_l, 3),
            "algorithmic_bytes_per_launch": int(alg), "achieved_gbs": round(ach, 2), "frac": round(ach / peak, 6),
            "traffic": traffic, "traffic_over_algorithmic": round(traffic / alg, 3) if traffic else None,
            "sm_issue_frac_ncu": prof.get(f"{name}_sm_issue_frac"),
            # each (ray, slab, Gaussian) pair evaluates 8 samples in the forward and again in the backward
            "g_hit_samples_per_s": round(8 * hit_pairs / 2 / (ms_l * 1e-3) / 1e9, 3)}
    dom = "forward" if fwd_ms >= bwd_ms else "backward"
    d = rl_launches[dom]
    roofline = {"bound": "hbm", "achieved": d["achieved_gbs"], "peak": peak, "unit": "GB/s", "frac": d["frac"],
                "traffic": d["traffic"], "peak_source": peak_kind, "kernel": d["kernel"],
                "algorithmic_bytes_per_launch": d["algorithmic_bytes_per_launch"],
                "traffic_over_algorithmic": d["traffic_over_algorithmic"],
                "sm_issue_frac_ncu": d["sm_issue_frac_ncu"], "launches": rl_launches,
                "note": "the dominant launch is the longer of the two render launches; both are bound by SM "
                        "instruction issue (gathers of L2-resident Gaussian records, FP32 and SFU sample math), "
                        "not by HBM: the HBM fraction is small by construction and sm_issue_frac_ncu is the "
                        "compute-side figure; traffic above the algorithmic bytes is the forward's hit-list "
                        "record and per-view colour tables"}
    # step-level algorithmic bytes (parameters read twice, gradients written once, 36 B per ray)
    b_step = 2 * n * p_store + n * g_bytes + 36 * R

    # ---- the same step captured as one CUDA graph (refit + forward + loss + backward) ----
    graph = None
    if not args.no_graph:
        from ray_gauss_b200.graph import GraphedStep
        gleaves = {k: v.detach().clone() for k, v in Pb.items()}
        gstep = GraphedStep(gleaves, views, target)
        gstep.replay()
        torch.cuda.synchronize()
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record()
        for _ in range(args.steps):
            gstep.replay()
        g1.record()
        torch.cuda.synchronize()
        g_ms = g0.elapsed_time(g1) / args.steps
        graph = {"value": round(R / (g_ms * 1e-3) / 1e6, 3), "unit": "Mrays/s", "ms_per_step": round(g_ms, 3),
                 "form": "GraphedStep.replay(): LBVH refit + colour + forward + MSE + backward in one CUDA graph"}
        views.update = False
        del gstep, gleaves

    # ---- a whole training iteration on the FP32 trained tensors of the reference's point cloud:
    #      get_data activations + the graph above + the fused Adam / statistics / clamp tail; and
    #      that tail alone ----
    train = None
    if not args.no_graph:
        from ray_gauss_b200.graph import GraphedStep
        from ray_gauss_b200.train_tail import FusedTrainTail, LrSchedule, point_cloud_data, raw_from_render_inputs
        tleaves = {k: v.detach().contiguous() for k, v in raw_from_render_inputs(P32).items()}
        tparams = {k: v for k, v in tleaves.items() if v.numel()}
        tail = FusedTrainTail(tparams, {k: LrSchedule(1e-5) for k in tparams},
                              roles={"positions": "positions", "densities": "densities", "scales": "scales",
                                     "quaternions": "quaternions"})
        min_scale = torch.full((n,), -12.0, device=dev)
        tstep = GraphedStep(tleaves, views, target, tail=tail, min_scale=min_scale,
                            activation=lambda r: point_cloud_data(r, normalized_quaternion=False))
        tstep.replay()
        torch.cuda.synchronize()
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record()
        for _ in range(args.steps):
            tstep.replay()
        g1.record()
        torch.cuda.synchronize()
        t_ms = g0.elapsed_time(g1) / args.steps
        tgrads = {k: tstep.grads[k].contiguous() for k in tparams}
        tail.step(min_scale=min_scale, grads=tgrads)
        torch.cuda.synchronize()
        g0.record()
        for _ in range(args.steps):
            tail.step(min_scale=min_scale, grads=tgrads)
        g1.record()
        torch.cuda.synchronize()
        tail_ms = g0.elapsed_time(g1) / args.steps
        # param, exp_avg, exp_avg_sq read + written and the gradient read per float; per Gaussian the
        # three statistics read + written and min_scale read
        tail_bytes = 28 * sum(v.numel() for v in tparams.values()) + 28 * n
        tail_gbs = tail_bytes / (tail_ms * 1e-3) / 1e9
        train = {"value": round(R / (t_ms * 1e-3) / 1e6, 3), "unit": "Mrays/s", "ms_per_step": round(t_ms, 3),
                 "form": "GraphedStep(tail=FusedTrainTail, activation=point_cloud_data).replay() on the FP32 "
                         "trained tensors: get_data activations + LBVH refit + colour + forward + MSE + backward + "
                         "Adam on every tensor + statistics + clamps in one CUDA graph",
                 "tail": {"kernel": "k_train_tail (rg_train_tail_step)", "ms_per_launch": round(tail_ms, 4),
                          "algorithmic_bytes_per_launch": int(tail_bytes), "achieved_gbs": round(tail_gbs, 1),
                          "peak_gbs": peak, "frac": round(tail_gbs / peak, 4), "bound": "hbm"}}
        views.update = False
        # densify + prune (every few hundred iterations in the reference) on the trained statistics
        # of these replays: 80th-percentile gradient threshold, clone/split boundary at the median
        # scale; one untimed call (the allocator grows to the new size), then three on fresh copies
        from ray_gauss_b200.densify import densify_and_prune
        mean_g = tail.stats["xyz_gradient_accum_norm"] / tail.stats["num_accum"].clamp(min=1)
        thr = float(torch.quantile(mean_g[:1 << 20], 0.8))
        extent = float(torch.exp(tparams["scales"].detach()).max(dim=1).values[:1 << 20].median()) * 100.0
        d_ms, d_out = [], None
        for _ in range(4):
            dt = FusedTrainTail({k: v.detach().clone() for k, v in tparams.items()},
                                {k: LrSchedule(1e-5) for k in tparams}, roles=tail.roles)
            for k in tparams:
                dt.exp_avg[k].copy_(tail.exp_avg[k])
                dt.exp_avg_sq[k].copy_(tail.exp_avg_sq[k])
            for k in tail.stats:
                dt.stats[k].copy_(tail.stats[k])
            f3d = torch.full((n, 1), -12.0, device=dev)
            torch.cuda.synchronize()
            g0.record()
            d_out = densify_and_prune(dt, f3d, thr, 0.05, extent)
            g1.record()
            torch.cuda.synchronize()
            d_ms.append(g0.elapsed_time(g1))
            del dt, f3d
        floats = sum(v.numel() for v in tparams.values()) // n
        moved = 2 * d_out["n"] * 4 * (3 * floats + 4)     # each output row: params, moments, stats read + written
        dens_ms = sorted(d_ms[1:])[1]
        densify = {"ms": round(dens_ms, 3), "gaussians_in": n, "gaussians_out": d_out["n"],
                   "cloned": d_out["n_clone"], "split": d_out["n_split"], "pruned": d_out["n_pruned"],
                   "bytes_moved": int(moved), "achieved_gbs": round(moved / (dens_ms * 1e-3) / 1e9, 1),
                   "form": "densify_and_prune(): rg_densify_plan (classify + scan + count read-back) + "
                           "rg_densify_apply (one gather over every tensor, moment and statistic)"}
        train["densify"] = densify
        # scene I/O: this cloud as a trained-scene PLY (the reference's convertpth_to_ply layout),
        # loaded back: wall time of load_trained_ply (page-cache read into pinned memory, one copy,
        # one conversion kernel) and the conversion kernel alone on CUDA events
        import tempfile
        from ray_gauss_b200.io import PlyVertices, load_trained_ply, write_trained_ply
        with tempfile.TemporaryDirectory() as td:
            nsg_t = tleaves["bandwidth_sharpness"].shape[1]
            hn = tleaves["spherical_harmonics"].shape[2] + 1
            path = write_trained_ply(f"{td}/scene.ply", tleaves, hn, nsg_t, tail.stats["xyz_gradient_accum_norm"])
            fsize = os.path.getsize(path)
            load_trained_ply(path, dev)
            torch.cuda.synchronize()
            w0 = time.perf_counter()
            loaded = load_trained_ply(path, dev)
            torch.cuda.synchronize()
            load_s = time.perf_counter() - w0
            same = all(torch.equal(loaded["params"][k], tleaves[k].detach()) for k in tleaves)
            ply = PlyVertices(path, dev)
            cols = torch.empty((ply.n, len(ply.names)), dtype=torch.float32, device=dev)
            targets = [(nm, cols[:, j], None) for j, nm in enumerate(ply.names)]
            ply.fill(targets)
            torch.cuda.synchronize()
            g0.record()
            ply.fill(targets)
            g1.record()
            torch.cuda.synchronize()
            k_ms = g0.elapsed_time(g1)
            del loaded, ply, cols
        train["scene_io"] = {"file_bytes": int(fsize), "load_trained_ply_ms": round(load_s * 1e3, 2),
                             "load_gbs": round(fsize / load_s / 1e9, 2), "round_trip_equal": bool(same),
                             "records_to_columns_ms": round(k_ms, 3),
                             "records_to_columns_gbs": round(2 * fsize / (k_ms * 1e-3) / 1e9, 1),
                             "form": "write_trained_ply then load_trained_ply of the 1M-Gaussian cloud; kernel: "
                                     "every field of every record read once and written once"}
        # the training loop's other per-Gaussian passes: the 3D filter over this step's cameras
        # (every 100 iterations) and the k-NN initial scales (once, for clouds without scales)
        from ray_gauss_b200.filter3d import compute_3D_filter
        from ray_gauss_b200.knn import dist_cuda2
        pos = tleaves["positions"].detach().contiguous()
        compute_3D_filter(pos, cams)
        dist_cuda2(pos)
        torch.cuda.synchronize()
        g0.record()
        compute_3D_filter(pos, cams)
        g1.record()
        torch.cuda.synchronize()
        f_ms = g0.elapsed_time(g1)
        g0.record()
        dist_cuda2(pos)
        g1.record()
        torch.cuda.synchronize()
        k_ms = g0.elapsed_time(g1)
        train["filter_3D"] = {"ms": round(f_ms, 3), "gaussians": n, "cameras": len(cams),
                              "form": "compute_3D_filter(): two kernels, cameras in shared memory"}
        train["knn_scales"] = {"ms": round(k_ms, 3), "points": n,
                               "form": "dist_cuda2(): Morton sort + warp-shared box search, exact 3-NN"}
        del tstep, tleaves, tparams, tail, tgrads

    # ---- e2e through the public API: host parameters and targets in, loss out ----
    # Every step copies its parameters and target from pinned host memory and reads its loss back.
    # The copies run on a copy stream into the other of two device buffers while the previous step
    # computes (double buffering, as a training loop prefetches its next batch): the first step's
    # copy and every other step's copy lie inside the timed region, none beyond it.
    e2e = None
    if rank == 0 or True:
        host = {k: v.detach().cpu().pin_memory() for k, v in Pb.items()}
        host_target = target.cpu().pin_memory()
        bufs = [({k: torch.empty_like(v) for k, v in Pb.items()}, torch.empty_like(target)) for _ in range(2)]
        h2d = sum(v.numel() * v.element_size() for v in host.values()) + host_target.numel() * 4
        loss_host = torch.empty((), dtype=torch.float32).pin_memory()
        copy_stream = torch.cuda.Stream(device=dev)
        copied = [torch.cuda.Event() for _ in range(2)]
        released = [torch.cuda.Event() for _ in range(2)]

        def copy_in(b):
            with torch.cuda.stream(copy_stream):
                copy_stream.wait_event(released[b])   # the step that last read buffer b is done
                for k in host:
                    bufs[b][0][k].copy_(host[k], non_blocking=True)
                bufs[b][1].copy_(host_target, non_blocking=True)
                copied[b].record(copy_stream)

        def step_e2e(i, last):
            b = i % 2
            if not last:
                copy_in(1 - b)                        # the next step's inputs, behind this step
            torch.cuda.current_stream().wait_event(copied[b])
            P = {k: v.requires_grad_(True) for k, v in bufs[b][0].items()}
            out = BatchedRenderFunction.apply(P["positions"], P["scales"], P["quaternions"], P["densities"],
                                              P["color_features"], P["sph_gauss_features"],
                                              P["bandwidth_sharpness"], P["lobe_axis"], views)
            loss = torch.nn.functional.mse_loss(out, bufs[b][1])
            loss.backward()
            loss_host.copy_(loss.detach(), non_blocking=True)
            for v in P.values():
                v.grad = None
                v.requires_grad_(False)
            released[b].record(torch.cuda.current_stream())

        for b in range(2):
            released[b].record(torch.cuda.current_stream())
        copy_in(0)
        for i in range(2):
            step_e2e(i, i == 1)
        torch.cuda.synchronize()
        n_e2e = max(3, args.steps)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        copy_stream.wait_event(e0)            # no copy of the timed steps starts before the timer
        copy_in(0)
        for i in range(n_e2e):
            step_e2e(i, i == n_e2e - 1)
        e1.record()
        torch.cuda.synchronize()
        e_ms = e0.elapsed_time(e1) / n_e2e
        e2e = {"value": round(world * R / (e_ms * 1e-3) / 1e6, 3), "unit": "Mrays/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": 4, "ms_per_step": round(e_ms, 3),
               "form": "BatchedRenderFunction forward + MSE + backward on parameters and target copied from pinned "
                       "host memory every step (double-buffered on a copy stream), loss read back every step"}
        del bufs

    # ---- inference render (launch_pipeline_test form) of the same views: forward only ----
    inference = None
    if not args.no_plain:
        from ray_gauss_b200.batched import render_views_inference
        for _ in range(2):
            render_views_inference(Pb, views)
        torch.cuda.synchronize()
        i0 = torch.cuda.Event(enable_timing=True)
        i1 = torch.cuda.Event(enable_timing=True)
        isteps = max(2, args.steps)
        i0.record()
        for _ in range(isteps):
            render_views_inference(Pb, views)
        i1.record()
        torch.cuda.synchronize()
        i_ms = i0.elapsed_time(i1) / isteps
        inference = {"value": round(R / (i_ms * 1e-3) / 1e6, 3), "unit": "Mrays/s", "ms_per_step": round(i_ms, 3),
                     "form": "render_views_inference: bbox + LBVH + colour + inference launch, BF16, fast arithmetic"}

    # ---- plain FP32 single-view drop-in form on the same views ----
    plain = None
    if not args.no_plain:
        Pp = {k: v.clone().requires_grad_(True) for k, v in P32.items()}
        tviews = [target[views.offsets[v]:views.offsets[v + 1]] for v in range(V)]

        def step_plain():
            for v, cam in enumerate(cams):
                s = RenderOptixSettings(eng, False, None, None, None, None, None, cam, 1024, nsg, 0, 0, 0, (1, 1),
                                        white, None, mode="parity")
                img = RenderOptixFunction.apply(Pp["positions"], Pp["scales"], Pp["quaternions"], Pp["densities"],
                                                Pp["color_features"], Pp["sph_gauss_features"],
                                                Pp["bandwidth_sharpness"], Pp["lobe_axis"], s)
                loss = torch.nn.functional.mse_loss(img, tviews[v])
                loss.backward()

        step_plain()
        torch.cuda.synchronize()
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        psteps = max(1, args.steps // 2)
        p0.record()
        for _ in range(psteps):
            zero(Pp)
            step_plain()
        p1.record()
        torch.cuda.synchronize()
        p_ms = p0.elapsed_time(p1) / psteps
        plain = {"value": round(R / (p_ms * 1e-3) / 1e6, 3), "unit": "Mrays/s", "ms_per_step": round(p_ms, 3),
                 "form": "RenderOptixFunction per view, FP32 storage, parity arithmetic"}

    # ---- attribution of batched_over_plain: arithmetic, storage and batching one at a time ----
    attribution = None
    bounded = None
    if not args.no_plain:
        tviews = [target[views.offsets[v]:views.offsets[v + 1]] for v in range(V)]

        def per_view_step(P, mode):
            def run():
                for v, cam in enumerate(cams):
                    s = RenderOptixSettings(eng, False, None, None, None, None, None, cam, 1024, nsg, 0, 0, 0,
                                            (1, 1), white, None, mode=mode)
                    img = RenderOptixFunction.apply(*(P[k] for k in GRAD_KEYS), s)
                    torch.nn.functional.mse_loss(img, tviews[v]).backward()
            return run

        def batched_step(P, bviews, tgt):
            def run():
                out = BatchedRenderFunction.apply(*(P[k] for k in GRAD_KEYS), bviews)
                torch.nn.functional.mse_loss(out, tgt).backward()
            return run

        def timed(run, P, reps):
            zero(P)
            run()
            torch.cuda.synchronize()
            a0 = torch.cuda.Event(enable_timing=True)
            a1 = torch.cuda.Event(enable_timing=True)
            a0.record()
            for _ in range(reps):
                zero(P)
                run()
            a1.record()
            torch.cuda.synchronize()
            return a0.elapsed_time(a1) / reps

        reps = max(1, args.steps // 2)
        L32 = {k: v.clone().requires_grad_(True) for k, v in P32.items()}
        Lb = {k: v.clone().requires_grad_(True) for k, v in Pb.items()}
        bviews32 = BatchedViews(cams, white_background=white, mode="fast", engine=eng)
        legs = [("single_view_parity_fp32", per_view_step(L32, "parity"), L32),
                ("single_view_fast_fp32", per_view_step(L32, "fast"), L32),
                ("single_view_fast_bf16", per_view_step(Lb, "fast"), Lb),
                ("batched_fast_fp32", batched_step(L32, bviews32, target), L32),
                ("batched_fast_bf16", batched_step(Lb, views, target), Lb)]
        attribution = {}
        for name, run, P in legs:
            a_ms = timed(run, P, reps)
            attribution[name] = {"value": round(R / (a_ms * 1e-3) / 1e6, 3), "unit": "Mrays/s",
                                 "ms_per_step": round(a_ms, 3)}
        attribution["note"] = ("fwd+bwd of the same 16 views, one factor changed per line: arithmetic (parity -> "
                               "fast), storage (FP32 -> BF16), launch (one view per launch -> all views in one "
                               "launch)")
        del L32, Lb, bviews32

        # ---- the bounded-object configuration: 300k Gaussians on shells, SH3 + 8 SG, one 800x800 view ----
        from ray_gauss_b200 import synthetic as S
        pb, bcams, bwhite = S.workload("bounded_object", seed=0, device="cpu")
        bcam = bcams[0].to(dev)
        B32 = {k: v.to(dev).requires_grad_(True) for k, v in pb.items()}
        Bb = _bf16({k: v.detach() for k, v in B32.items()})
        Bb = {k: v.clone().requires_grad_(True) for k, v in Bb.items()}
        bR = bcam.image_width * bcam.image_height
        btgt = torch.rand((bR, 3), device=dev, generator=torch.Generator(device=dev).manual_seed(3))
        bounded = {"workload": "bounded_object: 300k Gaussians on 8 seeded shells, SH3 + 8 SG, one 800x800 view, "
                               "white background", "rays_per_step": bR}
        for name, P, mode in (("parity_fp32", B32, "parity"), ("fast_fp32", B32, "fast"), ("fast_bf16", Bb, "fast")):
            def run(P=P, mode=mode):
                s = RenderOptixSettings(eng, False, None, None, None, None, None, bcam, 1024, 8, 0, 0, 0, (1, 1),
                                        bwhite, None, mode=mode)
                img = RenderOptixFunction.apply(*(P[k] for k in GRAD_KEYS), s)
                torch.nn.functional.mse_loss(img, btgt).backward()
            b_ms = timed(run, P, max(2, args.steps))
            bounded[name] = {"value": round(bR / (b_ms * 1e-3) / 1e6, 3), "unit": "Mrays/s",
                             "ms_per_step": round(b_ms, 3)}
        del B32, Bb

    # ---- accuracy of the headline form: PSNR against the FP64 oracle on 64x64 crops (reported) ----
    accuracy = None
    cpu_baseline = None
    if rank == 0 and not args.no_cpu:
        accuracy, cpu_baseline = _host_side(args, p_host, cams, white, views, leaves, Pb, eng)

    drift = _drift_leg(args, dev) if args.drift > 0 and rank == 0 else None

    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_max, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{WORKLOAD}: {n} Gaussians (80% unit ball, 20% log-uniform radius 1-50), SH3 + "
                               f"{nsg} SG, {V} views 400x300..1600x1200, batched one launch, BF16-stored "
                               "density/SH/SG, fast arithmetic",
                   "gaussians": n, "views": V, "rays_per_step": R, "storage": "bf16", "arith": "f32",
                   "parallelism": f"replicas{world}", "l2": "inputs larger than L2 (no flush)"},
        "e2e": e2e, "gpu_launches": int(launches // max(1, args.steps)) * args.steps,
        "gpu_launches_per_step": int(launches // max(1, args.steps)),
        "roofline": roofline,
        "step_roofline": {"algorithmic_bytes": int(b_step), "achieved_gbs": round(b_step / (ms_max * 1e-3) / 1e9, 2),
                          "frac": round(b_step / (ms_max * 1e-3) / 1e9 / peak, 5)},
        "stage_ms": {"prepare(bbox+bvh+colour)": round(prep_ms, 3), "forward": round(fwd_ms, 3),
                     "backward": round(bwd_ms, 3), "backward_sh": round(shb_ms, 3)},
        "counters_per_step": {k: (v if k == "record_words" else v // max(1, args.steps)) for k, v in st.items()},
        "tuning": {k: v for k, v in tuning.items() if k != "ms"},
        "graph_replay": graph,
        "train_step": train,
        "forward_only": {"value": round(R / (fwd_ms * 1e-3) / 1e6, 3), "unit": "Mrays/s",
                         "ms_per_launch": round(fwd_ms, 3), "form": "the headline step's forward launch"},
        "hit_samples": {"value": round(8 * st.get("hit_pairs", 0) / max(1, args.steps) / (ms_max * 1e-3) / 1e9, 3),
                        "unit": "G hit-samples/s", "form": "8 samples per (ray, slab, Gaussian) pair, forward + "
                                                          "backward recompute, per step time"},
        "inference": inference,
        "plain_fp32_single_view": plain,
        "batched_over_plain": round(value / world / plain["value"], 3) if plain else None,
        "batched_over_plain_attribution": attribution,
        "bounded_object": bounded,
        "accuracy": accuracy,
        "refit_drift": drift,
        "cpu_baseline": cpu_baseline,
        "clocks": clk,
    }
    print(json.dumps(line))
    return 0


def _drift_leg(args, dev):
    """Refit-only LBVH drift: the captured training iteration (GraphedStep with the fused Adam tail,
    the reference's base learning rates, positions scaled by the cameras' extent as in
    scripts/train.py:46-47) refits the tree built at capture time, while the reference rebuilds its
    GAS every iteration.  At a few iterations, the forward's node visits and time on the refitted
    tree are compared with those on a tree rebuilt from the same parameters (a second engine)."""
    import torch
    from ray_gauss_b200 import synthetic as S
    from ray_gauss_b200.batched import BatchedRenderFunction, BatchedViews
    from ray_gauss_b200.engine import Engine
    from ray_gauss_b200.graph import GraphedStep
    from ray_gauss_b200.train_tail import FusedTrainTail, LrSchedule, point_cloud_data, raw_from_render_inputs
    p, cams, white = S.workload(WORKLOAD, seed=0, device="cpu", n=args.n)
    cams = [c.to(dev) for c in cams[:4]]
    centres = np.stack([c.camera_center.cpu().numpy() for c in cams])
    extent = 1.1 * float(np.linalg.norm(centres - centres.mean(0), axis=1).max())
    raw = {k: v.to(dev).contiguous() for k, v in raw_from_render_inputs({k: v for k, v in p.items()}).items()}
    trained = {k: v for k, v in raw.items() if v.numel()}
    exp = LrSchedule.exponential
    sched = {"positions": exp(1.7e-5 * extent, 1e-6 * extent, 30000), "densities": exp(0.5, 1e-4, 30000),
             "rgb": LrSchedule(1e-3), "spherical_harmonics": LrSchedule(2.6e-4), "scales": LrSchedule(0.0115),
             "quaternions": LrSchedule(2.2e-4), "sph_gauss_features": LrSchedule(3.6e-4),
             "bandwidth_sharpness": LrSchedule(0.045), "lobe_axis": LrSchedule(0.003)}
    tail = FusedTrainTail(trained, {k: sched[k] for k in trained},
                          roles={"positions": "positions", "densities": "densities", "scales": "scales",
                                 "quaternions": "quaternions"})
    eng = Engine(dev.index or 0)
    views = BatchedViews(cams, white_background=white, mode="fast", engine=eng)
    target = torch.rand((views.n_rays, 3), device=dev, generator=torch.Generator(device=dev).manual_seed(9))
    act = lambda r: point_cloud_data(r, normalized_quaternion=False)  # noqa: E731
    step = GraphedStep(raw, views, target, tail=tail, min_scale=torch.full((raw["positions"].shape[0],), -12.0,
                                                                             device=dev), activation=act)
    fresh = Engine(dev.index or 0)
    fviews = BatchedViews(cams, white_background=white, mode="fast", engine=fresh)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def forward_stats(e, v, refit):
        v.update = refit
        e.set_tuning(diagnostics=1)
        e.status(reset=True)
        with torch.no_grad():
            X = act(raw)
            BatchedRenderFunction.apply(*(X[k] for k in GRAD_KEYS), v)
        torch.cuda.synchronize()
        visits = e.status(reset=True)["node_visits"]
        e.set_tuning(diagnostics=0)
        with torch.no_grad():
            X = act(raw)
            e0.record()
            BatchedRenderFunction.apply(*(X[k] for k in GRAD_KEYS), v)
            e1.record()
        torch.cuda.synchronize()
        return int(visits), round(e0.elapsed_time(e1), 3)

    marks = sorted({1, max(1, args.drift // 3), args.drift})
    out = {"iterations": args.drift, "views": len(cams), "gaussians": int(raw["positions"].shape[0]),
           "cameras_extent": round(extent, 3), "points": []}
    done = 0
    for m in marks:
        while done < m:
            step.replay()
            done += 1
        torch.cuda.synchronize()
        e0.record()
        for _ in range(3):
            step.replay()
        e1.record()
        torch.cuda.synchronize()
        done += 3
        replay_ms = e0.elapsed_time(e1) / 3
        v_refit, f_refit = forward_stats(eng, views, True)
        v_build, f_build = forward_stats(fresh, fviews, False)
        out["points"].append({"iteration": done, "replay_ms": round(replay_ms, 3),
                              "forward_node_visits_refit": v_refit, "forward_node_visits_rebuilt": v_build,
                              "visits_refit_over_rebuilt": round(v_refit / max(1, v_build), 4),
                              "forward_ms_refit": f_refit, "forward_ms_rebuilt": f_build})
    views.update = False
    return out


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


GRAD_KEYS = ("positions", "scales", "quaternions", "densities", "color_features", "sph_gauss_features",
             "bandwidth_sharpness", "lobe_axis")


def _oracle_rays(O, P, cv, W, H, white, ids, dL, prec):
    """Oracle image of the rays `ids` of one view and every parameter gradient of sum(image * dL)."""
    rgb = O.forward_sh(cv[:3], P["positions"], P["color_features"], P["sph_gauss_features"],
                       P["bandwidth_sharpness"], P["lobe_axis"], prec=prec)
    aabb, box = O.bbox(P["positions"], P["scales"], P["quaternions"], P["densities"], prec)
    img, _, _ = O.render_forward(P["positions"], P["scales"], P["quaternions"], P["densities"], rgb, cv, W, H, white,
                                 ray_ids=ids, aabb=aabb, scene_box=box, prec=prec)
    g = O.render_backward(P["positions"], P["scales"], P["quaternions"], P["densities"], rgb, cv, W, H, img, dL,
                          ray_ids=ids, aabb=aabb, scene_box=box, prec=prec)
    dt = np.float64 if prec == "f64" else np.float32
    dsh, dpos, dsg, dkap, dax = O.backward_sh(cv[:3], P["positions"], P["color_features"], P["sph_gauss_features"],
                                              P["bandwidth_sharpness"], P["lobe_axis"], g["d_rgb"].astype(dt),
                                              prec=prec, ref_quirks=True)
    grads = dict(positions=g["d_pos"] + dpos, scales=g["d_scl"], quaternions=g["d_quat"], densities=g["d_dens"],
                 color_features=dsh, sph_gauss_features=dsg, bandwidth_sharpness=dkap, lobe_axis=dax)
    return img, grads


def _rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def _psnr(a, b, digits=2):
    mse = float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))
    return 99.0 if mse == 0 else round(-10 * math.log10(mse), digits)


def _host_side(args, p_host, cams, white, views, leaves, Pb, eng):
    """Accuracy of the benchmarked form against the FP64 oracle, and the host-core baseline.

    Rays: 4096 seeded random rays of each of views 0 and 1.  The headline form (BF16 storage, fast
    arithmetic, all views in one launch) renders the whole batch; the loss gradient is non-zero only
    on the sampled rays, so its FP32 parameter gradients (read from the engine, before autograd
    casts them to the BF16 leaves' dtype) are sums over those rays and the oracle computes them from
    the same rays.  References: the FP64 oracle of the BF16-rounded parameters (the arithmetic's
    error) and of the FP32 parameters (storage rounding included).  The baseline times the FP32 C
    restatement, with its grid candidate prefilter, over the same rays on all host cores."""
    import torch
    from oracle import oracle as O
    from ray_gauss_b200 import _lib
    from ray_gauss_b200.engine import make_gaussians, settings_struct
    rng = np.random.default_rng(7)
    V = len(cams)
    n_views = min(2, V)
    rays = args.cpu_rays
    R = views.n_rays
    ids = []
    for v in range(n_views):
        W, H = cams[v].image_width, cams[v].image_height
        ids.append(np.sort(rng.choice(W * H, min(rays, W * H), replace=False)).astype(np.int32))
    dLs = [rng.normal(0.0, 1e-3, (len(i), 3)).astype(np.float32) for i in ids]
    # the benchmarked form through the engine: FP32 gradients of the sampled rays' loss
    g = make_gaussians(*(Pb[k] for k in GRAD_KEYS))
    cams_t, _, _ = eng.cameras(views.cameras, views.supersampling)
    st = settings_struct(white, mode=_lib.RG_MODE_FAST)
    with torch.no_grad():
        out, _ = eng.render_forward(g, cams_t, V, R, st)
        dL = torch.zeros((R, 3), dtype=torch.float32, device=out.device)
        for v in range(n_views):
            idx = torch.from_numpy(ids[v].astype(np.int64) + int(views.offsets[v])).to(out.device)
            dL[idx] = torch.from_numpy(dLs[v]).to(out.device)
        gr = eng.render_backward(g, cams_t, V, st, out, dL)
        torch.cuda.synchronize()
    gpu_img = out.cpu().numpy()
    gpu_g = {k: gr[k].cpu().numpy() for k in GRAD_KEYS}
    P_round = {k: v.double().cpu().numpy() for k, v in Pb.items()}                 # BF16-rounded
    P_full = {k: np.asarray(v, np.float64) for k, v in p_host.items()}              # FP32 parameters
    P32 = {k: np.asarray(v, np.float32) for k, v in p_host.items()}
    acc = {"rays_per_view": int(rays), "views": n_views, "form": "BF16 storage, fast arithmetic, batched launch",
           "images": []}
    sums = {"round": {k: 0.0 for k in GRAD_KEYS}, "full": {k: 0.0 for k in GRAD_KEYS}}
    t_cpu, rays_cpu = 0.0, 0
    for v in range(n_views):
        cam = cams[v]
        W, H = cam.image_width, cam.image_height
        cv = O.camera_vector(cam)
        img_r, g_r = _oracle_rays(O, P_round, cv, W, H, white, ids[v], dLs[v], "f64")
        img_f, g_f = _oracle_rays(O, P_full, cv, W, H, white, ids[v], dLs[v], "f64")
        for k in GRAD_KEYS:
            sums["round"][k] = sums["round"][k] + g_r[k]
            sums["full"][k] = sums["full"][k] + g_f[k]
        gi = gpu_img[int(views.offsets[v]) + ids[v]]
        # PSNR against a training-like target (the FP64 image of the FP32 parameters plus seeded
        # noise of sd 0.03, about 30 dB): the benchmarked form's against the FP64 oracle's
        target = img_f + rng.normal(0.0, 0.03, img_f.shape)
        p_form, p_orc = _psnr(gi, target, 4), _psnr(img_f, target, 4)
        acc["images"].append({"view": v, "psnr_vs_fp64_of_bf16_params_db": _psnr(gi, img_r),
                              "max_abs_vs_fp64_of_bf16_params": float(np.abs(gi - img_r).max()),
                              "psnr_vs_fp64_of_fp32_params_db": _psnr(gi, img_f),
                              "max_abs_vs_fp64_of_fp32_params": float(np.abs(gi - img_f).max()),
                              "target_psnr_db": {"form": p_form, "fp64_oracle": p_orc,
                                                 "delta": round(abs(p_form - p_orc), 4)}})
        # host-core baseline: the FP32 restatement over the same rays (grid build included)
        t = time.perf_counter()
        _oracle_rays(O, P32, cv, W, H, white, ids[v], dLs[v], "f32")
        t_cpu += time.perf_counter() - t
        rays_cpu += len(ids[v])
    acc["grad_rel_l2_vs_fp64_of_bf16_params"] = {k: _rel_l2(gpu_g[k], sums["round"][k]) for k in GRAD_KEYS}
    acc["grad_rel_l2_vs_fp64_of_fp32_params"] = {k: _rel_l2(gpu_g[k], sums["full"][k]) for k in GRAD_KEYS}
    acc["grad_rel_l2_max_vs_fp64_of_bf16_params"] = max(acc["grad_rel_l2_vs_fp64_of_bf16_params"].values())
    acc["psnr_delta_db_max"] = max(im["target_psnr_db"]["delta"] for im in acc["images"])
    threads = O.num_threads()
    cpu = {"value": round(rays_cpu / t_cpu / 1e6, 6), "unit": "Mrays/s", "cores": threads, "kind": "port",
           "cpu_model": _cpu_model(),
           "sample": f"{rays_cpu} seeded random rays ({rays} per view, views 0-{n_views - 1}) of the 1M-Gaussian "
                     "workload, FP32 forward+backward (SH/SG, bbox, render, adjoint) with the C restatement on "
                     f"{threads} OpenMP threads; ray candidates from a nested uniform grid over the AABBs (built "
                     "per call, included) and a per-ray slab sweep"}
    return acc, cpu


def reference_arm(args, rank, world):
    """The reference's own CPU implementation of the path on the host cores: its training device
    programs (cuda_train/forward and backward gaussians_aabb.cu, utils/sh_utils.cu) compiled for the
    CPU under oracle/_ref when that build is present, otherwise the C restatement; bounded sample of
    rays per step, same metric and unit."""
    if rank != 0:
        return 0
    from oracle import oracle as O
    from ray_gauss_b200 import synthetic as S
    p, cams, white = S.workload(WORKLOAD, seed=0, device="cpu", n=args.n)
    cams = cams[: args.views]
    Pn = {k: v.numpy().astype(np.float32) for k, v in p.items()}
    use_ref = O.ref_available()
    rng = np.random.default_rng(3)
    rays = max(64, args.cpu_rays // 2)   # per step: about 2-4 s on 8-16 host cores
    prepared = []
    for cam in cams[:2]:
        cv = O.camera_vector(cam)
        sh = (Pn["color_features"], Pn["sph_gauss_features"], Pn["bandwidth_sharpness"], Pn["lobe_axis"])
        rgb = O.ref_forward_sh(cv[:3], Pn["positions"], *sh) if use_ref else O.forward_sh(cv[:3], Pn["positions"], *sh)
        aabb, box = O.bbox(Pn["positions"], Pn["scales"], Pn["quaternions"], Pn["densities"], "f32")
        prepared.append((cam, cv, rgb, aabb, box))
    times = []
    for s in range(args.warmup + args.steps):
        cam, cv, rgb, aabb, box = prepared[s % len(prepared)]
        W, H = cam.image_width, cam.image_height
        ids = rng.integers(0, W * H, rays).astype(np.int32)
        t = time.perf_counter()
        if use_ref:
            img, _ = O.ref_render_forward(Pn["positions"], Pn["scales"], Pn["quaternions"], Pn["densities"], rgb, cv,
                                          W, H, white, aabb=aabb, scene_box=box, ray_ids=ids)
            dL = np.zeros_like(img)
            dL[ids] = 1e-3
            O.ref_render_backward(Pn["positions"], Pn["scales"], Pn["quaternions"], Pn["densities"], rgb, cv, W, H,
                                  img, dL, aabb=aabb, scene_box=box, ray_ids=ids)
        else:
            img, _, _ = O.render_forward(Pn["positions"], Pn["scales"], Pn["quaternions"], Pn["densities"], rgb, cv,
                                         W, H, white, ray_ids=ids, aabb=aabb, scene_box=box, prec="f32")
            O.render_backward(Pn["positions"], Pn["scales"], Pn["quaternions"], Pn["densities"], rgb, cv, W, H, img,
                              np.full(img.shape, 1e-3, np.float32), ray_ids=ids, aabb=aabb, scene_box=box,
                              prec="f32")
        if s >= args.warmup:
            times.append(time.perf_counter() - t)
    ms = statistics.mean(times) * 1e3
    value = rays / (ms * 1e-3) / 1e6
    kind = "reference" if use_ref else "port"
    what = ("the reference's training device programs compiled for the CPU (oracle/_ref); each optixTrace "
            "call finds its primitives through a nested uniform grid over the AABBs, built per launch like the "
            "reference's per-iteration GAS build" if use_ref else
            "the C restatement (oracle/liboracle.so) with its grid candidate prefilter")
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 6), "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{WORKLOAD}: {args.n} Gaussians, views 0-1, {rays} random rays per step, "
                                   "FP32 forward+backward on host cores"},
            "cpu_baseline": {"value": round(value, 6), "unit": "Mrays/s", "cores": O.num_threads(), "kind": kind,
                             "cpu_model": _cpu_model(),
                             "sample": f"{rays} random rays of view 0 or 1 per step, forward+backward, {what}"},
            "e2e": {"value": round(value, 6), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
