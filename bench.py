"""Benchmark of the B200 rmeshvk tiled training step.

Workload (one "step"): the batched configuration of the reference's benchmark
set -- a Delaunay mesh of 100,000 points from an 8-component Gaussian mixture
(~650k tets), 16 cameras on a sphere of radius U[2.5, 4] with resolutions drawn
from {256^2, 512^2, 800x600, 1024^2}; one step renders all 16 views, computes
the L2 loss against seeded targets, back-propagates and applies one Adam update
(forward + backward + Adam).  Synthetic, seeded data.  Colours are degree-3
spherical harmonics (the benchmark's sh_degree 3), evaluated per view with the
reference shader's formula and trained with lr_sh 2.5e-3; ``--sh-degree -1``
selects the reference binding's base-colour training path instead.

Line printed by rank 0 (one JSON object):
  value          train-steps/s of the batched, graph-captured path, inputs in HBM
  e2e            same metric through the public API with the targets in pinned
                 host memory copied every step (double-buffered on a copy
                 stream: step i+1's upload runs under step i's kernels) and
                 the losses read back
  plain          train-steps/s of the one-view-per-launch path on the same step
  roofline       dominant kernel (fused forward+loss+adjoint compositing):
                 algorithmic bytes / measured launch time vs measured HBM peak
  issue_roofline the same kernel against its real ceiling, instruction issue
  cpu_baseline   the CPU oracle (C port of the reference kernels) on all host
                 cores, timed on a sample of the step and scaled to the metric

``--impl reference`` times the CPU port of the reference's kernels instead (the
reference itself is a wgpu/Vulkan program that cannot run on this machine).
Multi-GPU (torchrun): every rank trains its own 16 views (weak scaling) and
the ranks' gradients are summed before Adam.
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

RES = ((256, 256), (512, 512), (800, 600), (1024, 1024))
N_VIEWS = 16
LR = dict(lr_verts=1e-4, lr_dens=1e-2, lr_grads=1e-3)
LR_SH = 2.5e-3
# DRAM bytes (read + write) per (tile, tet) pair of the fused compositing
# kernel, from a one-kernel ncu capture of a 4-view case of this workload's
# mesh and resolution mix (bench.py --views 4: 8.13 M pairs,
# dram__bytes_read.sum + dram__bytes_write.sum = 2.907 GB); the roofline's
# "traffic" scales it to the run's pair count.
TILE_DRAM_BYTES_PER_PAIR = 358.0
# Warp instructions per (tile, tet) pair of the same kernel, from the same
# capture (smsp__inst_executed.sum = 9.408 G); the issue ceiling is 148 SMs x
# 4 schedulers x one instruction per clock.
TILE_WARP_INST_PER_PAIR = 1157.0


def issue_roofline(n_pairs: int, launch_ms: float, sm_mhz) -> dict:
    """The tile kernel's bound in practice: instruction issue, not HBM."""
    mhz = float(sm_mhz) if sm_mhz else 1965.0
    peak = 148 * 4 * mhz * 1e6 / 1e12
    achieved = TILE_WARP_INST_PER_PAIR * n_pairs / (launch_ms * 1e-3) / 1e12
    return {"achieved": round(achieved, 4), "peak": round(peak, 4), "unit": "T warp-instructions/s",
            "frac": round(achieved / peak, 4),
            "basis": f"{TILE_WARP_INST_PER_PAIR:.0f} warp instructions per pair (ncu) x pairs / launch time; "
                     f"peak 148 SMs x 4 schedulers x {mhz:.0f} MHz"}


def res_text(res) -> str:
    return ",".join(f"{w}^2" if w == h else f"{w}x{h}" for w, h in res)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def build_workload(points: int, seed: int, rank: int, n_views: int = N_VIEWS, res=RES, sh_degree: int = 3,
                   cloud: str = "gmm"):
    from rmesh_b200.camera import orbit_cameras
    from rmesh_b200.scenes import gmm_cloud, make_scene, shell_cloud, uniform_cloud

    rng = np.random.default_rng(seed)
    if cloud == "gmm":
        pts = gmm_cloud(points, rng)
    else:  # uniform in [-1,1]^3 plus 10 % jittered near a random sphere shell
        pts = np.concatenate([uniform_cloud(points, rng), shell_cloud(points // 10, rng)], axis=0)
    scene = make_scene(pts, rng, sh_degree=max(sh_degree, 0))
    cams = orbit_cameras(n_views, seed=seed + 1 + 1000 * rank, radius=(2.5, 4.0), resolutions=res)
    trng = np.random.default_rng(seed + 2 + 1000 * rank)
    gts = [trng.uniform(0, 1, (c.height, c.width, 3)).astype(np.float32) for c in cams]
    return scene, cams, gts


def build_training(args):
    """Training-loop workload: a seeded GMM teacher mesh with randomised SH
    colours and densities, ``args.targets`` target cameras, one held-out camera,
    and the student: the teacher perturbed (SH + N(0, 0.3), log-density +
    N(0, 0.5), vertices + N(0, 0.01)) on the same topology."""
    from rmesh_b200.camera import orbit_cameras
    from rmesh_b200.scenes import gmm_cloud, make_scene

    rng = np.random.default_rng(args.seed)
    teacher = make_scene(gmm_cloud(args.points, rng), rng, sh_degree=args.sh_degree)
    cams = orbit_cameras(args.targets, seed=args.seed + 1, radius=(2.5, 4.0), resolutions=args.res)
    hold = orbit_cameras(1, seed=args.seed + 99, radius=(3.0, 3.0), resolutions=args.res)[0]
    prng = np.random.default_rng(args.seed + 2)
    student = dict(teacher)
    student["sh_coeffs"] = (teacher["sh_coeffs"] + prng.normal(0, 0.3, teacher["sh_coeffs"].shape)).astype(np.float32)
    student["densities"] = np.exp(np.log(teacher["densities"]) + prng.normal(0, 0.5, teacher["densities"].shape)
                                  ).astype(np.float32)
    student["vertices"] = (teacher["vertices"] + prng.normal(0, 0.01, teacher["vertices"].shape)).astype(np.float32)
    return teacher, student, cams, hold


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, gpu_index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={gpu_index}", f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.f:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.f.name)
        load = [s for s in sm if s > 0.5 * max(sm)] if sm else []
        return {"sm_mhz": float(np.median(load)) if load else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_bytes(n_pairs: int, n_pix: int, N: int, M: int) -> int:
    """Unique traffic of the fused forward+loss+adjoint compositing kernel:
    both passes read each (tile, tet) slot (4 B) and its tet record (64 B) plus
    colour (16 B); per pixel the 12 B target; gradients 80 B per tet slot."""
    rec = 4 + 64 + 16
    return 2 * n_pairs * rec + 12 * n_pix + 80 * M


def run_gpu(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from rmesh_b200 import RMeshRenderer, TargetStager
    from rmesh_b200 import _lib

    scene, cams, gts = build_workload(args.points, args.seed, rank, args.views, args.res, args.sh_degree, args.cloud)
    sh_kw = dict(sh_coeffs=scene["sh_coeffs"], sh_degree=args.sh_degree) if args.sh_degree >= 0 else {}
    lr_sh = LR_SH if args.sh_degree >= 0 else 0.0
    r = RMeshRenderer(scene["vertices"], scene["indices"], scene["base_colors"], scene["densities"],
                      scene["color_grads"], scene["circumdata"], cams[0].width, cams[0].height,
                      tile_size=args.tile_size, device=local, **sh_kw)
    stream = torch.cuda.Stream(device=local)
    r.set_stream(stream.cuda_stream)
    n_pix = sum(c.width * c.height for c in cams)
    gt_host = torch.from_numpy(np.concatenate([g.ravel() for g in gts])).pin_memory()
    gt_dev = gt_host.to(f"cuda:{local}")
    torch.cuda.synchronize()

    # tile configuration (tile size x threads per tile, and per resolution)
    # picked by timing the step's forward + adjoint over the whole grid
    # (parameters unchanged); the pair-key width follows from the tile count
    tune = None if args.no_autotune else r.autotune(cams, gt_dev, loss_type=1)
    tile_size, tile_threads = r.tile_config()
    slots = r.grad_slots() if world > 1 else None

    def step(mode, gt):
        if dist is None:
            return r.train_step_views(cams, gt, loss_type=1, mode=mode, lr_sh=lr_sh, **LR)
        # data parallel: this rank's views -> sum of all ranks' gradients -> Adam
        losses = r.accumulate_views(cams, gt, loss_type=1, mode=mode)
        with torch.cuda.stream(stream):
            dist.all_reduce(slots)
        r.apply_adam(lr_sh=lr_sh, **LR)
        return losses

    stager = TargetStager(r, gt_host.numel())

    def timed(mode, gt, steps):
        """ms per step; with pinned host targets every step's upload is inside
        the timed region, step i+1's copy running under step i's kernels."""
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        staged = not gt.is_cuda
        nxt = stager.put(gt) if staged else gt  # the first copy starts after e0
        for i in range(steps):
            cur = nxt
            if staged and i + 1 < steps:
                nxt = stager.put(gt)
            step(mode, cur)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if dist is not None:
            t = torch.tensor([ms], device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms / steps

    # warm-up (also sizes the pair buffers and captures the graph)
    for mode in ("graph", "batched", "plain"):
        for _ in range(max(1, args.warmup)):
            step(mode, gt_dev)
    for _ in range(max(2, args.warmup)):  # the graphs of the two staging buffers
        step("graph", stager.put(gt_host))
    r.stage_times()  # reset counters

    clk = Clocks(local)
    ms_graph = timed("graph", gt_dev, args.steps)
    _, launches, total_launches = r.stage_times()
    ms_e2e = timed("graph", gt_host, args.steps)
    clocks = clk.stop()
    ms_plain = timed("plain", gt_dev, max(1, args.steps // 2))
    r.stage_times()

    # render only: the batched forward of the same views into a device buffer
    # (rmesh_forward_views), device-timed
    fwd_ms = None
    if dist is None:
        out_dev = torch.empty(n_pix * 4, dtype=torch.float32, device=f"cuda:{local}")

        def fwd():
            r.forward_views(cams, out=out_dev)

        for _ in range(2):
            fwd()
        torch.cuda.synchronize()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(5):
            fwd()
        f1.record(stream)
        f1.synchronize()
        fwd_ms = f0.elapsed_time(f1) / 5

    # per-stage device times of the batched path (CUDA events on the library stream)
    r.set_profiling(True)
    for _ in range(max(1, args.steps // 2)):
        step("batched", gt_dev)
    stage_ms, stage_n, _ = r.stage_times()
    r.set_profiling(False)
    nsteps_prof = max(1, args.steps // 2)
    info = r.info()
    comp_ms = stage_ms["composite"] / max(stage_n["composite"], 1)
    alg = algorithmic_bytes(int(info.n_pairs_last), n_pix, r.n_vertices, r.n_tets)
    peak, peak_kind = peaks()
    achieved = alg / (comp_ms * 1e-3) / 1e9

    steps_per_s = world * 1000.0 / ms_graph
    out = {
        "metric": metric_name(args),
        "value": round(steps_per_s, 4),
        "unit": "train-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_graph, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded Delaunay mesh, seeded targets)",
        "config": {**workload_config(args, r.n_tets, r.n_vertices, n_pix, world), "tile_size": tile_size,
                   "threads_per_tile": tile_threads, "autotune": tune},
        "mpix_per_s": round(world * n_pix / (ms_graph * 1e-3) / 1e6, 2),
        "plain": {"value": round(world * 1000.0 / ms_plain, 4), "unit": "train-steps/s", "ms_per_step": round(ms_plain, 4)},
        "batched_graph_vs_plain": round(ms_plain / ms_graph, 3),
        "forward_only": None if fwd_ms is None else {
            "ms_per_render": round(fwd_ms, 4), "mpix_per_s": round(n_pix / (fwd_ms * 1e-3) / 1e6, 2),
            "what": "batched forward of the same views (rmesh_forward_views) into device memory"},
        "e2e": {"value": round(world * 1000.0 / ms_e2e, 4), "unit": "train-steps/s",
                "h2d_bytes_per_step": int(n_pix * 12 + args.views * 160 + 48),
                "d2h_bytes_per_step": int(_lib.COUNTERS_BYTES)},
        "gpu_launches": int(total_launches),
        "device_memory_gb": round(int(info.device_bytes) / 1e9, 2),
        "stage_ms_per_step": {k: round(v / nsteps_prof, 4) for k, v in stage_ms.items()},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4),
                     "traffic": int(TILE_DRAM_BYTES_PER_PAIR * int(info.n_pairs_last)),
                     "kernel": f"tile_kernel<{tile_size},kModeTrain> (fused forward+loss+adjoint, "
                               f"{tile_threads} threads per tile)",
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else
                     "fallback 6.65 TB/s", "launch_ms": round(comp_ms, 4), "algorithmic_bytes": alg,
                     "n_pairs": int(info.n_pairs_last)},
        "issue_roofline": issue_roofline(int(info.n_pairs_last), comp_ms, clocks.get("sm_mhz")),
        "clocks": clocks,
    }
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(scene, cams, gts, args)
    if rank == 0 and not args.no_parity_check:
        out["parity_check"] = parity_check(scene, cams, gts, args, local)
        out["grad_relerr"] = out["parity_check"]["grad_relerr_max"]
    if rank == 0:
        print(json.dumps(out), flush=True)
    r.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def metric_name(args) -> str:
    if args.workload == "training":
        return (f"fwd+bwd train-steps/s (training loop: {args.views} of {args.targets} {res_text(args.res)} "
                f"teacher views per graph-captured step)")
    return (f"fwd+bwd train-steps/s ({args.views} views, batched graph-captured step)" if args.workload == "large"
            else "fwd+bwd train-steps/s (16 mixed-resolution views, batched graph-captured step)")


def workload_config(args, n_tets, n_vertices, n_pix, world):
    """The config object of the JSON line (both arms)."""
    mesh = ("8-component GMM" if args.cloud == "gmm" else
            f"uniform [-1,1]^3 + {args.points // 10}-point sphere-shell")
    if args.workload == "training":
        text = (f"training: {args.points}-point {mesh} teacher/student Delaunay mesh ({n_tets} tets), "
                f"{args.targets} target views at {res_text(args.res)}, {args.views} per step in fixed batches, "
                f"{args.steps} steps, L2 loss, Adam (lr_sh {LR_SH}, lr_verts {LR['lr_verts']}, "
                f"lr_dens {LR['lr_dens']}, lr_grads {LR['lr_grads']})")
    else:
        text = (f"{args.workload}: {args.points}-point {mesh} Delaunay mesh ({n_tets} tets), "
                f"{args.views} views from {{{res_text(args.res)}}}, L2 loss, Adam")
    return {
        "workload": text,
        "n_tets": n_tets, "n_vertices": n_vertices, "views_per_gpu": args.views,
        "pixels_per_step_per_gpu": n_pix, "tile_size": args.tile_size,
        "color_mode": f"sh_degree {args.sh_degree}" if args.sh_degree >= 0 else "base_colors",
        "parallelism": f"dp{world} (views sharded, gradients summed)" if world > 1 else "single GPU",
        "l2": "inputs larger than L2 (mesh records + pair lists > 126 MB per step)",
    }


def _oracle_sh(o, scene, args):
    """The oracle's SH inputs for the workload's colour mode."""
    if args.sh_degree < 0:
        return None, 0
    return o.sh_values(scene["sh_coeffs"]), args.sh_degree


def cpu_baseline(scene, cams, gts, args, budget_s=20.0):
    """The oracle's train step (project, emit, sort, ranges, rasterize, loss,
    adjoint, Adam) on all host cores for views of the step until ~budget_s,
    scaled by pixels to a full step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle

    o = Oracle("f32")
    threads = o.max_threads
    shv, deg = _oracle_sh(o, scene, args)
    # cheapest views first so the sample covers several views within the budget
    order = sorted(range(len(cams)), key=lambda i: cams[i].width * cams[i].height)
    t0 = time.perf_counter()
    px_done, views_done = 0, 0
    for i in order:
        cam, gt = cams[i], gts[i]
        fwd = o.forward_tiled(scene, cam, args.tile_size, sh=shv, sh_degree=deg)
        _, dl = o.loss(fwd["image"], gt, 1)
        o.backward(scene, cam, dl, fwd, args.tile_size, threads=threads, sh=shv, sh_degree=deg)
        px_done += cam.width * cam.height
        views_done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    n_pix = sum(c.width * c.height for c in cams)
    t_step = dt * n_pix / px_done
    return {"value": round(1.0 / t_step, 6), "unit": "train-steps/s", "cores": threads, "kind": "port",
            "sample": f"{views_done} of {len(cams)} views ({px_done} px) in {dt:.1f} s, scaled by pixels "
                      f"to the {n_pix}-px step; C oracle, OpenMP {threads} threads",
            "mpix_per_s": round(px_done / dt / 1e6, 4)}


def parity_check(scene, cams, gts, args, device):
    """Outside the timed region: one of the step's views (the first 800x600
    one, else the largest) rendered and back-propagated by the library from
    the workload's initial parameters, against the CPU oracle on the same
    inputs: image max-abs and relative L2 of every gradient group."""
    from rmesh_b200 import RMeshRenderer

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle

    pick = next((i for i, c in enumerate(cams) if (c.width, c.height) == (800, 600)),
                max(range(len(cams)), key=lambda i: cams[i].width * cams[i].height))
    cam, gt = cams[pick], gts[pick]
    o = Oracle("f32")
    shv, deg = _oracle_sh(o, scene, args)
    ref = o.forward_tiled(scene, cam, args.tile_size, sh=shv, sh_degree=deg)
    _, dl = o.loss(ref["image"], gt, 1)
    go = o.backward(scene, cam, dl, ref, args.tile_size, threads=o.max_threads, sh=shv, sh_degree=deg)
    sh_kw = dict(sh_coeffs=scene["sh_coeffs"], sh_degree=args.sh_degree) if args.sh_degree >= 0 else {}
    r = RMeshRenderer(scene["vertices"], scene["indices"], scene["base_colors"], scene["densities"],
                      scene["color_grads"], scene["circumdata"], cam.width, cam.height, tile_size=args.tile_size,
                      device=device, **sh_kw)
    img = r.forward_tiled(cam.cam_pos, cam.vp, cam.c2w_intrinsics)
    g = r.backward(dl)
    r.close()

    def rel(a, b):
        a = np.asarray(a, np.float64).ravel()
        b = np.asarray(b, np.float64).ravel()
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))

    pairs = [("d_vertices", "d_vertices"), ("d_densities", "d_densities"), ("d_color_grads", "d_color_grads")]
    pairs.append(("d_sh_coeffs", "d_sh") if args.sh_degree >= 0 else ("d_base_colors", "d_base_colors"))
    errs = {k: round(rel(g[k], go[ko]), 8) for k, ko in pairs}
    return {"view": f"{cam.width}x{cam.height} (view {pick} of the step)", "pairs": int(ref["P"]),
            "image_max_abs": float(np.abs(img - ref["image"]).max()), "grad_relerr": errs,
            "grad_relerr_max": max(errs.values()), "bars": "image max-abs <= 1e-4, gradient rel-L2 <= 1e-3",
            "oracle": f"C restatement of the reference kernels, OpenMP {o.max_threads} threads"}


def run_profile_step(args):
    """For profiler captures (ncu --profile-from-start off): the default
    workload's batched step, three times unprofiled, then once between
    cudaProfilerStart and cudaProfilerStop.  Prints the step's counts."""
    import torch

    from rmesh_b200 import RMeshRenderer

    torch.cuda.set_device(0)
    scene, cams, gts = build_workload(args.points, args.seed, 0, args.views, args.res, args.sh_degree, args.cloud)
    sh_kw = dict(sh_coeffs=scene["sh_coeffs"], sh_degree=args.sh_degree) if args.sh_degree >= 0 else {}
    r = RMeshRenderer(scene["vertices"], scene["indices"], scene["base_colors"], scene["densities"],
                      scene["color_grads"], scene["circumdata"], cams[0].width, cams[0].height,
                      tile_size=args.tile_size, **sh_kw)
    gt = torch.from_numpy(np.concatenate([g.ravel() for g in gts])).cuda()
    lr_sh = LR_SH if args.sh_degree >= 0 else 0.0
    for _ in range(3):
        r.train_step_views(cams, gt, loss_type=1, mode="batched", lr_sh=lr_sh, **LR)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    r.train_step_views(cams, gt, loss_type=1, mode="batched", lr_sh=lr_sh, **LR)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    inf = r.info()
    print(json.dumps({"n_visible": int(inf.n_visible_last), "n_pairs": int(inf.n_pairs_last), "n_tets": r.n_tets,
                      "n_vertices": r.n_vertices, "pixels": sum(c.width * c.height for c in cams)}), flush=True)
    r.close()


def run_training(args):
    """The training loop: the teacher renders the targets on the GPU, then a
    fresh student renderer takes ``args.steps`` graph-replayed Adam steps of
    ``args.views`` views each, cycling through the targets in fixed batches.
    The timed region is the whole loop from the unperturbed start (the first
    pass over the batches captures their CUDA graphs, inside it).  e2e repeats
    the loop on another fresh student with the targets in pinned host memory,
    uploaded each step through TargetStager; its loss trajectory must follow
    the first run's."""
    import torch

    from rmesh_b200 import RMeshRenderer, TargetStager
    from rmesh_b200 import _lib

    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        raise SystemExit("the training-loop workload runs on one GPU")
    torch.cuda.set_device(0)
    teacher, student, cams, hold = build_training(args)
    W, H = cams[0].width, cams[0].height

    def renderer(sc, tile):
        """tile: a tile size or a (tile size, threads per tile) configuration"""
        ts, th = (tile, 0) if isinstance(tile, int) else tile
        r = RMeshRenderer(sc["vertices"], sc["indices"], sc["base_colors"], sc["densities"], sc["color_grads"],
                          sc["circumdata"], W, H, tile_size=ts, sh_coeffs=sc["sh_coeffs"],
                          sh_degree=args.sh_degree)
        r.set_tile_config(ts, th)
        st = torch.cuda.Stream()
        r.set_stream(st.cuda_stream)
        return r, st

    rt, _ = renderer(teacher, args.tile_size)
    targets = [rt.forward_tiled(c.cam_pos, c.vp, c.c2w_intrinsics)[..., :3].copy() for c in cams]
    want = rt.forward_tiled(hold.cam_pos, hold.vp, hold.c2w_intrinsics)
    rt.close()
    vps = args.views
    nb = len(cams) // vps
    batches = [cams[k * vps:(k + 1) * vps] for k in range(nb)]
    host = [torch.from_numpy(np.concatenate([t.ravel() for t in targets[k * vps:(k + 1) * vps]])).pin_memory()
            for k in range(nb)]
    dev = [h.cuda() for h in host]
    n_pix = sum(c.width * c.height for c in batches[0])

    # warm-up on a disposable student: module load, allocator, tile-size autotune
    rw, _ = renderer(student, args.tile_size)
    tune = None if args.no_autotune else rw.autotune(batches[0], dev[0], loss_type=1)
    tile = rw.tile_config()
    for i in range(args.warmup):
        rw.train_step_views(batches[i % nb], dev[i % nb], loss_type=1, mode="graph", lr_sh=LR_SH, **LR)
    r0, _ = renderer(student, tile)
    before = float(np.abs(r0.forward_tiled(hold.cam_pos, hold.vp, hold.c2w_intrinsics) - want).mean())
    r0.close()
    rw.close()

    lr = dict(LR, lr_verts=LR["lr_verts"] if args.lr_verts is None else args.lr_verts)

    def loop(mode, staged, steps):
        """Returns (renderer, ms per step, per-step mean losses, per-step ms)."""
        r, st = renderer(student, tile)
        stager = TargetStager(r, host[0].numel()) if staged else None
        losses = []
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        ev[0].record(st)
        nxt = stager.put(host[0]) if staged else None
        for i in range(steps):
            k = i % nb
            if staged:
                cur = nxt
                if i + 1 < steps:
                    nxt = stager.put(host[(i + 1) % nb])
            else:
                cur = dev[k]
            losses.append(float(np.mean(r.train_step_views(batches[k], cur, loss_type=1, mode=mode, lr_sh=LR_SH,
                                                           **lr))))
            ev[i + 1].record(st)
        ev[-1].synchronize()
        per = np.array([ev[i].elapsed_time(ev[i + 1]) for i in range(steps)])
        return r, ev[0].elapsed_time(ev[-1]) / steps, np.array(losses), per

    clk = Clocks(0)
    r1, ms_graph, losses, per_step = loop("graph", False, args.steps)
    clocks = clk.stop()
    _, _, total_launches = r1.stage_times()
    after = float(np.abs(r1.forward_tiled(hold.cam_pos, hold.vp, hold.c2w_intrinsics) - want).mean())
    r1.set_profiling(True)
    for k in range(nb):
        r1.train_step_views(batches[k], dev[k], loss_type=1, mode="batched", lr_sh=LR_SH, **lr)
    stage_ms, stage_n, _ = r1.stage_times()
    r1.set_profiling(False)
    info = r1.info()
    dev_gb = int(info.device_bytes) / 1e9
    r1.close()
    r2, ms_e2e, losses_e2e, _ = loop("graph", True, args.steps)
    r2.close()
    n_plain = min(args.steps, 40)
    r3, ms_plain, _, _ = loop("plain", False, n_plain)
    r3.close()

    def diverged_at(ls):
        """First step whose mean loss is not finite or above 10x the first pass's."""
        bad = ~np.isfinite(ls) | (ls > 10.0 * ls[:nb].mean())
        return int(np.argmax(bad)) if bad.any() else None

    def fin(x):
        return round(float(x), 6) if np.isfinite(x) else None

    d1, d2 = diverged_at(losses), diverged_at(losses_e2e)
    n_ok = min(d for d in (d1, d2, args.steps) if d is not None)
    healthy = per_step[:d1] if d1 else per_step

    comp_ms = stage_ms["composite"] / max(stage_n["composite"], 1)
    n_tets, n_verts = student["indices"].size // 4, student["vertices"].size // 3
    alg = algorithmic_bytes(int(info.n_pairs_last), n_pix, n_verts, n_tets)
    peak, peak_kind = peaks()
    achieved = alg / (comp_ms * 1e-3) / 1e9
    out = {
        "metric": metric_name(args), "value": round(1000.0 / ms_graph, 4), "unit": "train-steps/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_graph, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded GMM teacher mesh renders the targets; perturbed student)",
        "config": {**workload_config(args, n_tets, n_verts, n_pix, 1), "tile_size": tile[0],
                   "threads_per_tile": tile[1], "autotune": tune},
        "mpix_per_s": round(n_pix / (ms_graph * 1e-3) / 1e6, 2),
        "plain": {"value": round(1000.0 / ms_plain, 4), "unit": "train-steps/s", "ms_per_step": round(ms_plain, 4),
                  "steps": n_plain},
        "batched_graph_vs_plain": round(ms_plain / ms_graph, 3),
        "e2e": {"value": round(1000.0 / ms_e2e, 4), "unit": "train-steps/s",
                "h2d_bytes_per_step": int(n_pix * 12 + vps * 160 + 48), "d2h_bytes_per_step": int(_lib.COUNTERS_BYTES)},
        "gpu_launches": int(total_launches),
        "device_memory_gb": round(dev_gb, 2),
        "stage_ms_per_step": {k: round(v / nb, 4) for k, v in stage_ms.items()},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4),
                     "traffic": int(TILE_DRAM_BYTES_PER_PAIR * int(info.n_pairs_last)),
                     "kernel": f"tile_kernel<{tile[0]},kModeTrain> (fused forward+loss+adjoint, "
                               f"{tile[1]} threads per tile)",
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else
                     "fallback 6.65 TB/s", "launch_ms": round(comp_ms, 4), "algorithmic_bytes": alg,
                     "n_pairs": int(info.n_pairs_last)},
        "issue_roofline": issue_roofline(int(info.n_pairs_last), comp_ms, clocks.get("sm_mhz")),
        "clocks": clocks,
        "training": {"lr_verts": lr["lr_verts"],
                     "loss_first_pass": fin(losses[:nb].mean()), "loss_last_pass": fin(losses[-nb:].mean()),
                     "loss_min": fin(np.nanmin(np.where(np.isfinite(losses), losses, np.nan))),
                     "loss_min_step": int(np.nanargmin(np.where(np.isfinite(losses), losses, np.nan))),
                     "diverged_at_step": d1, "e2e_diverged_at_step": d2,
                     "ms_per_step_before_divergence": round(float(healthy.mean()), 4),
                     "heldout_l1_before": fin(before), "heldout_l1_after": fin(after),
                     "e2e_trajectory_max_rel_diff_before_divergence":
                         fin(np.max(np.abs(losses_e2e[:n_ok] - losses[:n_ok]) / losses[:n_ok])),
                     "loss_every_25": [fin(x) for x in losses[::25]],
                     "note": "at lr_verts 1e-4 the loop diverges in the reference algorithm itself: vertex steps "
                             "flatten tets of the densest component, and a ray through a flat tet with no exit "
                             "face keeps t_max = 3.4e38, so its colour runs to the 1e20 clip (the oracle gives "
                             "the same pixels); --lr-verts 0 converges"},
    }
    if not args.no_cpu_baseline:
        trng = np.random.default_rng(args.seed + 3)
        gts = [trng.uniform(0, 1, (c.height, c.width, 3)).astype(np.float32) for c in batches[0]]
        out["cpu_baseline"] = cpu_baseline(student, batches[0], gts, args)
    print(json.dumps(out), flush=True)


def run_reference(args):
    """CPU port of the reference kernels (the reference's wgpu pipeline needs a
    Vulkan/Metal device, unavailable on this machine).

    A full step of the workload (every view's forward, loss and adjoint, then
    Adam over all parameter groups) takes tens of seconds on the host, so each
    timed step is a bounded sample of it: the next of the step's views in turn
    (forward, L2 loss, adjoint, SH adjoint) followed by the complete Adam update
    of every group (train_step, crates/rmesh-python/src/lib.rs:2405-2636).
    ``steps`` and ``ms_per_step`` are those sampled steps as timed; ``value``
    is the full step's rate, estimated from the same samples as (view time
    scaled by pixels to all of the step's views) + one Adam update."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if args.workload == "training":  # the student scene and one step's batch (uniform targets: same cost)
        _, scene, cams, _ = build_training(args)
        cams = cams[:args.views]
        trng = np.random.default_rng(args.seed + 3)
        gts = [trng.uniform(0, 1, (c.height, c.width, 3)).astype(np.float32) for c in cams]
    else:
        scene, cams, gts = build_workload(args.points, args.seed, 0, args.views, args.res, args.sh_degree, args.cloud)
    n_pix = sum(c.width * c.height for c in cams)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle

    o = Oracle("f32")
    threads = o.max_threads
    shv, deg = _oracle_sh(o, scene, args)
    # Adam state of every trained group (vertices, densities, colour gradients,
    # and the SH coefficients or the base colours)
    params = {"vertices": o._r(scene["vertices"]), "densities": o._r(scene["densities"]),
              "color_grads": o._r(scene["color_grads"])}
    lrs = {"vertices": LR["lr_verts"], "densities": LR["lr_dens"], "color_grads": LR["lr_grads"]}
    if args.sh_degree >= 0:
        params["sh"] = o._r(scene["sh_coeffs"])
        lrs["sh"] = LR_SH
    else:
        params["base_colors"] = o._r(scene["base_colors"])
        lrs["base_colors"] = 0.0
    moments = {k: (np.zeros_like(p), np.zeros_like(p)) for k, p in params.items()}
    gkey = {"vertices": "d_vertices", "densities": "d_densities", "color_grads": "d_color_grads", "sh": "d_sh",
            "base_colors": "d_base_colors"}
    counter = {"step": 0}

    def one(i):
        """Sampled step i: forward, loss and adjoint of the step's i-th view
        (cycling), then Adam over every group.  Returns (pixels, view s, Adam s)."""
        cam, gt = cams[i % len(cams)], gts[i % len(cams)]
        t0 = time.perf_counter()
        fwd = o.forward_tiled(scene, cam, args.tile_size, sh=shv, sh_degree=deg)
        _, dl = o.loss(fwd["image"], gt, 1)
        g = o.backward(scene, cam, dl, fwd, args.tile_size, threads=threads, sh=shv, sh_degree=deg)
        t1 = time.perf_counter()
        counter["step"] += 1
        for k, p in params.items():
            m, v = moments[k]
            o.adam(p, g[gkey[k]], m, v, counter["step"], lrs[k])
        return cam.width * cam.height, t1 - t0, time.perf_counter() - t1

    smallest = min(range(len(cams)), key=lambda i: cams[i].width * cams[i].height)
    for _ in range(args.warmup):
        one(smallest)
    t0 = time.perf_counter()
    res = [one(i) for i in range(args.steps)]
    dt = time.perf_counter() - t0
    px = sum(r[0] for r in res)
    t_views = sum(r[1] for r in res) * n_pix / px
    t_adam = sum(r[2] for r in res) / len(res)
    t_full = t_views + t_adam
    v = round(1.0 / t_full, 6)
    sample = (f"each timed step = one of the step's {len(cams)} views in turn (forward, L2 loss, adjoint) + the "
              f"full Adam update of every group; {args.steps} sampled steps ({px} px) in {dt:.1f} s; full "
              f"{args.views}-view step estimated as view time scaled by pixels to {n_pix} px "
              f"({t_views:.2f} s) + one Adam update ({t_adam:.3f} s) = {t_full:.2f} s; C port of the reference "
              f"kernels, OpenMP {threads} threads")
    print(json.dumps({
        "impl": "reference", "metric": metric_name(args),
        "value": v, "unit": "train-steps/s", "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(dt * 1e3 / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Delaunay mesh, seeded targets)",
        "config": workload_config(args, scene["indices"].size // 4, scene["vertices"].size // 3, n_pix,
                                  int(os.environ.get("WORLD_SIZE", "1"))),
        "full_step_ms_estimate": round(t_full * 1e3, 1),
        "cpu_baseline": {"value": v, "unit": "train-steps/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": "train-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's own pipeline is wgpu (Vulkan/Metal) and cannot run here; this is its CPU port. "
                "steps/ms_per_step are the sampled steps as timed (one view + Adam each); value is the full "
                "step's rate estimated from them",
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="batched", choices=["batched", "large", "training"],
                    help="batched: 100k-point GMM mesh, 16 mixed views (default); large: 1M-point mesh, 8 views "
                         "1080p; training: 250k-point teacher/student loop, 8 of 32 800^2 views per step, 500 steps")
    ap.add_argument("--targets", type=int, default=32, help="target views of the training loop")
    ap.add_argument("--lr-verts", type=float, default=None, help="training loop: vertex learning rate (1e-4)")
    ap.add_argument("--profile-one-step", action="store_true",
                    help="run one batched step of the workload between cudaProfilerStart/Stop (for ncu) and exit")
    ap.add_argument("--points", type=int, default=None)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--tile-size", type=int, default=12)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity-check", action="store_true",
                    help="skip the oracle check of one view's image and gradients (outside the timed region)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep --tile-size instead of searching tile size x threads per tile (and per resolution)")
    ap.add_argument("--views", type=int, default=None, help="views per step (default: the workload's)")
    ap.add_argument("--sh-degree", type=int, default=3, choices=[-1, 0, 1, 2, 3],
                    help="SH degree of the colours (-1: base colours)")
    ap.add_argument("--res", default=None,
                    help="comma-separated WxH choices for the views (default 256x256,512x512,800x600,1024x1024); "
                         "smaller cases serve profiler captures")
    args = ap.parse_args()
    steps_given = any(a == "--steps" or a.startswith("--steps=") for a in sys.argv[1:])
    if args.workload == "training":  # teacher/student loop
        args.points = 250_000 if args.points is None else args.points
        args.views = 8 if args.views is None else args.views
        args.res = args.res or "800x800"
        args.cloud = "gmm"
        args.steps = args.steps if steps_given else 500
        if args.sh_degree < 0 or args.targets % args.views:
            raise SystemExit("training needs SH colours and a target count divisible by --views")
    elif args.workload == "large":  # memory-bound configuration: 1M uniform + 10 % shell points, 8 HD views
        args.points = 1_000_000 if args.points is None else args.points
        args.views = 8 if args.views is None else args.views
        args.res = args.res or "1920x1080"
        args.cloud = "uniform+shell"
    else:
        args.points = 100_000 if args.points is None else args.points
        args.views = N_VIEWS if args.views is None else args.views
        args.cloud = "gmm"
    args.res = RES if args.res is None else tuple(tuple(int(v) for v in x.split("x")) for x in args.res.split(","))
    args.warmup = max(3, args.warmup)
    if args.profile_one_step:
        run_profile_step(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload == "training":
        run_training(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
