"""Benchmark of the caustics hot path: specular paths solved per second and ms/frame of the
batched persistent solver against the plain per-tuple solver, on the two-refraction
dispersive sphere (icosphere subdivided 5 times = 20,480 triangles, r 0.5 at (0,1,0),
Cauchy 1.5 + 4200/nm^2, 4x4 receiver, light at (0,4,0), 1024x1024, 64 wavelength bins,
205 photons per triangle = 4.2M ~ 2^22 Sobol-seeded photons, event string TT).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one frame with the scene and its LBVH resident in HBM: eye pass, photon pass
into the PathCache, lookup/flatten of (pixel, tuple) work items with the count read back,
tuple-coherence sort and reorder, the batched solve of every item for all 64 bins, and the
spectral resolve.  The unit is one (pixel, tuple, wavelength-bin) specular path solve,
counted on the device.  The same frame is then rendered with the plain per-tuple solver
(one thread per path and bin, the reference's kernel structure) for the speed-up and the
relative RMSE between the two images.

Under torchrun each rank renders its own replica of the frame (weak scaling, no data-path
collective): value = all ranks' path solves / the slowest rank's device time.
``--impl reference`` times the reference's own CPU solve (solveConstraints,
contributableThroughput, dAdw, built from the reference sources into oracle/_ref) on the
host cores over a bounded sample of the frame's work items, rank 0 only.
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

METRIC = "specular paths solved/s and ms/frame, batched vs plain GPU at 1e-3 image RMSE"
UNIT = "paths/s"
WORKLOAD = {
    "workload": "two-refraction dispersive sphere",
    "triangles": 20480, "scene": "icosphere-5 r=0.5 at (0,1,0), 4x4 receiver at y=0",
    "light": "0.2x0.2 area light centred at (0,4,0), one point sample per frame (R2 sequence)",
    "ior": "cauchy 1.5 + 4200/nm^2", "image": "1024x1024", "bins": 64, "lambda_nm": [380, 780],
    "photons": 20480 * 205, "events": "TT", "path_cache": 1 << 22,
    "l2": "no flush: every frame streams buffers larger than L2 (PathCache 252 MB, spectral image 268 MB)",
    "fp64_polish": "batched solve: FP64 polish and admissibility of roots whose relative |det J| is below 1e-6",
}
POLISH_DET = 1.0e-6
# kernels of this library launched per frame: k_primary, k_photon, k_lookup, sort k_hist + 4 x k_pass,
# k_reorder, k_probe, k_phase1, 8 phase-2 waves x (k_p2_solve, k_p2_vis, k_p2_contrib) (waves
# without records exit at once), k_resolve_spectral
LAUNCHES_PER_FRAME = 12 + 8 * 3
# Per work item of the batched solve stage (k_probe, k_phase1 and the 8 phase-2 waves of
# k_p2_solve / k_p2_vis / k_p2_contrib), from one ncu capture of every launch of one frame
# of this workload at 256x256 (1,256,661 work items; summarised under profiles/):
# DRAM bytes read + written (1046.5 MB) and warp instructions issued (4.640 G).
NCU_SOLVE_DRAM_PER_ITEM = 832.7
NCU_SOLVE_WARP_INST_PER_ITEM = 3692.0
ISSUE_PER_SM_PER_CLOCK = 4  # one warp instruction per cycle on each of an SM's 4 schedulers


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        threading.Thread(target=self._read, daemon=True).start()
        time.sleep(0.3)

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self) -> dict:
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        rows = [r for r in self.rows if len(r) >= 9]

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [v for v in (num(r[1]) for r in rows) if v is not None]
        mx = [v for v in (num(r[2]) for r in rows) if v is not None]
        reasons = sorted({self.NAMES[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# -------------------------------------------------------------------------------- ranks
def setup_dist():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    """Every rank's device work done, then a process-group barrier (nccl on the GPUs; the
    host-side logic also runs on gloo, without a device)."""
    import torch
    if torch.cuda.is_available():
        torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        if torch.cuda.is_available():
            torch.cuda.synchronize()


def reduce(world, v: float, op: str) -> float:
    """max or sum of a per-rank figure over the ranks (value = all ranks' path solves over the
    slowest rank's device time)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def sphere(image: int = 0):
    from palzilla_b200 import scenes as S
    sc = S.sphere_scene()
    sc.photons_per_triangle = 205
    if image:
        sc.width = sc.height = image
    return sc


# -------------------------------------------------------------------------------- our arm
class Renderer:
    """One frame of the hot path on the current device (all buffers allocated up front)."""

    def __init__(self, sc, fold_det: float = 0.0):
        import torch
        self.fold_det = fold_det
        from palzilla_b200 import api as A
        from palzilla_b200.scenes import event_descriptor
        self.A, self.sc = A, sc
        self.ds = A.DeviceScene(sc)
        self.frame = A.Frame(sc, path_capacity=1 << 25)
        self.cache = A.PathCache(capacity=1 << 22, step=sc.cell_step)
        self.sorter = A.OnesweepSort()
        self.scratch = A.Scratch()
        self.ev = event_descriptor(sc.events)
        self.etas = torch.from_numpy(sc.bin_etas()).cuda()
        npx = sc.width * sc.height
        self.spectral = torch.zeros((npx, sc.n_bins), device="cuda")
        self.rgb = torch.zeros((npx, 4), device="cuda")
        self.pixels = torch.zeros(npx, dtype=torch.int32, device="cuda")
        self.stats = torch.zeros(3, dtype=torch.int64, device="cuda")
        self.n_paths = 0
        self.iteration = 0

    def prepare(self, iteration: int):
        """Eye pass, photon pass, lookup/flatten (count read back), sort and reorder, with
        the light point of this iteration (one sample of the area light)."""
        A, fr = self.A, self.frame
        self.iteration = iteration
        A.solve_primary(self.ds, fr, iteration=iteration)
        self.cache.clear()
        A.photon_trace(self.ds, self.cache, iteration=iteration)
        self.n_paths = A.lookup_flatten(fr, self.cache, self.ev)
        A.sort_and_reorder(fr, self.n_paths, self.sorter)

    def solve(self, plain: bool = False, exact: bool = True, solve_events=None):
        """Specular solve of the prepared work list into a cleared spectral image, then resolve."""
        A, sc = self.A, self.sc
        self.spectral.zero_()
        d = A.solve_desc(self.ds, self.frame, self.cache, sc.events, self.n_paths, spectral=self.spectral,
                         etas=self.etas, stats=self.stats, exact=exact, iteration=self.iteration,
                         polish_det=0.0 if plain else POLISH_DET, fold_det=self.fold_det)
        if solve_events:
            solve_events[0].record()
        if plain:
            A.solve_specular_plain(d)
        else:
            A.solve_specular_batched(d, self.scratch)
        if solve_events:
            solve_events[1].record()
        A.resolve_spectral(self.spectral, sc, rgb=self.rgb, pixels=self.pixels)

    def frame_step(self, iteration: int, plain: bool = False, solve_events=None):
        self.prepare(iteration)
        self.solve(plain=plain, solve_events=solve_events)


def run_ours(args):
    import torch
    world, rank, local = setup_dist()
    sc = sphere(args.image)
    R = Renderer(sc, fold_det=args.fold_det)

    def ev():
        return torch.cuda.Event(enable_timing=True)

    def timed_frames(k, first, plain):
        """k frames bracketed by barriers; returns (device ms, path solves, solve-stage ms list)."""
        solve = [(ev(), ev()) for _ in range(k)]
        e0, e1 = ev(), ev()
        R.stats.zero_()
        barrier(world)
        e0.record()
        for i in range(k):
            R.frame_step(first + i, plain=plain, solve_events=solve[i])
        e1.record()
        barrier(world)
        return e0.elapsed_time(e1), float(R.stats[0].item()), [a.elapsed_time(b) for a, b in solve]

    for i in range(args.warmup):
        R.frame_step(i)
    barrier(world)

    # ---- timed batched frames, clocks sampled meanwhile
    clocks = ClockSampler(local)
    clocks.start()
    ms, paths, solve_ms = timed_frames(args.steps, 100, plain=False)
    clk = clocks.stop()
    t_max = reduce(world, ms, "max")
    paths_all = reduce(world, paths, "sum")
    value = paths_all / (t_max / 1e3)
    counters = R.A.batched_counters(R.scratch)
    n_items = R.n_paths
    contributing = float(R.stats[2].item()) / args.steps

    # ---- end to end through the C ABI: pinned host scene -> HBM, LBVH build, frame, RGBA8 image -> host
    tris_h = torch.from_numpy(np.ascontiguousarray(sc.tris)).pin_memory()
    att_h = torch.from_numpy(np.ascontiguousarray(sc.attribs).view(np.uint8)).pin_memory()
    img_h = torch.empty(sc.width * sc.height, dtype=torch.int32).pin_memory()
    # (right after the timed frames, before the plain solves, at the same clocks; sampled too)
    ke = max(1, min(args.steps, 3))
    e0, e1 = ev(), ev()
    R.stats.zero_()
    clocks_e2e = ClockSampler(local)
    clocks_e2e.start()
    barrier(world)
    e0.record()
    for i in range(ke):
        R.ds.tris.copy_(tris_h, non_blocking=True)
        R.ds.attribs.copy_(att_h, non_blocking=True)
        R.ds.builder.build(R.ds.tris, R.ds.n, 0)
        R.frame_step(200 + i)
        img_h.copy_(R.pixels, non_blocking=True)
    e1.record()
    barrier(world)
    clk_e2e = clocks_e2e.stop()
    e2e_ms = reduce(world, e0.elapsed_time(e1), "max")
    e2e_paths = reduce(world, float(R.stats[0].item()), "sum")

    # ---- plain per-tuple solve of the same frames (fewer of them: it is several times slower)
    kp = max(1, min(args.steps, args.plain_steps))
    R.frame_step(100, plain=True)
    p_ms, p_paths, p_solve_ms = timed_frames(kp, 100, plain=True)
    p_tmax = reduce(world, p_ms, "max")
    p_value = reduce(world, p_paths, "sum") / (p_tmax / 1e3)

    # ---- the reference's own plain per-tuple solve kernel (solveSpecularPath_K2 of main_gpu.cu,
    # compiled for sm_100a with the compiler's default contraction, as its run-time compile
    # builds it) on the same work list: one launch per bin, each with the pixels' wavelength set
    # to the bin's centre, so eta = cauchy(lambda_b) is the bin's eta.  Solve stage only.
    ref_gpu = reference_gpu_solve(R, steps=kp) if rank == 0 and world == 1 and not args.no_ref_gpu else None

    # ---- image agreement on identical solver inputs (one PathCache and work list).  The photon
    # pass itself is not deterministic: the first photon to claim a PathCache slot supplies the
    # tuple's Newton start, as in the reference, so two frames of one iteration already differ.
    def rel(a, b):
        return float(torch.sqrt(((a - b).double() ** 2).mean()) / torch.sqrt((b.double() ** 2).mean()))
    imgs = {}
    # "plain" is the product's plain solve (no FMA contraction: the reference's float arithmetic),
    # the denominator of the speed-up; "plain_fma" is its opt-in FMA-contracted build
    for tag, plain, exact in (("plain", True, True), ("plain_fma", True, False), ("batched", False, True)):
        R.solve(plain=plain, exact=exact)
        torch.cuda.synchronize()
        imgs[tag] = (R.spectral.clone(), R.rgb[:, :3].clone())
    rmse = {}
    for a, b in (("batched", "plain"), ("plain_fma", "plain")):
        rmse[f"{a}_vs_{b}"] = {"spectral": rel(imgs[a][0], imgs[b][0]), "rgb": rel(imgs[a][1], imgs[b][1])}
    del imgs

    # ---- roofline of the dominant kernel pair (the batched solve)
    hbm, hbm_kind = peaks()
    solve_avg = float(np.mean(solve_ms))
    # algorithmic bytes per work item: SpecularPath 8 + FirstDiffuse 40 + PathCache tuple 16 + params 32
    # + two triangles 72 + two attributes 80 = 248 B read once; 4 B per contributing (item, bin) added
    alg_bytes = n_items * 248.0 + contributing * 4.0
    achieved = alg_bytes / (solve_avg / 1e3) / 1e9
    # issue roofline of the same stage: warp instructions (per work item, from the capture)
    # over the stage's time, against 4 schedulers x SMs x the SM clock sampled meanwhile
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    clk_mhz = clk.get("sm_mhz") or 1965.0
    inst = NCU_SOLVE_WARP_INST_PER_ITEM * n_items
    issue_achieved = inst / (solve_avg / 1e3) / 1e9
    issue_peak = ISSUE_PER_SM_PER_CLOCK * sms * clk_mhz * 1e6 / 1e9
    roofline = {"kernel": "batched solve stage: k_probe, k_phase1, 8 waves of k_p2_solve / k_p2_vis / k_p2_contrib",
                "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "peak_kind": hbm_kind, "traffic": NCU_SOLVE_DRAM_PER_ITEM * n_items, "algorithmic_bytes": alg_bytes,
                "traffic_note": "DRAM bytes per work item from an ncu capture of every launch of a 256x256 frame, "
                                "scaled by this frame's work items",
                "issue": {"bound": "issue", "achieved": issue_achieved, "peak": issue_peak,
                          "unit": "G warp instructions/s", "frac": issue_achieved / issue_peak,
                          "warp_instructions": inst,
                          "note": "warp instructions per work item from the same capture; peak = 4 schedulers x "
                                  f"{sms} SMs x the sampled SM clock"},
                "note": "the stage is issue-bound (FP32 Newton/QR and BVH queries in registers, scene and BVH in "
                        "L2): its HBM fraction is small by design, its issue fraction is the bound"}

    stages = frame_stages(R, with_reference=rank == 0 and world == 1 and not args.no_ref_gpu)
    sort_build = bench_sort_build(hbm, hbm_kind) if (rank == 0 and not args.no_sort) else None

    cpu = fp64 = flops = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(R, seconds=args.cpu_seconds)
        fp64 = fp64_error(R)
        flops = newton_flops(R, counters, solve_avg, clk.get("sm_mhz") or 1965.0, sms)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(WORKLOAD, image=f"{sc.width}x{sc.height}",
                           parallelism=f"{world} independent frame replicas" if world > 1 else "1 GPU",
                           **({"fold_det": args.fold_det} if args.fold_det else {})),
            "ms_per_frame": t_max / args.steps,
            "work_items_per_frame": n_items,
            "path_solves_per_frame": paths / args.steps,
            "newton_solves": {
                "per_frame": counters["newton_bins"] + 3 * n_items,
                "per_s": (counters["newton_bins"] + 3 * n_items) / (solve_avg / 1e3),
                "note": "Newton solves the batched solve ran (3 probes per work item, then the bins phase 2 "
                        "solved) over the solve stage's time; value counts every (item, bin) decided, as the "
                        "plain path decides each by a Newton solve"},
            "solve_ms_per_frame": solve_avg,
            "solve_ms_frames": [round(float(t), 3) for t in solve_ms],
            "frame_stages": stages,
            "plain": {"value": p_value, "ms_per_frame": p_tmax / kp, "solve_ms_per_frame": float(np.mean(p_solve_ms)),
                      "steps": kp},
            "speedup_paths_per_s_vs_plain": value / p_value,
            "speedup_solve_vs_plain": float(np.mean(p_solve_ms)) / solve_avg,
            "reference_gpu_plain": None if ref_gpu is None else dict(
                ref_gpu, speedup_solve=ref_gpu["solve_ms_per_frame"] / solve_avg,
                speedup_paths_per_s=(t_max / args.steps - solve_avg + ref_gpu["solve_ms_per_frame"]) /
                (t_max / args.steps),
                frame_note="frame-level speed-up: this frame with its solve stage replaced by the reference "
                           "kernel's"),
            "image_rel_rmse": rmse,
            "fp64_error": fp64,
            "fp32_flops": flops,
            "batched_counters": counters,
            "e2e": {"value": e2e_paths / (e2e_ms / 1e3), "unit": UNIT, "steps": ke, "ms_per_step": e2e_ms / ke,
                    "h2d_bytes_per_step": int(tris_h.numel() * 4 + att_h.numel()),
                    "d2h_bytes_per_step": int(img_h.numel() * 4),
                    "path": "pinned host scene -> device, pz_bvh_build, full frame, RGBA8 image -> pinned host",
                    "clocks": clk_e2e},
            "gpu_launches": LAUNCHES_PER_FRAME * args.steps,
            "roofline": roofline,
            "sort_build": sort_build,
            "cpu_baseline": cpu,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def frame_stages(R, first=300, frames=3, with_reference=False):
    """CUDA-event times of a frame's stages before the solve (median over `frames` frames):
    eye pass (primary and shadow rays), photon pass, lookup/flatten with the count read back,
    tuple sort and reorder; with rays/s and photons/s."""
    import torch
    A, fr, sc = R.A, R.frame, R.sc

    def ev():
        return torch.cuda.Event(enable_timing=True)
    t = {"eye_pass": [], "photon_pass": [], "lookup": [], "sort_reorder": []}
    for i in range(frames):
        e = [ev() for _ in range(5)]
        torch.cuda.synchronize()
        e[0].record()
        A.solve_primary(R.ds, fr, iteration=first + i)
        e[1].record()
        R.cache.clear()
        A.photon_trace(R.ds, R.cache, iteration=first + i)
        e[2].record()
        n = A.lookup_flatten(fr, R.cache, R.ev)
        e[3].record()
        A.sort_and_reorder(fr, n, R.sorter)
        e[4].record()
        torch.cuda.synchronize()
        for k, (a, b) in zip(t, zip(e[:-1], e[1:])):
            t[k].append(a.elapsed_time(b))
    ms = {k: float(np.median(v)) for k, v in t.items()}
    photons = sc.n * sc.photons_per_triangle
    out = {"ms": ms, "primary_rays_per_s": sc.width * sc.height / (ms["eye_pass"] / 1e3),
           "photons_per_s": photons / (ms["photon_pass"] / 1e3),
           "note": "each pixel: one primary ray and a shadow ray; each photon: up to 5 closest-hit rays"}
    if with_reference:
        out["reference_gpu_photon_pass"] = reference_gpu_photons(R, first, frames)
        ref = out["reference_gpu_photon_pass"]
        if "photons_per_s" in ref:
            ref["speedup_photons_per_s"] = out["photons_per_s"] / ref["photons_per_s"]
    return out


def reference_gpu_photons(R, first, frames):
    """The reference's photonTrace (main_gpu.cu:56-211, its sources built for sm_100a): one
    256-thread block per triangle (256 photons each, its fixed block size) into its own
    PathCache, on the same scene, BVH and light samples; median of `frames` launches."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_gpu as G
    if not G.available("default"):
        return {"unavailable": "reference GPU kernels not built (oracle/build_ref_gpu.sh needs the reference sources)"}
    rg = G.RefGpu("default")
    sc = R.sc
    rc = rg.new_cache()
    stack = rg.new_stack()
    emin, emax = sc.eta_range()
    ts = []
    for i in range(frames + 1):
        rc["hashes"].zero_()
        rc["count"].zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        rg.photon_trace(rc, R.ds.internals, R.ds.root_dev, R.ds.tris, R.ds.attribs, R.ds.n, sc.light_point(first + i),
                        emin, emax, first + i, sc.cell_step, sc.min_throughput, stack)
        e1.record()
        torch.cuda.synchronize()
        if i > 0:
            ts.append(e0.elapsed_time(e1))
    ms = float(np.median(ts))
    photons = sc.n * 256
    del stack, rc
    return {"ms": ms, "photons": photons, "photons_per_s": photons / (ms / 1e3),
            "kernel": "photonTrace (main_gpu.cu:56-211), default build, 256 photons per triangle"}


def reference_gpu_solve(R, steps=2):
    """Times the reference's solveSpecularPath_K<K> (default build) over the prepared frame's
    work list for every bin: per bin, a FirstDiffuse copy with lambda set to the bin's centre."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_gpu as G
    import torch
    if not G.available("default"):
        return {"unavailable": "reference GPU kernels not built (oracle/build_ref_gpu.sh needs the reference sources)"}
    rg = G.RefGpu("default")
    sc, fr = R.sc, R.frame
    K = len(sc.events)
    rc = rg.cache_from_ours(R.cache.views())
    fds = []
    for lam in sc.bin_lambdas():
        f = fr.fd.clone()
        f.view(torch.float32).view(fr.npx, 10)[:, 9] = float(lam)
        fds.append(f)
    accum = torch.zeros((fr.npx, 4), device="cuda")
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in fds]

    def run():
        for f, (e0, e1) in zip(fds, ev):
            e0.record()
            rg.solve_specular(K, accum, fr.paths, R.n_paths, f, R.ds.root_dev, R.ds.internals, R.ds.tris,
                              R.ds.attribs, sc.light_point(R.iteration), sc.light_intensity, sc.radiance_clamp, rc,
                              sc.cell_step, R.ev, sc.cauchy_a, sc.cauchy_b, R.iteration)
            e1.record()
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in ev)
    run()
    ms = float(np.mean([run() for _ in range(max(1, steps))]))
    del fds, rc
    return {"solve_ms_per_frame": ms, "value": R.n_paths * sc.n_bins / (ms / 1e3), "unit": UNIT,
            "kernel": f"solveSpecularPath_K{K} (main_gpu.cu:418-497), {sc.n_bins} launches per frame",
            "build": "reference sources, nvcc -gencode arch=compute_100a,code=sm_100a -O3 (default FMA contraction)"}


def bench_sort_build(hbm, hbm_kind, n=1 << 24):
    """Onesweep sort of n {32-bit key, 32-bit index} pairs and the LBVH build of n random
    triangles (the sort + build workload at its largest size), L2 flushed between reps."""
    import torch
    from palzilla_b200 import scenes as S
    from palzilla_b200.api import BVHGPUBuilder, OnesweepSort
    g = torch.Generator(device="cuda").manual_seed(1)
    base = torch.randint(0, 1 << 30, (n,), device="cuda", generator=g, dtype=torch.int64) | \
        (torch.arange(n, device="cuda", dtype=torch.int64) << 32)
    keys, tmp = base.clone(), torch.empty_like(base)
    sorter = OnesweepSort()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def med(fn, reps=7, warm=3):
        ts = []
        for i in range(warm + reps):
            keys.copy_(base)
            flush.fill_(i & 0xFF)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            if i >= warm:
                ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))
    sort_ms = med(lambda: sorter.sort(keys, None, tmp, None, n, 0, 32))
    tris = torch.from_numpy(S.random_soup(n, seed=1001)).cuda()
    b = BVHGPUBuilder()
    build_ms = med(lambda: b.build(tris, n, 0))
    # the reference's own LBVH kernels (getSceneAABB, buildMortons, computeDeltas, build;
    # minimum_lbvh.cu:6-120, built from its sources for sm_100a) on the same triangles, with
    # this library's sort between them (the reference's onesweep reorder is not run: it takes
    # its tile from blockIdx.x and waits on its predecessors without a bound)
    ref_build = None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_gpu as G
    if G.available("default"):
        rg = G.RefGpu("default")
        ref_build = {"ms": med(lambda: rg.bvh_build(tris, n, lambda k, t, m: sorter.sort(k, None, t, None, m, 0, 32))),
                     "kernels": "the reference's minimum_lbvh.cu kernels (default build) + this library's sort"}
        ref_build["speedup"] = ref_build["ms"] / build_ms
    sort_gbs = 72.0 * n / (sort_ms / 1e3) / 1e9
    build_gbs = (189.0 + 72.0) * n / (build_ms / 1e3) / 1e9
    return {"n": n, "sort_ms": sort_ms, "keys_per_s": n / (sort_ms / 1e3),
            "sort_roofline": {"bound": "hbm", "achieved": sort_gbs, "peak": hbm, "unit": "GB/s",
                              "frac": sort_gbs / hbm, "peak_kind": hbm_kind, "bytes_per_key": 72},
            "build_ms": build_ms, "triangles_per_s": n / (build_ms / 1e3), "reference_gpu_build": ref_build,
            "build_roofline": {"bound": "hbm", "achieved": build_gbs, "peak": hbm, "unit": "GB/s",
                               "frac": build_gbs / hbm, "peak_kind": hbm_kind, "bytes_per_triangle": 261}}


def run_uneven_batch(args):
    """Uneven batch: 256 heightfield lenses (grid side log-uniform in 16..256, 450 to 130,050
    triangles, 1-2 refractions, amplitude U[0.005, 0.03]), 256 x 256 image and 16 bins
    each, 16 photons per triangle.  A frame renders every scene: eye pass, photon pass,
    lookup / flatten with device item counts, the batched solve, resolve.  Three ways:
    one batched solve per scene with the item count read back (the reference's host
    flow), one batched solve per K over all scenes, and that frame captured in a CUDA
    graph and replayed with the autotuned launch shapes."""
    import torch
    from palzilla_b200 import api as A
    from palzilla_b200 import scenes as S
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    scenes = S.uneven_batch(n_scenes=args.batch_scenes, seed=3001, width=256, height=256, n_bins=16,
                            photons_per_triangle=16)
    items = []
    for sc in scenes:
        ds = A.DeviceScene(sc)
        fr = A.Frame(sc, path_capacity=1 << 19)
        # PathCache sized to the photon count (every photon inserts up to 8 cells)
        cap = 1 << max(16, int(np.ceil(np.log2(4 * sc.n * sc.photons_per_triangle))))
        items.append(dict(sc=sc, ds=ds, fr=fr, cache=A.PathCache(capacity=cap, step=sc.cell_step),
                          ev=S.event_descriptor(sc.events), etas=torch.from_numpy(sc.bin_etas()).cuda(),
                          spec=torch.zeros((sc.width * sc.height, sc.n_bins), device="cuda"),
                          pixels=torch.zeros(sc.width * sc.height, dtype=torch.int32, device="cuda")))
    stats = torch.zeros(3, dtype=torch.int64, device="cuda")

    def size_work_list(it):
        """One eye pass, photon pass and lookup; the work list then gets room for 1.25x the
        item count it saw (the lookup counter counts past the capacity)."""
        prep(it, 0, None)
        n = int(it["fr"].counter.item())
        need = 1 << max(16, int(np.ceil(np.log2(max(1, int(1.25 * n))))))
        if need > it["fr"].path_capacity:
            it["fr"] = A.Frame(it["sc"], path_capacity=need)

    def prep(it, iteration, stream):
        A.solve_primary(it["ds"], it["fr"], iteration=iteration, stream=stream)
        it["cache"].clear(stream)
        A.photon_trace(it["ds"], it["cache"], iteration=iteration, stream=stream)
        it["fr"].counter.zero_()
        A._lib.call("pz_lookup_flatten", A.C.c_uint32(it["ev"]), A._vp(it["fr"].paths), A._vp(it["fr"].indexed),
                    A._vp(it["fr"].counter), A.C.c_uint32(it["fr"].path_capacity), A._vp(it["fr"].fd),
                    A.C.c_int(it["fr"].npx), A._vp(it["cache"].buf), A.C.c_uint32(it["cache"].capacity),
                    A.C.c_float(it["cache"].step), A.C.c_void_p(A._stream(stream)))
        it["spec"].zero_()

    def desc(it, cap):
        return A.solve_desc(it["ds"], it["fr"], it["cache"], it["sc"].events, cap, spectral=it["spec"],
                            etas=it["etas"])

    for it in items:
        size_work_list(it)
    groups = {}
    for it in items:
        groups.setdefault(len(it["sc"].events), []).append(it)
    batches = {K: A.SceneBatch([desc(it, it["fr"].path_capacity) for it in g], counts=[it["fr"].counter for it in g])
               for K, g in groups.items()}

    def frame_multi(iteration, stream=None, tuned=False):
        for it in items:
            prep(it, iteration, stream)
        for K, sb in batches.items():
            sb.solve(tuning=None if tuned else (8, 2, 1), stats=stats, stream=stream)
        for it in items:
            A.resolve_spectral(it["spec"], it["sc"], pixels=it["pixels"], stream=stream)

    scratch = A.Scratch()

    def frame_per_scene(iteration):
        for it in items:
            prep(it, iteration, None)
            n = min(int(it["fr"].counter.item()), it["fr"].path_capacity)
            d = desc(it, n)
            d.stats = stats.data_ptr()
            A.solve_specular_batched(d, scratch)
            A.resolve_spectral(it["spec"], it["sc"], pixels=it["pixels"])

    def timed(fn, k):
        stats.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for i in range(k):
            fn(i)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k, float(stats[0].item()) / k

    for i in range(args.warmup):
        frame_per_scene(i)
        frame_multi(i)
    tunings = {K: sb.autotune(stats=stats) for K, sb in batches.items()}
    per_ms, paths = timed(frame_per_scene, args.steps)
    multi_ms, paths_m = timed(frame_multi, args.steps)
    stream = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        frame_multi(0, stream, tuned=True)  # warm the capture stream
        torch.cuda.synchronize()
        with torch.cuda.graph(graph, stream=stream):
            frame_multi(0, stream, tuned=True)
    graph_ms, paths_g = timed(lambda i: graph.replay(), args.steps)
    tri = sum(it["sc"].n for it in items)
    cache_status = sum(int(it["cache"].status() != 0) for it in items)
    line = {"metric": "specular paths solved/s and ms/frame, uneven batch of scenes", "workload": "uneven_batch",
            "path_cache_overflows": cache_status,
            "value": paths_g / (graph_ms / 1e3), "unit": "paths/s", "higher_is_better": True, "dtype": "f32",
            "data": "synthetic", "scenes": len(items), "triangles": tri, "steps": args.steps, "warmup": args.warmup,
            "path_solves_per_frame": paths_g,
            "ms_per_frame": {"per_scene_solves": per_ms, "one_solve_per_K": multi_ms, "graph_autotuned": graph_ms},
            "paths_per_s": {"per_scene_solves": paths / (per_ms / 1e3), "one_solve_per_K": paths_m / (multi_ms / 1e3),
                            "graph_autotuned": paths_g / (graph_ms / 1e3)},
            "tuning": {str(K): {"p1_blocks_per_sm": t[0][0], "p2_blocks_per_sm": t[0][1], "p2_chunk": t[0][2],
                                "solve_ms": t[1]} for K, t in tunings.items()}}
    print(json.dumps(line), flush=True)


def run_pathcuts(args):
    """Path Cuts (traverseAdmissibleNodes<2>, TT) on the two-sheet heightfield lens (side 64:
    8,388 triangles, USE_NORMAL BVH): admissible tuples of 4,096 receiver points on a grid,
    round-to-nearest and directed rounding; the subdivision solve of the tuples of the first
    256 points; the reference's CPU traversal (oracle/_ref) is timed on a bounded sample of
    the points (one OpenMP thread per query)."""
    import torch
    from palzilla_b200 import api as A
    from palzilla_b200 import scenes as S
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    sc = S.lens_scene(side=64, seed=1, width=64, height=64, n_bins=1, events="TT")
    t = torch.from_numpy(np.ascontiguousarray(sc.tris)).cuda()
    at = torch.from_numpy(np.ascontiguousarray(sc.attribs).view(np.uint8).reshape(-1)).cuda()
    b = A.BVHGPUBuilder()
    b.build(t, sc.n, 1)
    nbs = A.normal_bounds(b, at)
    g = np.linspace(-0.45, 0.45, 64, dtype=np.float32)
    X, Z = np.meshgrid(g, g)
    ends = np.stack([X.ravel(), np.zeros(X.size, np.float32), Z.ravel()], 1).astype(np.float32)
    ends_d = torch.from_numpy(ends).cuda()
    pc = A.PathCuts(frontier_capacity=1 << 26, tuple_capacity=1 << 25)
    ev = S.event_descriptor("TT")
    res = {}
    for mode in ("rn", "dr"):
        for i in range(args.warmup):
            pc.run(2, ev, 1.52, sc.p_light, ends_d, b, nbs, t, at, directed=mode == "dr")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in range(args.steps):
            rows, visited = pc.run(2, ev, 1.52, sc.p_light, ends_d, b, nbs, t, at, directed=mode == "dr")
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1e3 / args.steps
        res[mode] = {"ms": ms, "tuples": int(rows.shape[0]), "node_tuples": int(visited),
                     "node_tuples_per_s": visited / (ms / 1e3), "queries_per_s": len(ends) / (ms / 1e3)}
    # every root of the admissible tuples of the first 256 receiver points: the subdivision
    # solve on the round-to-nearest Path Cuts rows (one bin, eta 1.52; the visibility BVH is
    # the same tree, any BVH over the triangles answers the same any-hit queries)
    sub_q = 256
    rows_q, _ = pc.run(2, ev, 1.52, sc.p_light, ends_d[:sub_q], b, nbs, t, at)
    solver = A.SubdivisionSolver(box_capacity=1 << 26, root_capacity=1 << 22)
    eta1 = torch.tensor([1.52], device="cuda")
    for i in range(args.warmup):
        solver.run(2, ev, sc.p_light, ends_d, rows_q, eta1, t, at, b, t)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(args.steps):
        _, _, _, sst = solver.run(2, ev, sc.p_light, ends_d, rows_q, eta1, t, at, b, t)
    torch.cuda.synchronize()
    sub_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    subdivision = {"queries": sub_q, "rows": int(rows_q.shape[0]), "ms": sub_ms, "stats": sst,
                   "rows_per_s": int(rows_q.shape[0]) / (sub_ms / 1e3)}
    cpu = None
    lib, kind = _cpu_lib()
    if lib.has("path_cuts"):
        import oracle as O
        bo = lib.build_bvh(sc.tris, 1)
        nbo = lib.normal_bounds(bo["nodes"], sc.tris, sc.attribs)
        sample = ends[:: max(1, len(ends) // args.cuts_sample)]
        t0 = time.perf_counter()
        n_cpu = 0
        for pe in sample:
            n_cpu += len(lib.path_cuts(2, ev, 1.52, sc.p_light, pe, bo["nodes"], nbo, sc.tris, sc.attribs, bo["root"]))
        dt = time.perf_counter() - t0
        cpu = {"value": len(sample) / dt, "unit": "queries/s", "cores": 1, "kind": kind,
               "sample": f"{len(sample)} of the {len(ends)} receiver points, {n_cpu} tuples, {dt:.1f} s"}
    print(json.dumps({"metric": "Path Cuts queries/s (admissible K=2 tuples per receiver point)",
                      "workload": "pathcuts", "value": res["rn"]["queries_per_s"], "unit": "queries/s",
                      "higher_is_better": True, "data": "synthetic", "triangles": sc.n, "queries": len(ends),
                      "round_to_nearest": res["rn"], "directed_rounding": res["dr"],
                      "subdivision_of_the_tuples": subdivision, "cpu_baseline": cpu}),
          flush=True)


def run_subdivision(args):
    """Subdivision workload: the single-refraction heightfield lens (64 x 64 vertices, 7,938
    lens triangles), 256 x 256 image, 16 bins, point light at (0,3,0).  The photon pass's
    work list -- one row per (pixel, cached tuple) -- is solved by per-tuple domain
    subdivision (depth limit 12, eps 1e-4, affine bounds with directed rounding) and the
    roots go to the binned spectral image; each step is pz_subdivide_solve +
    pz_subdivide_contribute on inputs already in HBM (the work list is 701 k rows x 8 B, L2
    is not flushed: the rows, boxes and leaves stream through buffers of up to 800 MB).
    The unit is one (work item, bin) domain solved for all its roots.  The single-start
    plain solve of the same work list is timed beside it, and the CPU oracle of the
    subdivision on a sample of the rows."""
    import torch
    from palzilla_b200 import api as A
    from palzilla_b200 import scenes as S
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    sc = S.lens_scene(side=64, seed=1, width=256, height=256, n_bins=16, events="T")
    ds = A.DeviceScene(sc)
    frame = A.Frame(sc, path_capacity=1 << 24)
    cache = A.PathCache(capacity=1 << 22, step=sc.cell_step)
    ev = S.event_descriptor("T")
    A.solve_primary(ds, frame, iteration=0)
    A.photon_trace(ds, cache, iteration=0)
    n = A.lookup_flatten(frame, cache, ev)
    A.sort_and_reorder(frame, n, A.OnesweepSort())
    rows = A.work_list_rows(frame, cache, n, 1)
    ends = A.receiver_points(frame)
    etas = torch.from_numpy(sc.bin_etas()).cuda()
    spectral = torch.zeros((sc.width * sc.height, sc.n_bins), device="cuda")
    solver = A.SubdivisionSolver(box_capacity=1 << 25, root_capacity=1 << 24)

    def step():
        spectral.zero_()
        _, _, _, st = solver.run(1, ev, sc.light_point(0), ends, rows, etas, ds.tris, ds.attribs, ds.builder, ds.tris)
        solver.contribute(1, ev, sc, rows, st["roots"], frame, etas, ds.tris, ds.attribs, spectral)
        return st

    for _ in range(args.warmup):
        st = step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        st = step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    plain = torch.zeros_like(spectral)
    d = A.solve_desc(ds, frame, cache, "T", n, spectral=plain, etas=etas)
    A.solve_specular_plain(d)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        A.solve_specular_plain(d)
    e1.record()
    torch.cuda.synchronize()
    ms_plain = e0.elapsed_time(e1) / args.steps
    plain.zero_()
    A.solve_specular_plain(d)
    torch.cuda.synchronize()
    domains = n * sc.n_bins
    cpu = None
    if not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        orc = O.oracle()
        bo = orc.build_bvh(sc.tris, 0)
        rows_h, ends_h = rows.cpu().numpy(), ends.cpu().numpy()
        sample = rows_h[:: max(1, len(rows_h) // 300000)]
        t0 = time.perf_counter()
        orc.subdivide_solve(1, ev, sc.light_point(0), ends_h, sample, sc.bin_etas(), sc.tris, sc.attribs, bo, sc.tris,
                            cap=1 << 24)
        dt = time.perf_counter() - t0
        cpu = {"value": len(sample) * sc.n_bins / dt, "unit": "(work item, bin) domains/s", "cores": orc.max_threads(),
               "kind": "port", "sample": f"{len(sample)} of the {n} work items, all {sc.n_bins} bins, {dt:.1f} s"}
    print(json.dumps({"metric": "subdivision solve: (work item, bin) domains solved/s",
                      "workload": "subdivision", "value": domains / (ms / 1e3), "unit": "(work item, bin) domains/s",
                      "higher_is_better": True, "data": "synthetic", "dtype": "f32",
                      "config": {"workload": "single-refraction heightfield lens", "triangles": sc.n,
                                 "image": "256x256", "bins": sc.n_bins, "max_depth": 12, "eps": 1e-4},
                      "work_items": n, "ms_per_step": ms, "stats": st, "steps": args.steps, "warmup": args.warmup,
                      "roots_per_s": st["roots"] / (ms / 1e3), "boxes_per_s": st["boxes_tested"] / (ms / 1e3),
                      "leaf_newton_solves_per_s": st["solves"] / (ms / 1e3),
                      "plain_single_start": {"ms": ms_plain, "value": domains / (ms_plain / 1e3)},
                      "image_energy_subdivision_over_single_start": float(spectral.sum() / plain.sum()),
                      "cpu_baseline": cpu}),
          flush=True)


def run_adjoint(args):
    """Adjoint workload: 128 x 128 heightfield lens (32,258 triangles), 512 x 512 image, 8
    bins, L2 loss against a second seeded heightfield: forward (exact-arithmetic binned
    solve) and backward (roots recomputed, implicit-function gradients) per step."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from grad_harness import CausticProblem
    from palzilla_b200 import scenes as S
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    sc, corners, h0 = S.adjoint_scene(side=128, seed=1)
    P = CausticProblem(sc, corners)
    sc2, c2, h2 = S.adjoint_scene(side=128, seed=2)
    P2 = CausticProblem(sc2, c2)
    cauchy = torch.tensor([1.5, 4200.0], dtype=torch.float32, device="cuda")
    target = P2.forward(torch.from_numpy(h2).cuda(), cauchy).clone()
    del P2
    h = torch.from_numpy(h0).cuda()
    for i in range(args.warmup):
        I = P.forward(h, cauchy)
        P.backward(h, cauchy, (2.0 * (I - target)).contiguous())
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    fwd, bwd = [], []
    for i in range(args.steps):
        ev[0].record()
        I = P.forward(h, cauchy)
        ev[1].record()
        gh, gc = P.backward(h, cauchy, (2.0 * (I - target)).contiguous())
        ev[2].record()
        torch.cuda.synchronize()
        fwd.append(ev[0].elapsed_time(ev[1]))
        bwd.append(ev[1].elapsed_time(ev[2]))
    paths = P.n_paths * sc.n_bins
    print(json.dumps({"metric": "adjoint forward + backward ms (gradient of an L2 image loss)",
                      "workload": "adjoint", "value": float(np.mean(fwd) + np.mean(bwd)), "unit": "ms",
                      "higher_is_better": False, "data": "synthetic", "triangles": sc.n, "image": "512x512x8",
                      "path_solves": paths, "forward_ms": float(np.mean(fwd)), "backward_ms": float(np.mean(bwd)),
                      "backward_paths_per_s": paths / (float(np.mean(bwd)) / 1e3),
                      "note": "forward includes the LBVH rebuild from the heights; backward includes it too"}),
          flush=True)


def run_sort_build(args):
    """Sort + build alone: n uniform random triangles (edges of 1e-3 to 1e-2), 32-bit Morton
    keys with 32-bit index payloads, onesweep sort and LBVH build, one line per size."""
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    hbm, hbm_kind = peaks()
    for lg in [int(x) for x in args.sizes.split(",") if x]:
        r = bench_sort_build(hbm, hbm_kind, n=1 << lg)
        print(json.dumps({"metric": "keys/s and LBVH build ms (onesweep sort + build)", "workload": "sort_build",
                          "value": r["keys_per_s"], "unit": "keys/s", "higher_is_better": True,
                          "dtype": "u64 (32-bit key + 32-bit index)", "data": "synthetic", **r}), flush=True)


# -------------------------------------------------------------------------------- CPU
def _cpu_lib():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    ref = O.reference()
    return (ref, "reference") if ref is not None else (O.oracle(), "port")


def _sample(pairs, n, seed):
    rng = np.random.default_rng(seed)
    return pairs[np.sort(rng.choice(len(pairs), size=min(n, len(pairs)), replace=False))].copy()


def cpu_baseline(R, seconds=15.0):
    """The reference's CPU solve over a bounded sample of this frame's work items (with the
    frame's light point), OpenMP over all host threads; about `seconds` of CPU work."""
    lib, kind = _cpu_lib()
    import oracle as O
    sc = R.sc
    n = R.n_paths
    pairs = R.frame.paths[: n * 8].cpu().numpy().view(np.int32).reshape(-1, 2)
    cache = R.cache.to_host()
    fd = R.frame.fd.cpu().numpy().view(np.float32).reshape(-1, 10)
    nodes = np.frombuffer(R.ds.internals[: (R.ds.n - 1) * 64].cpu().numpy().tobytes(), O.NODE_DTYPE)
    bvh = {"nodes": nodes, "root": R.ds.builder.root}
    etas = sc.bin_etas()
    probe = _sample(pairs, 512, 1)
    t0 = time.perf_counter()
    lib.render_pairs(2, probe, cache, fd, bvh, sc, etas, iteration=R.iteration)
    dt = time.perf_counter() - t0
    m = int(min(len(pairs), max(512, len(probe) * seconds / max(dt, 1e-3))))
    sel = _sample(pairs, m, 2)
    t0 = time.perf_counter()
    _, st = lib.render_pairs(2, sel, cache, fd, bvh, sc, etas, iteration=R.iteration)
    dt = time.perf_counter() - t0
    paths_per_s = float(st[0]) / dt
    out = {"value": paths_per_s, "unit": UNIT, "cores": lib.max_threads(), "kind": kind,
           "sample": f"solve stage: {len(sel)} of the frame's {n} (pixel, tuple) work items x 64 bins "
                     f"= {int(st[0])} path solves in {dt:.1f} s"}
    out["stages"] = cpu_stages(R, lib, kind, solve_paths_per_s=paths_per_s)
    return out


def fp64_error(R, n=100000):
    """Error of the headline image against FP64 on a sample of the frame's work items: the
    batched solve (the headline's settings) of the sample alone on the GPU, against the
    oracle's FP64 instantiation of the same per-path functions on the same inputs (and the
    oracle's FP32 instantiation, which equals the reference's float arithmetic, beside it)."""
    import torch
    import oracle as O
    A, sc = R.A, R.sc
    m = R.n_paths
    pairs = R.frame.paths[: m * 8].cpu().numpy().view(np.int32).reshape(-1, 2)
    sel = _sample(pairs, n, 3)
    cache = R.cache.to_host()
    fd = R.frame.fd.cpu().numpy().view(np.float32).reshape(-1, 10)
    nodes = np.frombuffer(R.ds.internals[: (R.ds.n - 1) * 64].cpu().numpy().tobytes(), O.NODE_DTYPE)
    bvh = {"nodes": nodes, "root": R.ds.builder.root}
    paths = torch.from_numpy(np.ascontiguousarray(sel).reshape(-1)).cuda()
    spectral = torch.zeros_like(R.spectral)
    d = A.solve_desc(R.ds, R.frame, R.cache, sc.events, len(sel), spectral=spectral, etas=R.etas,
                     iteration=R.iteration, polish_det=POLISH_DET, fold_det=R.fold_det)
    d.paths = paths.data_ptr()
    A.solve_specular_batched(d, A.Scratch())
    torch.cuda.synchronize()
    gpu = spectral.cpu().numpy().astype(np.float64)
    orc = O.oracle()
    etas = sc.bin_etas()
    img64, _ = orc.render_pairs(2, sel, cache, fd, bvh, sc, etas, dtype=np.float64, iteration=R.iteration)
    img32, _ = orc.render_pairs(2, sel, cache, fd, bvh, sc, etas, dtype=np.float32, iteration=R.iteration)

    def rel(a, b):
        b = b.astype(np.float64)
        return float(np.sqrt(((a.astype(np.float64) - b) ** 2).mean() / max((b ** 2).mean(), 1e-300)))
    return {"batched_vs_fp64": rel(gpu, img64), "oracle_fp32_vs_fp64": rel(img32, img64),
            "batched_vs_oracle_fp32": rel(gpu, img32),
            "sample": f"{len(sel)} of the frame's {m} work items x {sc.n_bins} bins, spectral image rel. RMSE"}


def newton_flops(R, counters, solve_ms, sm_mhz, sms):
    """FP32 operations of the solve stage's Newton iterations: one iteration of the
    restated solveConstraints<2> (the reference's algorithm: 2K single-tangent dual
    evaluations, Householder QR, update) counted with a counting scalar type on the
    frame's first work item's chain, times the Newton iterations phase 2 ran, over the
    solve stage's time.  The probes' and phase 1's iterations are not in the count, so the
    figure is a lower bound.  Peak: 128 FP32 lanes x 148 SMs x 2 (FMA) x the SM clock; the
    solver units are built without FMA contraction, so one lane does one operation a clock
    and half that peak is their ceiling."""
    import oracle as O
    from palzilla_b200.scenes import event_descriptor
    sc = R.sc
    pairs = R.frame.paths[:8].cpu().numpy().view(np.int32).reshape(-1, 2)
    px, slot = int(pairs[0, 0]), int(pairs[0, 1])
    cache = R.cache.to_host()
    fd = R.frame.fd[px * 40:(px + 1) * 40].cpu().numpy().view(np.float32)
    tup = cache["tris"][slot, :2]
    c = O.oracle().count_newton_flops(2, cache["params"][slot, :4], sc.light_point(R.iteration), fd[:3],
                                      sc.tris[tup], sc.attribs[tup], float(sc.bin_etas()[sc.n_bins // 2]),
                                      event_descriptor(sc.events))
    iters = float(counters["newton_iterations"])
    achieved = c["total"] * iters / (solve_ms / 1e3) / 1e9
    peak = 128 * sms * 2 * sm_mhz * 1e6 / 1e9
    return {"per_newton_iteration": c, "newton_iterations": iters, "achieved": achieved, "peak": peak,
            "unit": "GFLOP/s", "frac": achieved / peak,
            "note": "phase-2 Newton iterations only (a lower bound); peak with FMA, the solver units run "
                    "without contraction (ceiling half of it)"}


def cpu_stages(R, lib, kind, solve_paths_per_s, reps=5):
    """The reference's CPU code per stage of the frame, median of `reps` runs each, OpenMP
    over all host threads: BVHCPUBuilder with BUILD_OPTION_CPU_PARALLEL (minimum_lbvh.h:518-684;
    its std::sort of the Morton keys is inside) on a 2^20-triangle soup and on the frame's
    scene, the photon loop (photonTrace's body, main_gpu.cu:56-211) at a bounded number of
    photons per triangle, and the eye pass (solvePrimary, main_gpu.cu:213-371; the oracle's
    restatement); with the solve stage's paths/s, an estimate of the CPU's ms per frame."""
    import oracle as O
    from palzilla_b200 import scenes as S
    sc = R.sc

    def med(fn):
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            fn()
            ts.append(time.perf_counter() - t0)
        return float(np.median(ts))

    soup = S.random_soup(1 << 20, seed=7)
    cpu_parallel = 2  # BUILD_OPTION_CPU_PARALLEL
    t_soup = med(lambda: lib.cpu_builder(soup, cpu_parallel))
    t_scene = med(lambda: lib.cpu_builder(sc.tris, cpu_parallel))
    b = lib.cpu_builder(sc.tris, cpu_parallel)
    bvh = {"nodes": b["nodes"], "root": b["root"]}
    ppt = 32
    t_ph = med(lambda: lib.photon_trace(bvh, sc, iteration=R.iteration, photons_per_tri=ppt))
    photons = sc.n * ppt
    orc = O.oracle()
    cam = sc.camera
    gen = orc.lookat(cam.eye, cam.center, cam.up, cam.fovy, sc.width, sc.height)
    t_eye = med(lambda: orc.solve_primary(bvh, sc, gen, iteration=R.iteration))
    frame_photons = sc.n * sc.photons_per_triangle
    frame_paths = float(R.n_paths) * sc.n_bins
    ms_photon = 1e3 * t_ph * frame_photons / photons
    ms_solve = 1e3 * frame_paths / solve_paths_per_s
    return {
        "cores": lib.max_threads(), "kind": kind, "reps": reps, "statistic": "median",
        "bvh_build_2p20": {"ms": 1e3 * t_soup, "keys_per_s": (1 << 20) / t_soup,
                           "what": "BVHCPUBuilder, BUILD_OPTION_CPU_PARALLEL, 2^20 random triangles"},
        "bvh_build_scene": {"ms": 1e3 * t_scene, "triangles": int(sc.n)},
        "photon_pass": {"photons_per_s": photons / t_ph, "photons": photons,
                        "ms_at_frame_photons": ms_photon,
                        "what": f"{ppt} photons per triangle (the frame traces {sc.photons_per_triangle})"},
        "eye_pass": {"ms": 1e3 * t_eye, "rays_per_s": sc.width * sc.height / t_eye, "kind": "port",
                     "what": f"{sc.width}x{sc.height} primary rays and their shadow rays"},
        "solve": {"paths_per_s": solve_paths_per_s, "ms_at_frame_work_items": ms_solve},
        "ms_per_frame_estimate": 1e3 * t_scene + ms_photon + 1e3 * t_eye + ms_solve,
    }


def run_reference(args):
    """The reference's own CPU implementation of the path on the host cores (rank 0 only):
    LBVH, photon pass, PathCache and work list are built once on the CPU; each step solves
    a bounded random sample of the frame's work items for all 64 bins."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from palzilla_b200.scenes import event_descriptor
    lib, kind = _cpu_lib()
    orc = O.oracle()
    sc = sphere()
    b = lib.build_bvh(sc.tris)
    bvh = {"nodes": b["nodes"], "root": int(np.asarray(b["root"]).ravel()[0])}
    recs = lib.photon_trace(bvh, sc, iteration=0)
    cache = lib.cache_build(recs, capacity=1 << 22, step=sc.cell_step)
    cam = sc.camera
    gen = orc.lookat(cam.eye, cam.center, cam.up, cam.fovy, sc.width, sc.height)
    _, fd = orc.solve_primary(bvh, sc, gen, iteration=0)
    valid = (fd[:, 6:9] != 0).any(1).astype(np.uint8)
    _, pairs = orc.lookup_flatten(cache, fd[:, 0:3], valid, event_descriptor(sc.events), pair_cap=1 << 25)
    etas = sc.bin_etas()
    times, solves = [], []
    for i in range(args.warmup + args.steps):
        sel = _sample(pairs, args.ref_items, 10 + i)
        t0 = time.perf_counter()
        _, st = lib.render_pairs(2, sel, cache, fd, bvh, sc, etas)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
            solves.append(float(st[0]))
    value = sum(solves) / sum(times)
    sample = (f"solve stage only: {min(args.ref_items, len(pairs))} random (pixel, tuple) work items x 64 bins "
              f"per step from the CPU-built frame's {len(pairs)} work items")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(times)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(WORKLOAD, parallelism="host cores"),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": lib.max_threads(), "kind": kind,
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--plain-steps", type=int, default=2)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-items", type=int, default=20000)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-sort", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true", help="skip the reference's own GPU solve kernel")
    ap.add_argument("--fold-det", type=float, default=0.0, help="batched solve: fold threshold (0 = the default)")
    ap.add_argument("--image", type=int, default=0, help="image side for small profiling runs (0 = 1024)")
    ap.add_argument("--workload", default="sphere", choices=["sphere", "sort_build", "uneven_batch", "pathcuts",
                                                             "adjoint", "subdivision"],
                    help="sphere: the frame benchmark; sort_build: onesweep sort + LBVH build alone; "
                         "uneven_batch: 256 heightfield lenses of uneven size per frame; subdivision: per-tuple "
                         "domain subdivision of the lens work list")
    ap.add_argument("--batch-scenes", type=int, default=256)
    ap.add_argument("--cuts-sample", type=int, default=64)
    ap.add_argument("--sizes", default="20,22,24", help="log2 sizes of the sort_build workload")
    args = ap.parse_args()
    if args.workload == "sort_build":
        run_sort_build(args)
    elif args.workload == "uneven_batch":
        run_uneven_batch(args)
    elif args.workload == "pathcuts":
        run_pathcuts(args)
    elif args.workload == "adjoint":
        run_adjoint(args)
    elif args.workload == "subdivision":
        run_subdivision(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
