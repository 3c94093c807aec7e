#!/usr/bin/env python
"""Backprojection throughput in pixel-pulses/s on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config large|point_targets]

One step = range compression + backprojection of one synthetic aperture onto
one image (sarbp_focus).  Default workload: the large mixed-precision
configuration, 1024 frequency samples x 2048 pulses (complex64), fc 9.6 GHz,
640 MHz, 30 deg of azimuth at 8 km and 45 deg elevation, 2000 Rayleigh
scatterers, a 1024 x 1024 image over 100 m, Nfft = 8192 (2.15e9 pixel-pulses
per step).  With N GPUs every rank forms its own 1024 x 1024 slab of a
(1024 N) x 1024 image from the same aperture (weak scaling, no collective on
the data path; the ranks only meet for the timing barrier and the max).

Printed on rank 0 as one JSON line:
  value     pixel-pulses/s over all ranks, inputs resident in HBM
  e2e       the same through the C ABI with pinned host buffers: H2D of the
            phase history and geometry, D2H of the image, every step, through
            the pipelined sarbp_focus_submit/wait (copies of neighbouring
            steps overlap the kernels); the synchronous sarbp_focus beside it
  roofline  the backprojection kernel against the pipe that bounds it, with
            per-pixel-pulse algorithmic work 10 FP64 + 16 FP32 flops,
            2 transcendental (MUFU) ops and 16 B of on-chip gather, and the
            pipe peaks measured by libsarbp_probes.so on this GPU in this run
  cpu_baseline  the reference's own CPU backprojection (run_bp, compiled from
            its sources into oracle/_ref) on a bounded pulse sample, all host
            threads, rank 0 at N = 1
  reference_gpu  the reference's own GPU kernels (oracle/_ref/libref_gpu.so,
            built from cuda_BackProjectionKernels.cuh) on the same GPU and
            inputs, CUDA-event timed, with their accuracy against FP64
  kernels.adjoint  sarbp_backproject_adjoint on the same range profiles
--impl reference prints the reference CPU implementation's line alone (with
the reference GPU kernels' timing beside it).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "BP pixel·pulses/s (mixed vs FP64, ≤1e-4 rel err); autofocus sec-to-focus"
UNIT = "pixel·pulses/s"
# algorithmic work per pixel-pulse (cpuBackProjection.hpp:65-87)
WORK = {"fp64_flops": 10, "fp32_flops": 16, "sfu_ops": 2, "smem_bytes": 16}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=["large", "point_targets", "volumetric"], default="large")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample length")
    ap.add_argument("--no-autofocus", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own GPU kernels (oracle/_ref/libref_gpu.so)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-configuration section")
    ap.add_argument("--no-volumetric", action="store_true", help="skip the volumetric-configuration section")
    ap.add_argument("--grid-seconds", type=float, default=20.0, help="bound on the grid-search baseline")
    ap.add_argument("--profile", action="store_true",
                    help="one warm-up and one focus step of the workload, then two adjoint calls (mixed), "
                         "nothing else (for ncu captures)")
    ap.add_argument("--pulses", type=int, default=0, help="use only the first N pulses (profiling)")
    ap.add_argument("--log", default="", help="append the result with the run's host, GPU and seed to this "
                                               "JSON-lines file")
    ap.add_argument("--profile-reference", action="store_true",
                    help="the reference's own GPU kernels on the workload, one untimed and one timed run, "
                         "nothing else (for ncu captures)")
    ap.add_argument("--profile-precision", choices=["mixed", "fp64"], default="mixed",
                    help="engine precision of the --profile run")
    return ap.parse_args()


def make_scene(config: str, rank: int, world: int, device):
    from uncc_sar_focusing_b200 import scenes as S

    from uncc_sar_focusing_b200 import sharding as SH

    if config == "large":
        sc = S.large_scene(device=device)
        desc = ("large: 1024 samples x 2048 pulses complex64, fc 9.6 GHz / 640 MHz, 30 deg at 8 km, 45 deg el, "
                "2000 Rayleigh scatterers, 1024x1024 image over 100 m, Nfft 8192")
    elif config == "volumetric":
        sc = S.volumetric_scene(device=device)
        desc = ("volumetric: 8 passes x 1024 pulses x 512 samples, 360 deg azimuth, el 30.0-31.4 deg, 500 "
                "Rayleigh scatterers on facets in a 10 m cube, 256x256x64 voxels, Nfft 4096")
    else:
        sc = S.point_target_scene(device=device)
        desc = ("point_targets: 424 samples x 512 pulses complex64, fc 9.6 GHz / 600 MHz, 4 deg at 10 km, "
                "30 deg el, 5 unit targets, 20 dB SNR, 256x256 image at 0.08 m, Nfft 3392")
    # weak scaling: rank r forms slab r of a (world x per-GPU) image along y
    sc.grid = SH.slab_grid(SH.weak_scaling_grid(sc.grid, world), rank, world)
    return sc, desc


def config_dict(sc, desc: str, world: int) -> dict:
    """The workload as both arms report it (identical dicts for the same
    --config and world size)."""
    return {"workload": desc, "pixels_per_gpu": sc.grid.npix, "pulses": sc.num_pulses,
            "range_samples": sc.num_range_samples, "nfft": sc.nfft, "pixel_pulses_per_step_per_gpu": sc.pixel_pulses,
            "l2": "inputs larger than L2 (range-profile pair rows of every pulse, 16 B per entry)",
            "parallelism": f"{world} image slab(s), one per GPU, no data-path collective"}


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.proc = None
        try:
            self.fh = tempfile.NamedTemporaryFile("w", suffix=".csv", delete=False)
            self.path = self.fh.name
            self.proc = subprocess.Popen(["nvidia-smi", "-i", gpu_id, f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            fh = getattr(self, "fh", None)
            if fh is not None:
                fh.close()
                os.unlink(fh.name)

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        rows = []
        with open(self.path) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# CPU: the reference's run_bp (oracle/_ref) on a bounded pulse sample
# ---------------------------------------------------------------------------
def cpu_reference_rate(scene, seconds: float, threads: int = 0):
    """pixel-pulses/s of the reference CPU backprojection on this host, all
    threads, each thread focusing its own slice of pulses (the operator is a
    sum over pulses, so slices run side by side through the reference's
    public focus_SAR_image call)."""
    import numpy as np

    from oracle import oracle as O

    kind = "reference" if O.ref_available(fast=True) else "port"
    threads = threads or os.cpu_count() or 1
    npix = scene.grid.npix

    def run(pulse_slices, keep=None):
        outs = [None] * len(pulse_slices)

        def work(i, sl):
            if kind == "reference":
                outs[i] = O.reference_focus(scene, "f32", fast=True, pulses=sl)[0]
            else:
                ph, _ = O.pad_for_reference(scene, pulses=sl)
                rc = O.range_compress_ref32(ph)
                g = scene.grid
                outs[i] = O.bp_ref32(rc, scene.ant_x[sl], scene.ant_y[sl], scene.ant_z[sl], scene.slant_range[sl],
                                     scene.start_freq[sl], scene.max_wr, g.nx, g.ny, g.x0, g.y0, g.wx, g.wy)

        ts = [threading.Thread(target=work, args=(i, sl)) for i, sl in enumerate(pulse_slices)]
        t0 = time.perf_counter()
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        dt = time.perf_counter() - t0
        if keep is not None:
            keep.extend(outs)
        return dt

    Np = scene.num_pulses
    # calibrate with two pulses per thread (the reference's aperture
    # statistics need at least two pulses, uncc_sar_focusing.hpp:350-392)
    t2 = run([slice(2 * i, 2 * i + 2) for i in range(min(threads, Np // 2))])
    per_thread = max(2, min(Np // threads, int(2.0 * seconds / max(t2, 1e-3))))
    stride = max(1, Np // (per_thread * threads))
    slices = [slice(i * per_thread * stride, (i + 1) * per_thread * stride, stride) for i in range(threads)]
    slices = [s for s in slices if s.start < Np]
    total_pulses = sum(len(range(*s.indices(Np))) for s in slices)
    images = []
    dt = run(slices, images)
    out = {"value": npix * total_pulses / dt, "unit": UNIT, "cores": len(slices), "kind": kind,
           "sample": f"{total_pulses} of {Np} pulses onto the full {scene.grid.nx}x{scene.grid.ny} grid, "
                     f"{len(slices)} threads x {per_thread} pulses, {dt:.1f} s",
           "seconds": dt}
    if total_pulses == Np:  # every pulse once: the slices add up to the reference's image
        out["image"] = sum(images)
    return out


def reference_gpu_rate(scene, img64=None, reps: int = 3):
    """The reference's own GPU kernels on this GPU (oracle/_ref/libref_gpu.so:
    cuifft + cufftNormalize_1DBatch + cufftShift_1DBatch + backprojection_loop
    <float>, launched as cuda_focus_SAR_image launches them), CUDA-event
    timed; with img64 (the FP64 image) also its accuracy."""
    import numpy as np

    from oracle import oracle as O

    if not O.ref_gpu_available():
        return {"unavailable": "oracle/_ref/libref_gpu.so not built (needs the reference sources at build time)"}
    try:
        img, fft_ms, bp_ms = O.reference_gpu_focus(scene, reps=reps)
    except (ValueError, RuntimeError) as e:
        # e.g. no CUDA device on this host: the CPU line still stands
        return {"unavailable": str(e)}
    pp = scene.pixel_pulses
    out = {"value": pp / (bp_ms * 1e-3), "unit": UNIT, "bp_ms": bp_ms, "range_compress_ms": fft_ms,
           "fft_plus_bp_value": pp / ((bp_ms + fft_ms) * 1e-3),
           "kind": "reference GPU kernels (cuda_BackProjectionKernels.cuh) built for sm_100a, launched as "
                   "cuda_focus_SAR_image does; per-call allocation, plan creation and cudaDeviceReset left out",
           "reps": reps}
    if img64 is not None:
        r = img.astype(np.complex128).reshape(img64.shape)
        out["accuracy"] = {"rel_l2_vs_fp64_gpu": float(np.linalg.norm(r - img64) / np.linalg.norm(img64)),
                           "peak_phase_error_rad": peak_phase(r, img64)}
    return out


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sc, desc = make_scene(args.config, 0, 1, None if args.config != "large" else _scene_device())
    per_step = max(2.0, 150.0 / max(1, args.steps + args.warmup))
    vals = []
    info = None
    for i in range(args.warmup + args.steps):
        info = cpu_reference_rate(sc, per_step)
        if i >= args.warmup:
            vals.append(info["value"])
    value = statistics.median(vals)
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": info["seconds"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (the reference's run_bp<float>)", "data": "synthetic",
            "config": config_dict(sc, desc, world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": info["cores"], "kind": info["kind"],
                             "sample": info["sample"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_reference_gpu:
        line["reference_gpu"] = reference_gpu_rate(sc)
    if args.log:
        append_run_log(args.log, line, sc.seed)
    print(json.dumps(line), flush=True)
    return 0


def _scene_device():
    try:
        import torch

        return "cuda" if torch.cuda.is_available() else None
    except Exception:
        return None


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def probe_peaks():
    from uncc_sar_focusing_b200 import build as B

    L = ctypes.CDLL(B.PROBE_LIB)
    L.sarbp_probe.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                              ctypes.POINTER(ctypes.c_float)]
    out = {}
    for which, name, iters, per_op in ((0, "fp32_flops_per_s", 4096, 2.0), (1, "fp64_flops_per_s", 2048, 2.0),
                                       (2, "sfu_ops_per_s", 1024, 2.0), (3, "smem_bytes_per_s", 2048, 16.0)):
        rate, ms = ctypes.c_double(), ctypes.c_float()
        st = L.sarbp_probe(which, iters, ctypes.byref(rate), ctypes.byref(ms))
        if st != 0:
            raise RuntimeError(f"probe {name} failed: {st}")
        out[name] = rate.value * per_op
    return out


def roofline_bound(peaks):
    t = {"fp64": WORK["fp64_flops"] / peaks["fp64_flops_per_s"], "fp32": WORK["fp32_flops"] / peaks["fp32_flops_per_s"],
         "sfu": WORK["sfu_ops"] / peaks["sfu_ops_per_s"], "smem": WORK["smem_bytes"] / peaks["smem_bytes_per_s"]}
    bound = max(t, key=t.get)
    return bound, 1.0 / t[bound], t


def autofocus_section(dev, grid_seconds: float):
    """Motion-error autofocus on the autofocus configuration (config-1
    geometry, 1024 pulses x 512 samples, 512^2 image; per-axis seeded cubic
    track error up to 1.5 m plus a 1 mm/pulse random walk): the gradient
    pipeline (cubic coefficients, then per-pulse line of sight, then PGA)
    against the reference's multiresolution grid search restated on the same
    engine (the reference's searched coefficients -- slope and quadratic term
    per axis -- 5 points each, halving boxes, every grid point scored with the
    reference's own 2-D DFT cost), bounded to grid_seconds.  Both final images
    carry the Shannon entropy and the reference's two costs (DFT and column
    histogram).  Seconds-to-focus = time for each method to reach the grid
    search's final Shannon entropy."""
    import numpy as np
    import torch

    from uncc_sar_focusing_b200 import autofocus as AF
    from uncc_sar_focusing_b200 import autograd as A
    from uncc_sar_focusing_b200 import focusing
    from uncc_sar_focusing_b200 import scenes as S

    sc = S.motion_error_scene(device=dev)
    torch.cuda.empty_cache()
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    ax, ay, az, r0, f0 = (d(v) for v in (sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq))
    with focusing.Plan.for_scene(sc, "mixed") as plan:
        plan.range_compress(d(sc.phase_history))
        ent = lambda x, y, z, r=r0: float(A.image_entropy(plan.backproject(x, y, z, r, f0)))  # noqa: E731
        e_measured = ent(ax, ay, az)
        e_true = ent(*(d(getattr(sc, a) + sc.true_error[i]) for i, a in enumerate(("ant_x", "ant_y", "ant_z"))))
        # warm-up past the descent's graph capture (its first 10 steps run eagerly)
        AF.focus_motion_error(plan, ax, ay, az, r0, f0, cubic_iters=15, los_iters=15, pga_iters=1)
        # three runs: the pipeline is deterministic (same entropies each run),
        # its wall time is not (a host stall early in a run delays the steps
        # that reach the target); the run of median total time is reported
        runs = [AF.focus_motion_error(plan, ax, ay, az, r0, f0) for _ in range(3)]
        runs.sort(key=lambda r: r["seconds"])
        grad = runs[1]
        motion = AF.CubicMotion(ax, ay, az)
        searches = {}
        for cost in ("reference_dft", "entropy"):
            g = AF.grid_search_autofocus(plan, motion, r0, f0, span=1.5, points=5, levels=4, batch=128,
                                         deadline_s=grid_seconds, cost=cost)
            a = motion.track(g.theta)
            img_g = plan.backproject(a[0].contiguous(), a[1].contiguous(), a[2].contiguous(), r0, f0)
            searches[cost] = (g, AF.focus_metrics(img_g))
        metrics_grad = AF.focus_metrics(grad["image"])

    def search_entry(cost):
        g, metrics = searches[cost]
        e = metrics["shannon_entropy"]
        reach = [AF.time_to_entropy(r["timeline"], e) for r in runs]
        t = None if any(x is None for x in reach) else sorted(reach)[1]  # median of the three runs
        return {"cost": cost, "entropy": e, "seconds": g.seconds, "images": g.images_formed,
                "levels_done": len(g.history), "bounded_to_s": grid_seconds, "final_image": metrics,
                "searched": "slope and quadratic term of each axis (the reference's quadratic search without "
                            "its velocity scale), 5 points each, box halved per level; the 12 cubic coefficients "
                            "at 5 points would be 5^12 images per level",
                "sec_to_focus": {"target_entropy": e, "gradient_s": t, "grid_search_s": g.seconds,
                                 "speedup": (g.seconds / t) if t else None,
                                 "gradient_s_runs": reach}}
    return {
        "workload": "autofocus: 9.6 GHz / 600 MHz, 4 deg at 10 km, 30 deg el, 1024 pulses x 512 samples, 512^2 "
                    "image at 0.08 m, 5 targets, 20 dB SNR; track error per axis = seeded cubic (1.5 m peak) + "
                    "1 mm/pulse random walk",
        "entropy_measured_track": e_measured, "entropy_true_track": e_true,
        "gradient": {"entropy_cubic": grad["entropy_cubic"], "entropy_line_of_sight": grad["entropy_los"],
                     "entropy_pga": grad["entropy_pga"], "seconds": grad["seconds"],
                     "seconds_runs": [r["seconds"] for r in runs],
                     "final_image": metrics_grad,
                     "cubic_steps": grad["cubic_steps"],
                     "stages": "Adam on 12 cubic coefficients (up to 300 it, stopped when the best entropy "
                               "gains < 2e-3 nats per 25 it) -> Adam on 1024 per-pulse ranges (200 it) -> PGA "
                               "(PGA.m semantics, on the device); gradients from the adjoint kernel"},
        # the reference's own method: every grid point scored with its DFT
        # cost; that cost rewards low-frequency energy of the 8-bit image, so
        # its optimum need not be the sharpest image
        "grid_search": search_entry("reference_dft"),
        # the same search scored with the gradient pipeline's objective
        "grid_search_entropy": search_entry("entropy"),
        # headline: time for the gradient pipeline to reach the final Shannon
        # entropy of the stronger of the two searches
        "sec_to_focus": min((search_entry(c)["sec_to_focus"] for c in searches),
                            key=lambda d: d["target_entropy"]),
    }


def batched_section(dev, steps: int):
    """Batched configuration: (a) 256 motion hypotheses (seeded perturbations
    of the autofocus scene's true cubic coefficients, 5 cm per coefficient) x
    a 512^2 image from one 1024 x 512 phase history, one launch
    (sarbp_backproject_hypotheses); (b) 64 independent point-target scenes of
    seeded uniform sizes (128^2-1024^2 pixels at 0.1 m, 256-2048 pulses of
    512 samples, 5-500 scatterers) focused as one batch (sarbp_batch_*): range
    compression and ONE backprojection launch over all scenes' tiles, a
    captured CUDA graph replayed per call, tile shape autotuned; throughput,
    per-image completion latency p50/p99 (GPU clock, from the call's start),
    and the same scenes focused one plan at a time beside it."""
    import numpy as np
    import torch

    from uncc_sar_focusing_b200 import autofocus as AF
    from uncc_sar_focusing_b200 import focusing
    from uncc_sar_focusing_b200 import scenes as S

    stream = torch.cuda.current_stream()

    def timed(fn, n):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(n):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / n

    d = lambda a: torch.as_tensor(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    out = {}
    # (a) hypotheses
    sc = S.motion_error_scene(device=dev)
    torch.cuda.empty_cache()
    H = 256
    ax, ay, az, r0, f0 = (d(v) for v in (sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq))
    motion = AF.CubicMotion(ax, ay, az)
    rng = np.random.default_rng(5)
    theta = torch.as_tensor(sc.true_cubic[None] + rng.normal(0.0, 0.05, size=(H, 3, 4)), device=dev)
    tracks = torch.stack([motion.track(theta[h]) for h in range(H)])  # [H, 3, Np]
    hx, hy, hz = (tracks[:, i].contiguous() for i in range(3))
    hr0 = r0.expand(H, -1).contiguous()
    hf0 = f0.expand(H, -1).contiguous()
    with focusing.Plan.for_scene(sc, "mixed", device=torch.cuda.current_device()) as plan:
        plan.range_compress(d(sc.phase_history))
        imgs = torch.empty((H, 1, sc.grid.nx, sc.grid.ny), dtype=torch.complex64, device=dev)
        step = lambda: plan.backproject_hypotheses(hx, hy, hz, hr0, hf0, out=imgs)  # noqa: E731
        step()
        plan.check()
        ms = timed(step, max(2, steps // 2))
        plan.check()
    pp = H * sc.grid.npix * sc.num_pulses
    out["hypotheses"] = {"workload": f"{H} hypotheses x {sc.grid.nx}x{sc.grid.ny} image x {sc.num_pulses} pulses "
                                     f"x {sc.num_range_samples} samples, one launch",
                         "pixel_pulses": pp, "ms": ms, "value": pp / (ms * 1e-3), "unit": UNIT}
    del imgs, tracks, hx, hy, hz, hr0, hf0
    torch.cuda.empty_cache()

    # (b) uneven scenes
    rng = np.random.default_rng(55)
    scenes = []
    for i in range(64):
        n = int(rng.integers(128, 1025))
        npulse = int(rng.integers(256, 2049))
        nt = int(rng.integers(5, 501))
        scenes.append(S.point_target_scene(K=512, Np=npulse, n=n, spacing=0.1, n_targets=nt, nfft=4096,
                                           seed=100 + i, extent=0.08 * n, device=dev))
    args = [tuple(d(getattr(s_, a)) for a in ("phase_history", "ant_x", "ant_y", "ant_z", "slant_range",
                                              "start_freq")) for s_ in scenes]
    pp_b = sum(s_.pixel_pulses for s_ in scenes)
    with focusing.Batch(scenes, device=torch.cuda.current_device()) as batch:
        default_info = batch.info
        imgs = batch.new_images(dev)
        t0 = time.perf_counter()
        best_ms = batch.autotune(args, imgs)
        tune_s = time.perf_counter() - t0
        batch.focus(args, imgs)
        batch.wait()
        ms_b = timed(lambda: batch.focus(args, imgs), max(3, steps // 2))
        lat = batch.wait()
        info = batch.info
        batch_img0 = imgs[0].clone()
    # the same scenes, one plan and one focus call each
    plans = [focusing.Plan.for_scene(s_, "mixed", device=torch.cuda.current_device()) for s_ in scenes]
    seq_imgs = [p.new_image(dev) for p in plans]
    seq = lambda: [p.focus(*a, out=o) for p, a, o in zip(plans, args, seq_imgs)]  # noqa: E731
    seq()
    ms_seq = timed(seq, 2)
    for p in plans:
        p.check()
    rel = float((seq_imgs[0] - batch_img0).abs().pow(2).sum().sqrt() / seq_imgs[0].abs().pow(2).sum().sqrt())
    for p in plans:
        p.close()
    del seq_imgs, plans, imgs
    torch.cuda.empty_cache()
    out["uneven_scenes"] = {
        "workload": "64 point-target scenes, seeded uniform sizes 128^2-1024^2 pixels at 0.1 m, 256-2048 pulses "
                    "x 512 samples (Nfft 4096), 5-500 scatterers; one batch call = range compression + one "
                    "backprojection launch over all scenes, CUDA graph replay",
        "pixel_pulses": pp_b, "ms": ms_b, "value": pp_b / (ms_b * 1e-3), "unit": UNIT,
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "max": float(lat.max()), "of": "per-image completion after the call's start, GPU clock"},
        "graph": bool(info["graph"]),
        "schedule": "one CTA per tile, scene order" if info["per_tile"] else "units split over resident CTAs",
        "autotune": {"tile_rows": 8 * info["tile_mx"], "stage_pulses": info["stage_pulses"],
                     "default_tile_rows": 8 * default_info["tile_mx"],
                     "default_stage_pulses": default_info["stage_pulses"], "best_ms": best_ms,
                     "seconds": tune_s},
        "sequential_plans": {"ms": ms_seq, "value": pp_b / (ms_seq * 1e-3),
                             "batch_speedup": ms_seq / ms_b, "rel_l2_scene0_batch_vs_plan": rel},
    }
    return out


def volumetric_section(dev, steps: int):
    """Volumetric configuration at full size: 8 circular passes at elevations
    30.0-31.4 deg (0.2 deg steps), 360 deg of azimuth, 1024 pulses per pass x
    512 samples (9.6 GHz / 600 MHz, 10 km), 500 Rayleigh scatterers on random
    planar facets in a 10 m cube, 256 x 256 x 64 voxels (3.44e10 voxel-pulses
    per focus): mixed and FP64 throughput, and the relative L2 of every z-slice
    of the mixed image against the FP64 path."""
    import numpy as np
    import torch

    from uncc_sar_focusing_b200 import focusing
    from uncc_sar_focusing_b200 import scenes as S

    stream = torch.cuda.current_stream()

    def timed(fn, n):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(n):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / n

    sc = S.volumetric_scene(device=dev)
    torch.cuda.empty_cache()
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    ph = d(sc.phase_history)
    geo = [d(v) for v in (sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq)]
    dv = torch.cuda.current_device()
    with focusing.Plan.for_scene(sc, "mixed", device=dv) as plan:
        img = plan.new_image(dev)
        plan.focus(ph, *geo, out=img)
        plan.check()
        ms = timed(lambda: plan.focus(ph, *geo, out=img), max(3, steps // 2))
        plan.check()
    with focusing.Plan.for_scene(sc, "fp64", device=dv) as plan64:
        img64 = plan64.new_image(dev)
        plan64.focus(ph, *geo, out=img64)
        plan64.check()
        ms64 = timed(lambda: plan64.focus(ph, *geo, out=img64), 2)
        plan64.check()
    diff = (img.to(torch.complex128) - img64).abs().pow(2).sum(dim=(1, 2)).sqrt()
    per_slice = (diff / img64.abs().pow(2).sum(dim=(1, 2)).sqrt()).cpu().numpy()
    total = float(diff.pow(2).sum().sqrt() / img64.abs().pow(2).sum().sqrt())
    pp = sc.pixel_pulses
    del img, img64
    torch.cuda.empty_cache()
    return {
        "workload": "volumetric: 8 passes x 1024 pulses x 512 samples, 360 deg azimuth, el 30.0-31.4 deg, "
                    "500 Rayleigh scatterers on facets in a 10 m cube, 256x256x64 voxels, Nfft 4096",
        "voxel_pulses": pp, "ms": ms, "value": pp / (ms * 1e-3), "unit": UNIT,
        "fp64": {"ms": ms64, "value": pp / (ms64 * 1e-3), "mixed_speedup": ms64 / ms},
        "rel_l2_vs_fp64": {"total": total, "slice_min": float(per_slice.min()),
                           "slice_median": float(np.median(per_slice)), "slice_max": float(per_slice.max()),
                           "tolerance": 1e-4},
    }


def append_run_log(path: str, line: dict, seed: int) -> None:
    """One JSON line per run: the result line, the scene seed, the command,
    and the host and GPU it ran on (CPU model and cores, GPU name, SMs,
    memory, compute capability, driver, CUDA and torch versions)."""
    import platform

    import torch

    cpu = platform.processor() or ""
    try:
        with open("/proc/cpuinfo") as fh:
            for row in fh:
                if row.startswith("model name"):
                    cpu = row.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    gpu = {}
    if torch.cuda.is_available():
        prop = torch.cuda.get_device_properties(torch.cuda.current_device())
        gpu = {"name": prop.name, "sms": prop.multi_processor_count, "memory_gib": prop.total_memory / 2**30,
               "cc": f"{prop.major}.{prop.minor}", "cuda": torch.version.cuda}
        try:
            out = subprocess.run(["nvidia-smi", "--query-gpu=driver_version", "--format=csv,noheader"],
                                 capture_output=True, text=True, timeout=20)
            gpu["driver"] = out.stdout.strip().splitlines()[0] if out.returncode == 0 and out.stdout else None
        except Exception:
            gpu["driver"] = None
    rec = {"time": time.strftime("%Y-%m-%dT%H:%M:%S%z"), "argv": sys.argv[1:], "scene_seed": seed,
           "host": {"cpu": cpu, "cores": os.cpu_count()}, "gpu": gpu, "torch": torch.__version__, "result": line}
    with open(path, "a") as fh:
        fh.write(json.dumps(rec) + "\n")


def profiled_traffic(config: str):
    """DRAM bytes per backprojection launch from the committed ncu summary of
    this workload (profiles/), or None."""
    if config != "large":
        return None
    p = os.path.join(ROOT, "profiles", "bp_mixed_large.md")
    try:
        with open(p) as fh:
            for line in fh:
                if line.startswith("dram_bytes_per_launch:"):
                    return int(line.split(":")[1])
    except OSError:
        pass
    return None


def peak_phase(a, b) -> float:
    """Phase of a relative to b (rad) at the magnitude peak of b."""
    import numpy as np

    i = int(np.argmax(np.abs(b).ravel()))
    return float(np.angle(a.ravel()[i] * np.conj(b.ravel()[i])))


def measured_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def gpu_arm(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    from uncc_sar_focusing_b200 import focusing

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    local = local % max(1, torch.cuda.device_count())
    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    if world > 1:
        from datetime import timedelta

        # NCCL for the barrier and the max over ranks; SARBP_BENCH_BACKEND=gloo
        # runs the multi-rank path with several ranks on one GPU (smoke tests)
        backend = os.environ.get("SARBP_BENCH_BACKEND", "nccl")
        kw = {"device_id": torch.device(dev)} if backend == "nccl" else {}
        dist.init_process_group(backend, timeout=timedelta(seconds=300), **kw)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev if dist.get_backend() == "nccl" else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    sc, desc = make_scene(args.config, rank, world, dev)
    pp = sc.pixel_pulses
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    ph_d = d(sc.phase_history)
    geo_d = [d(v) for v in (sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq)]
    plan = focusing.Plan.for_scene(sc, "mixed", device=local)
    img_d = plan.new_image(dev)
    stream = torch.cuda.current_stream()

    def timed(fn, n):
        barrier()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(n):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        barrier()
        return a.elapsed_time(b)

    step = lambda: plan.focus(ph_d, *geo_d, out=img_d)  # noqa: E731
    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    plan.check()

    props = torch.cuda.get_device_properties(local)
    uuid = str(getattr(props, "uuid", ""))
    gpu_id = uuid if uuid.startswith("GPU-") else (f"GPU-{uuid}" if uuid else str(local))
    # clocks are sampled from here to the end of the kernel-level timings
    # (the timed steps alone can be shorter than the sampling period)
    sampler = ClockSampler(gpu_id)
    ms = timed(step, args.steps)
    ms = max_over_ranks(ms)
    ms_step = ms / args.steps
    value = world * pp / (ms_step * 1e-3)

    # kernel-level timings: range compression alone, backprojection alone
    reps = max(3, args.steps)
    rc_ms = max_over_ranks(timed(lambda: plan.range_compress(ph_d), reps)) / reps
    plan.focus(ph_d, *geo_d, out=img_d)
    bp_ms = max_over_ranks(timed(lambda: plan.backproject(*geo_d, out=img_d), reps)) / reps
    plan.check()
    # the adjoint (dL/d antenna position and R0) on the same range profiles,
    # with the image itself as the upstream gradient
    grad_img = img_d.clone()
    plan.backproject_adjoint(*geo_d, grad_img)
    adj_ms = max_over_ranks(timed(lambda: plan.backproject_adjoint(*geo_d, grad_img), reps)) / reps
    plan.check()
    del grad_img
    # a second of back-to-back steps so the clock record covers steady load
    t_end = time.perf_counter() + 1.0
    while time.perf_counter() < t_end:
        for _ in range(20):
            step()
        torch.cuda.synchronize()
    clocks = sampler.stop()

    # FP64 GPU path on the same inputs: accuracy reference and the FP64 baseline
    img_mixed = img_d.clone()
    plan64 = focusing.Plan.for_scene(sc, "fp64", device=local)
    img64 = plan64.new_image(dev)
    plan64.focus(ph_d, *geo_d, out=img64)
    torch.cuda.synchronize()
    plan64.check()
    fp64_ms = max_over_ranks(timed(lambda: plan64.backproject(*geo_d, out=img64), max(2, args.steps // 3))) / max(
        2, args.steps // 3)
    diff = (img_mixed.to(torch.complex128) - img64).abs().pow(2).sum().sqrt()
    rel = float(diff / img64.abs().pow(2).sum().sqrt())
    img64_h = img64[0].cpu().numpy()
    phase_err = peak_phase(img_mixed[0].cpu().numpy(), img64_h)
    del plan64, img64
    torch.cuda.empty_cache()

    # end to end through the C ABI with pinned host buffers
    ph_h = torch.empty(ph_d.shape, dtype=ph_d.dtype, pin_memory=True)
    ph_h.copy_(ph_d.cpu())
    geo_h = []
    for v in geo_d:
        h = torch.empty(v.shape, dtype=v.dtype, pin_memory=True)
        h.copy_(v.cpu())
        geo_h.append(h)
    img_h = [torch.empty(img_d.shape, dtype=img_d.dtype, pin_memory=True) for _ in range(2)]
    ph_n, geo_n, img_n = ph_h.numpy(), [g.numpy() for g in geo_h], [h.numpy() for h in img_h]

    def e2e_run(n, pipelined):
        # every step uploads its aperture and downloads its image; pipelined
        # steps overlap step i's kernels with i+1's upload and i-1's download
        barrier()
        t0 = time.perf_counter()
        for i in range(n):
            if pipelined:
                plan.focus_submit(ph_n, *geo_n, out=img_n[i % 2])
            else:
                plan.focus(ph_n, *geo_n, out=img_n[i % 2])
        plan.focus_wait()
        return max_over_ranks(time.perf_counter() - t0) / n

    # a throughput figure: at least 50 submissions, so that filling and
    # draining the two-slot pipeline (the first upload and the last download
    # are not overlapped) weighs little against the steady state
    e2e_n = max(args.steps, 50)
    e2e_run(3, True)
    e2e_s = e2e_run(e2e_n, True)
    e2e_sync_s = e2e_run(e2e_n, False)
    h2d = ph_n.nbytes + sum(g.nbytes for g in geo_n)
    d2h = img_n[0].nbytes
    ref = img_mixed.cpu().numpy()
    for h in img_n:
        assert np.array_equal(h, ref)

    line = None
    if rank == 0:
        peaks = probe_peaks()
        bound, roof, tmin = roofline_bound(peaks)
        bp_rate = pp / (bp_ms * 1e-3)
        hbm, hbm_kind = measured_hbm()
        info = plan.info
        # range compression moves at least the phase history in and the pair
        # rows the backprojection reads out: 8 B per sample + 16 B per entry
        # (nfft + 1 entries per pulse)
        rc_bytes = sc.num_pulses * (sc.num_range_samples * 8 + (sc.nfft + 1) * 16)
        mixed_speedup = fp64_ms / bp_ms
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            # the north-star ratio first, so that a truncated record keeps it:
            # backprojection kernel, mixed precision against all-FP64, same
            # inputs and GPU, and the mixed image's error against the FP64 one
            "mixed_vs_fp64_gpu": {"bp_speedup": mixed_speedup, "rel_l2": rel, "peak_phase_error_rad": phase_err,
                                  "tolerance": 1e-4, "mixed_bp_ms": bp_ms, "fp64_bp_ms": fp64_ms},
            "dtype": "f32+f64 (FP64 per-tile geometry, FP32 per pixel-pulse)",
            "data": "synthetic",
            "config": config_dict(sc, desc, world),
            "plan_workspace_mib": plan.workspace_bytes / 2**20,
            "accuracy": {"rel_l2_mixed_vs_fp64_gpu": rel, "peak_phase_error_rad": phase_err, "tolerance": 1e-4,
                         "note": "against the FP64 GPU path on the full image; that path is checked against "
                                 "the FP64 CPU oracle on small scenes (1e-13) and on every pixel of this one (1.7e-11; "
                                 "tests/test_bp_gpu.py::test_large_config_full_image)"},
            "fp64_gpu": {"bp_value": pp / (fp64_ms * 1e-3), "unit": UNIT, "mixed_speedup": mixed_speedup},
            "e2e": {"value": world * pp / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e_s * 1e3, "steps": e2e_n,
                    "api": "sarbp_focus_submit/sarbp_focus_wait, pinned host buffers",
                    "synchronous": {"value": world * pp / e2e_sync_s, "ms_per_step": e2e_sync_s * 1e3,
                                    "api": "sarbp_focus, pinned host buffers"}},
            # per step: range compression (one fused kernel, or taper + pair
            # rows around cuFFT, whose kernel is the library's and not
            # counted), the backprojection (+ its fix-up when the tiles are
            # split over the resident CTAs)
            "gpu_launches": ((1 if info["fused_range_compression"] else 2) + info["kernels_per_backproject"])
            * args.steps,
            "kernels": {"bp_ms": bp_ms, "range_compress_ms": rc_ms,
                        "adjoint": {"ms": adj_ms, "value": pp / (adj_ms * 1e-3), "unit": UNIT,
                                    "vs_forward_bp_time": adj_ms / bp_ms,
                                    "what": "sarbp_backproject_adjoint: adjoint kernel + tile sum, "
                                            "dL/d(antenna xyz, R0) for all pulses"},
                        "range_compress_fused": bool(info["fused_range_compression"]),
                        "range_compress_hbm": {"bytes": rc_bytes, "achieved_gbs": rc_bytes / (rc_ms * 1e-3) / 1e9,
                                               "peak_gbs": hbm, "peak_kind": hbm_kind,
                                               "frac": rc_bytes / (rc_ms * 1e-3) / 1e9 / hbm}},
            "roofline": {"bound": bound, "achieved": bp_rate, "peak": roof, "unit": UNIT, "frac": bp_rate / roof,
                         "traffic": None, "peak_kind": "measured in this run by libsarbp_probes.so",
                         "work_per_pixel_pulse": WORK, "pipe_peaks": peaks,
                         "t_min_per_pixel_pulse_s": tmin},
            "clocks": clocks,
        }
        if world == 1 and not args.no_autofocus:
            line["autofocus"] = autofocus_section(dev, args.grid_seconds)
        if world == 1 and not args.no_batched:
            line["batched"] = batched_section(dev, args.steps)
        if world == 1 and not args.no_volumetric:
            vol = volumetric_section(dev, args.steps)
            line["volumetric"] = vol
            if "fp64" in vol:
                line["mixed_vs_fp64_gpu"]["volumetric_bp_speedup"] = vol["fp64"]["mixed_speedup"]
                line["mixed_vs_fp64_gpu"]["volumetric_rel_l2"] = vol["rel_l2_vs_fp64"]["total"]
        traffic = profiled_traffic(args.config)
        if traffic is not None:
            line["roofline"]["traffic"] = traffic
            line["roofline"]["traffic_source"] = "profiles/bp_mixed_large.md (ncu dram__bytes_read+write, per launch)"
            # the same kernel against the HBM roofline: profiled DRAM bytes per
            # launch over this run's CUDA-event time, measured copy bandwidth
            hbm_ach = traffic / (bp_ms * 1e-3) / 1e9
            line["roofline"]["hbm"] = {"bound": "hbm", "achieved": hbm_ach, "peak": hbm, "unit": "GB/s",
                                       "frac": hbm_ach / hbm, "peak_kind": hbm_kind,
                                       "what": "backprojection kernel's DRAM traffic: it is bound by the MUFU "
                                               "pipe and issue, not by HBM"}
        if world == 1 and not args.no_cpu_baseline:
            cb = cpu_reference_rate(sc, args.cpu_seconds)
            cb.pop("seconds", None)
            ref_img = cb.pop("image", None)
            if ref_img is not None:
                # the reference's float backprojection against the FP64 path
                r = np.asarray(ref_img, dtype=np.complex128).reshape(img64_h.shape)
                cb["accuracy"] = {"rel_l2_vs_fp64_gpu": float(np.linalg.norm(r - img64_h) / np.linalg.norm(img64_h)),
                                  "peak_phase_error_rad": peak_phase(r, img64_h)}
            line["cpu_baseline"] = cb
        if world == 1 and not args.no_reference_gpu:
            rg = reference_gpu_rate(sc, img64_h)
            if "value" in rg:
                rg["bp_speedup_of_mixed"] = bp_rate / rg["value"]
            line["reference_gpu"] = rg
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        if args.log:
            append_run_log(args.log, line, sc.seed)
        print(json.dumps(line), flush=True)
    return 0


def profile_arm(args):
    """A single focus of the workload after one warm-up, then (mixed
    precision) two adjoint calls with the image as the upstream gradient, with
    the scene synthesis temporaries released first so that a profiler's
    per-pass memory save/restore only covers the plan and the inputs."""
    import numpy as np
    import torch

    from uncc_sar_focusing_b200 import focusing

    torch.cuda.set_device(0)
    sc, _ = make_scene(args.config, 0, 1, "cuda")
    if args.pulses:
        n = args.pulses
        sc.phase_history = sc.phase_history[:n]
        sc.ant_x, sc.ant_y, sc.ant_z = sc.ant_x[:n], sc.ant_y[:n], sc.ant_z[:n]
        sc.slant_range, sc.start_freq = sc.slant_range[:n], sc.start_freq[:n]
    torch.cuda.empty_cache()
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()  # noqa: E731
    ph = d(sc.phase_history)
    geo = [d(v) for v in (sc.ant_x, sc.ant_y, sc.ant_z, sc.slant_range, sc.start_freq)]
    with focusing.Plan.for_scene(sc, args.profile_precision, device=0) as plan:
        img = plan.new_image("cuda")
        for _ in range(2):
            plan.focus(ph, *geo, out=img)
        if args.profile_precision == "mixed":
            for _ in range(2):
                plan.backproject_adjoint(*geo, img)
        torch.cuda.synchronize()
        plan.check()
    print(json.dumps({"profile": args.config, "pulses": sc.num_pulses, "pixel_pulses": sc.pixel_pulses}))
    return 0


def profile_reference_arm(args):
    """The reference's GPU kernels (oracle/_ref/libref_gpu.so) on the
    workload: scene synthesis, then one untimed and one timed repetition."""
    import torch

    from oracle import oracle as O

    torch.cuda.set_device(0)
    sc, _ = make_scene(args.config, 0, 1, "cuda")
    torch.cuda.empty_cache()
    _, fft_ms, bp_ms = O.reference_gpu_focus(sc, reps=1)
    print(json.dumps({"profile_reference": args.config, "bp_ms": bp_ms, "range_compress_ms": fft_ms}))
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.profile:
        return profile_arm(args)
    if args.profile_reference:
        return profile_reference_arm(args)
    return gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
