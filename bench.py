"""Benchmark: batched multi-camera tracking front-end on B200.

Workload ("batched multicamera"): 32 cameras of uneven resolution (12 x 640x480,
12 x 1280x720, 8 x 1920x1200, uint8), each with its own seeded synthetic scene and similarity warp,
and 300..3000 features per camera (seeded).  One step is one frame of all 32 cameras: build the
current pyramids and gradient pyramids, track every feature from the previous frame (pyramidal LK),
and select new Shi-Tomasi features with the survivors as alive tracks.  The step runs as one CUDA
graph over flattened (camera, tile) and (camera, track) work lists (`Batch.run`).

metric: tracks/s = features attempted per step (all cameras) / step time.
  value : device time, inputs resident in HBM (each step restores the tracks on the device).
  e2e   : the public API with host buffers: per step the 32 frames and the tracks are copied in
          from pinned host memory and the tracked records and new features are copied back.
Also reported: the plain per-camera launch sequence (`Batch.run_plain`, the drop-in pattern), the
dominant kernel's roofline, the CPU baseline (the restated reference CPU tracker), clocks.

Multi-GPU (torchrun, --gpus N): each rank runs its own 32-camera workload (cameras shard with no
exchange step; weak scaling); value = all tracks / max-over-ranks time.
--impl reference: times the restated reference CPU tracker (oracle/cpu_tracker.c) on the host
cores over the same workload, rank 0 only.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "LK tracks/s, batched multicamera frame step (pyramid+gradients+Shi-Tomasi+LK)"
UNIT = "tracks/s"
WORKLOAD = ("multicam32: 32 cameras (12x640x480, 12x1280x720, 8x1920x1200 uint8), 300-3000 features each, "
            "pyramid (6-7 levels) + gradients + Shi-Tomasi selection + pyramidal LK per frame")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the LK adjoint measurement")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the parity check against the reference's own kernels (after the timed regions)")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other workloads (stereo plain, 100-frame sequence, fwd+bwd stream, L2R, affine)")
    ap.add_argument("--profile", choices=["pyramid", "lk", "select", "step", "implicit", "unrolled", "affine"],
                    default=None,
                    help="for an ncu capture: run only this part of the step (inside NVTX ranges named "
                         "'part'), whole batched steps (ranges named 'step'), or the LK adjoint workload's "
                         "forward and backward in one mode (ranges 'fwd', 'bwd'), warmup + steps times, or "
                         "the affine tracker's workload alone")
    ap.add_argument("--adj-cams", type=int, default=None,
                    help="cameras of the LK adjoint workload under --profile implicit/unrolled (a smaller case "
                         "for an ncu capture; default 8)")
    return ap.parse_args()


def _pair(args):
    from cuvslam_b200 import synthetic

    cam, w, h = args
    p, n, _ = synthetic.frame_pair(cam, w, h)
    return p, n


def workload(seed_offset=0):
    """Frames (previous, next) and feature budgets of the 32 cameras.  Drawn in a spawned process
    pool before any CUDA call."""
    import multiprocessing as mp

    from cuvslam_b200 import synthetic

    shapes = synthetic.MULTICAM_SHAPES
    counts = synthetic.multicam_feature_counts()
    jobs = [(i + 100 * seed_offset, w, h) for i, (w, h) in enumerate(shapes)]
    with mp.get_context("spawn").Pool(min(len(jobs), os.cpu_count() or 1)) as pool:
        pairs = pool.map(_pair, jobs)
    return shapes, counts, [p for p, _ in pairs], [n for _, n in pairs]


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        import tempfile

        self.path = os.path.join(tempfile.gettempdir(), f"clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.fh, stderr=subprocess.DEVNULL)
            import atexit

            atexit.register(self.__exit__)  # stopped even if the measurements in between raise
            # the sampler takes a moment to start: wait (at most 5 s) for its first sample so that the
            # timed region is covered from its start
            t0 = time.time()
            while time.time() - t0 < 5.0 and os.path.getsize(self.path) == 0 and self.proc.poll() is None:
                time.sleep(0.02)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None and self.proc.poll() is None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None:
            return None
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                try:
                    rows.append((float(parts[0]), float(parts[1]), parts[3:7]))
                except ValueError:
                    pass
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for _, _, r in rows for k in range(4) if r[k].lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def reduce_max(x, dist, device):
    """Max over ranks of a per-rank scalar (timing); identity without a process group."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([float(x)], device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(x, dist, device):
    """Sum over ranks of a per-rank count; identity without a process group."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([float(x)], device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return int(round(t.item()))


def throughput(units_all_ranks, steps, ms_max):
    """Whole-job units/s: the units all ranks processed per step, over the slowest rank's time."""
    return units_all_ranks * steps / (ms_max / 1e3)


def cpu_reference_step_fn(shapes, counts, prevs, nexts, nthreads, features_parallel=False):
    """A callable running one frame step of the restated reference CPU tracker over all cameras: one
    camera per thread, or (features_parallel) the cameras in turn with each camera's tracking spread
    over the threads."""
    from oracle import oracle as O

    prev_cams = [O.CpuCamera(w, h).build(p) for (w, h), p in zip(shapes, prevs)]
    cur_cams = [O.CpuCamera(w, h) for (w, h) in shapes]
    feats = [c.select(None, n) for c, n in zip(prev_cams, counts)]
    attempted = sum(len(f) for f in feats)

    def step():
        return O.cpu_frame_step(prev_cams, cur_cams, nexts, feats, None, counts, nthreads, features_parallel)

    return step, attempted


def host_cpu():
    """The host's CPU model and the cores this process may use."""
    model = None
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    try:
        usable = len(os.sched_getaffinity(0))
    except AttributeError:
        usable = os.cpu_count() or 1
    return {"cpu_model": model, "nproc": os.cpu_count(), "usable_cores": usable}


def cpu_baseline_variants(shapes, counts, prevs, nexts, nthreads, reps):
    """Times both parallel forms of the restated CPU tracker (reps steps each after one warm-up);
    returns ({variant: tracks/s}, fastest variant's step function, attempted tracks per step)."""
    out, best = {}, None
    for name, fp in (("camera_per_thread", False), ("features_parallel", True)):
        step, att = cpu_reference_step_fn(shapes, counts, prevs, nexts, nthreads, fp)
        step()
        t0 = time.perf_counter()
        for _ in range(reps):
            step()
        out[name] = att * reps / (time.perf_counter() - t0)
        if best is None or out[name] > out[best[0]]:
            best = (name, step, att)
    return out, best


def run_reference(args, rank):
    if rank != 0:
        return
    cpu = host_cpu()
    nthreads = cpu["usable_cores"]
    shapes, counts, prevs, nexts = workload()
    variants, (variant, step, attempted) = cpu_baseline_variants(shapes, counts, prevs, nexts, nthreads, 1)
    for _ in range(max(args.warmup, 1)):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    value = attempted * args.steps / dt
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "tracks_per_step": attempted},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port",
                             "sample": f"full 32-camera frame step x {args.steps} steps, {variant.replace('_', ' ')} "
                                       f"(the faster of the two parallel forms: {variants})", **cpu},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


ADJ_CAMS, ADJ_W, ADJ_H, ADJ_TRACKS = 8, 1280, 720, 4096


def reference_parity(prevs, nexts, counts, host_tracks, frames, run_step):
    """Checker, run after every timed region: the batched step's results against the reference's own
    GPU kernels (oracle/_ref: cuVSLAM's lk_track_kernel and GPUSelection sequence, built from its
    sources) on the same frames and the same input tracks.  LK: status agreement over all tracks,
    and the distance between the positions of the tracks both keep (median, p99, max).  Selection:
    the features selected on the previous frames (the step's input tracks) and the step's new
    features (with the step's own survivors alive) equal the reference's selection as sets."""
    import torch

    from oracle import ref as R
    from cuvslam_b200.frontend import tracks_from_device

    if not R.available():
        return {"unavailable": "oracle/_ref (the reference's kernels built from its sources) is not built here"}
    run_step()
    torch.cuda.synchronize()
    dists, agree, sel_eq, n_all, n_new = [], 0, 0, 0, 0
    for i, f in enumerate(frames):
        got = tracks_from_device(f.tracks)
        want = R.lk(prevs[i], nexts[i], host_tracks[i])
        sg, sw = got["track_status"] != 0, want["track_status"] != 0
        both = sg & sw
        dists.append(np.linalg.norm(got["track"][both].astype(np.float64) - want["track"][both], axis=1))
        agree += int((sg == sw).sum())
        n_all += len(got)
        r0 = R.select(prevs[i], np.zeros((0, 2), np.float32), counts[i])["sel"]
        alive = got["track"][sg].astype(np.float32)
        n = int(f.new_count.item())
        new = f.new_xy[:n].cpu().numpy()
        r1 = R.select(nexts[i], alive, max(0, counts[i] - len(alive)))["sel"]
        n_new += n
        sel_eq += int(R.same_features(host_tracks[i]["track"], r0, 1e-5) and R.same_features(new, r1, 1e-5))
    d = np.concatenate(dists)
    return {"median_px": float(np.median(d)), "p99_px": float(np.percentile(d, 99)), "max_px": float(d.max()),
            "status_agree": agree / max(n_all, 1), "selection_equal": sel_eq == len(frames),
            "cameras_selection_equal": sel_eq, "cameras": len(frames), "tracks": n_all, "tracks_kept_both": len(d),
            "new_features": n_new,
            "against": "the reference's own kernels (lk_track_kernel, GPUSelection) built from its sources, "
                       "same frames and input tracks; checked after the timed regions"}


def adjoint_inputs(ctx, dev):
    """LK adjoint workload: 8 cameras at 1280x720, FP32 frames in [0, 1], 4096 Shi-Tomasi tracks each
    (selected on the previous frame; repeated when a frame has fewer), and the warp's ground truth."""
    import torch

    from cuvslam_b200 import synthetic as S
    from cuvslam_b200.frontend import ImagePyramid, Selection

    sel = Selection(ctx)
    prev, cur, xy, gt = [], [], [], []
    for b in range(ADJ_CAMS):
        p8, c8, warp = S.frame_pair(100 + b, ADJ_W, ADJ_H)
        pp = ImagePyramid(ADJ_W, ADJ_H, device=dev).build(ctx, torch.from_numpy(p8).to(dev))
        f = sel.compute_gftt_and_select_features(pp, 0, 0, 0, 0, None, None, ADJ_TRACKS).reshape(-1, 2).cpu()
        f = torch.cat([f] * (ADJ_TRACKS // max(len(f), 1) + 1))[:ADJ_TRACKS]
        gx, gy = warp.apply(f[:, 0].double().numpy(), f[:, 1].double().numpy())
        prev.append(torch.from_numpy(p8.astype(np.float32) / 255.0))
        cur.append(torch.from_numpy(c8.astype(np.float32) / 255.0))
        xy.append(f)
        gt.append(torch.from_numpy(np.stack([gx, gy], 1).astype(np.float32)))
    return torch.stack(prev).to(dev), torch.stack(cur).to(dev), torch.stack(xy).to(dev), torch.stack(gt).to(dev)


def adjoint_tracker(ctx, mode, inputs, stream):
    """A DiffTracker over the adjoint workload after one forward, with dL/dpos of the mean squared
    distance to ground truth loaded as its backward input."""
    import torch

    from cuvslam_b200.diff import DiffTracker

    prev, cur, xy, gt = inputs
    t = DiffTracker(ctx, ADJ_CAMS, ADJ_H, ADJ_W, ADJ_TRACKS, mode=mode)
    t.set_inputs(prev, cur, xy)
    t.build_pyramids(stream)
    t.forward_step(stream)
    pos, st = t.outputs()
    n = ADJ_CAMS * ADJ_TRACKS
    t.grad_xy.copy_(torch.where(st[..., None], 2.0 * (pos - gt) / n, torch.zeros_like(pos)))
    return t, st


def adjoint_bench(ctx, dev, stream, timed, reps=20):
    """Per mode: forward (both pyramids of every camera + the differentiable tracker) and backward
    (the adjoint) times, their ratio, and the kernel launches of each."""
    inputs = adjoint_inputs(ctx, dev)
    out = {"workload": f"{ADJ_CAMS} cameras {ADJ_W}x{ADJ_H}, {ADJ_TRACKS} tracks each, FP32 frames in [0, 1]"}
    for mode in ("implicit", "unrolled"):
        t, st = adjoint_tracker(ctx, mode, inputs, stream)

        def fwd():
            t.build_pyramids(stream)
            t.forward_step(stream)

        def bwd():
            t.backward_step(stream)

        fwd_ms = timed(fwd, reps, 3) / reps
        bwd_ms = timed(bwd, reps, 3) / reps
        out[mode] = {"fwd_ms": fwd_ms, "bwd_ms": bwd_ms, "bwd_over_fwd": bwd_ms / fwd_ms,
                     "tracks_kept": int(st.sum().item()), "dropped": t.dropped(),
                     "fwd_launches": t.kernel_count(2) + t.kernel_count(0), "bwd_launches": t.kernel_count(1),
                     "iterations": t.iterations}
        t.close()
    return out


# ---------------------------------------------------------------- the other workloads
SEQ_W, SEQ_H, SEQ_FRAMES, SEQ_FEATURES, SEQ_LEVELS = 1241, 376, 100, 1000, 5
SEQ_PARITY_FRAMES = 10  # frame pairs checked against the reference's own kernels


def _seq_frame(f):
    from cuvslam_b200 import synthetic

    img, pose = synthetic.sequence_frame(7, SEQ_W, SEQ_H, f)
    return img, pose


def sequence_frames():
    """The single-camera 100-frame sequence (per-frame translation up to 30 px, rotation up to 3 deg),
    drawn in a spawned pool before the timed work."""
    import multiprocessing as mp

    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        return pool.map(_seq_frame, range(SEQ_FRAMES))


def _gt_between(pose_a, pose_b, xy):
    """Positions in frame b of texture-coordinate points xy of frame a (both views of the base scene)."""
    bx, by = pose_a.inverse_apply(xy[:, 0] - 0.5, xy[:, 1] - 0.5)
    x, y = pose_b.apply(bx, by)
    return np.stack([x + 0.5, y + 0.5], 1)


def _dev_stats(a, b, ok):
    if ok.sum() == 0:
        return {"median_px": None, "p99_px": None, "n": 0}
    d = np.linalg.norm(a[ok] - b[ok], axis=1)
    return {"median_px": float(np.median(d)), "p99_px": float(np.percentile(d, 99)), "n": int(ok.sum())}


def config_sequence(ctx, dev, stream, frames):
    """Single-camera sequence: one camera, 1241x376, 100 frames, 5 levels, 1000 features kept by re-detection.
    The plain GPU path (the drop-in call sequence: build, track, select with its blocking readback)
    against the restated reference CPU tracker (single thread, one camera) in tracks/s; deviation of
    the GPU tracks from the CPU tracker's on the same inputs, and both from the ground truth."""
    import torch

    from oracle import oracle as O
    from cuvslam_b200.frontend import ImagePyramid, LKFeatureTracker, Selection, tracks_from_device, tracks_to_device
    from cuvslam_b200.types import make_tracks

    sel, lk = Selection(ctx), LKFeatureTracker(ctx)
    pyr = [ImagePyramid(SEQ_W, SEQ_H, SEQ_LEVELS, device=dev) for _ in range(2)]
    imgs = [torch.from_numpy(f).to(dev) for f, _ in frames]
    pyr[0].build(ctx, imgs[0], stream=stream)
    xy = sel.compute_gftt_and_select_features(pyr[0], 0, 0, 0, 0, None, None, SEQ_FEATURES, stream).cpu().numpy()
    gpu_s, attempted, dev_gc, gt_g, gt_c = 0.0, 0, [], [], []
    cpu_prev = O.CpuCamera(SEQ_W, SEQ_H).build(frames[0][0])
    cpu_cur = O.CpuCamera(SEQ_W, SEQ_H)
    cpu_s, cpu_xy = 0.0, cpu_prev.select(None, SEQ_FEATURES)
    cpu_attempted = 0
    from oracle import ref as R
    par_frames = SEQ_PARITY_FRAMES if R.available() else 0
    par_d, par_agree, par_n, par_sel = [], 0, 0, 0
    for f in range(1, SEQ_FRAMES):
        prev_p, cur_p = pyr[(f - 1) % 2], pyr[f % 2]
        recs = make_tracks(xy, None, float(SEQ_W), 0.8)
        td = tracks_to_device(recs, dev)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        cur_p.build(ctx, imgs[f], stream=stream)
        lk.track_points(prev_p, cur_p, td, stream=stream)
        out = tracks_from_device(td)
        ok = out["track_status"] == 1
        alive = torch.from_numpy(np.ascontiguousarray(out["track"][ok])).to(dev)
        new = sel.compute_gftt_and_select_features(cur_p, 0, 0, 0, 0, None, alive,
                                                   max(0, SEQ_FEATURES - int(ok.sum())), stream).cpu().numpy()
        gpu_s += time.perf_counter() - t0
        attempted += len(xy)
        if f <= par_frames:  # checker: the reference's own kernels on the same frame pair and tracks
            want = R.lk(frames[f - 1][0], frames[f][0], recs, SEQ_LEVELS)
            sw = want["track_status"] != 0
            par_d.append(np.linalg.norm(out["track"][ok & sw].astype(np.float64) - want["track"][ok & sw], axis=1))
            par_agree += int((ok == sw).sum())
            par_n += len(recs)
            rs = R.select(frames[f][0], out["track"][ok], max(0, SEQ_FEATURES - int(ok.sum())))["sel"]
            par_sel += int(R.same_features(new.reshape(-1, 2), rs, 1e-5))
        # the CPU tracker on the same inputs (deviation), and the ground truth
        cpu_cur.build(frames[f][0])
        cxy, cst = cpu_cur.track_from(cpu_prev, xy)
        both = ok & (cst == 1)
        dev_gc.append(np.linalg.norm(out["track"][both] - cxy[both], axis=1))
        gt = _gt_between(frames[f - 1][1], frames[f][1], xy.astype(np.float64))
        gt_g.append(np.linalg.norm(out["track"][ok] - gt[ok], axis=1))
        gt_c.append(np.linalg.norm(cxy[cst == 1] - gt[cst == 1], axis=1))
        xy = np.concatenate([out["track"][ok], new.reshape(-1, 2)]).astype(np.float32)
        # the CPU tracker's own sequence (timed): track, then re-detect
        t1 = time.perf_counter()
        nxy, nst = cpu_cur.track_from(cpu_prev, cpu_xy)
        keep = nxy[nst == 1]
        add = cpu_cur.select(keep, max(0, SEQ_FEATURES - len(keep)))
        cpu_s += time.perf_counter() - t1
        cpu_attempted += len(cpu_xy)
        cpu_xy = np.concatenate([keep, add.reshape(-1, 2)]).astype(np.float32)
        cpu_prev, cpu_cur = cpu_cur, cpu_prev
    d = np.concatenate(dev_gc)
    g, c = np.concatenate(gt_g), np.concatenate(gt_c)
    return {"workload": f"1 camera {SEQ_W}x{SEQ_H}, {SEQ_FRAMES} frames, {SEQ_LEVELS} levels, {SEQ_FEATURES} features",
            "gpu_plain": {"value": attempted / gpu_s, "unit": UNIT, "ms_per_frame": gpu_s / (SEQ_FRAMES - 1) * 1e3,
                          "timing": "host wall clock per frame (the plain path reads the selection back)"},
            "cpu_reference": {"value": cpu_attempted / cpu_s, "unit": UNIT, "cores": 1, "kind": "port",
                              "ms_per_frame": cpu_s / (SEQ_FRAMES - 1) * 1e3},
            "gpu_over_cpu": (attempted / gpu_s) / (cpu_attempted / cpu_s),
            "deviation_gpu_vs_cpu_px": {"median": float(np.median(d)), "p99": float(np.percentile(d, 99)), "n": len(d)},
            "error_vs_truth_px": {"gpu_median": float(np.median(g)), "cpu_median": float(np.median(c))},
            "parity": _parity_summary(par_d, par_agree, par_n, par_sel, par_frames)}


def _parity_summary(dists, agree, n, sel_equal, frames):
    if not frames:
        return {"unavailable": "oracle/_ref (the reference's kernels built from its sources) is not built here"}
    d = np.concatenate(dists)
    return {"frames": frames, "median_px": float(np.median(d)), "p99_px": float(np.percentile(d, 99)),
            "max_px": float(d.max()), "status_agree": agree / max(n, 1), "selection_equal": sel_equal == frames,
            "against": "the reference's own lk_track_kernel and GPUSelection on the same frame pairs and tracks"}


def config_stereo_plain(ctx, dev, stream):
    """Stereo pair, plain path: one stereo pair plus next frame at 752x480, 4 levels, 512 features: the plain GPU
    path (three pyramids, selection, LK left->next and the horizontal left->right) and the restated
    reference CPU tracker (left->next), per-frame latency."""
    import torch

    from cuvslam_b200 import synthetic
    from oracle import oracle as O
    from cuvslam_b200.frontend import ImagePyramid, LKFeatureTracker, Selection, tracks_from_device, tracks_to_device
    from cuvslam_b200.types import make_tracks

    W, H = 752, 480
    left, nxt, warp = synthetic.frame_pair(0, W, H)
    right = synthetic.stereo_right(0, W, H)
    imgs = [torch.from_numpy(a).to(dev) for a in (left, right, nxt)]
    pyr = [ImagePyramid(W, H, 4, device=dev) for _ in range(3)]
    sel, lk, lkh = Selection(ctx), LKFeatureTracker(ctx), LKFeatureTracker(ctx, horizontal=True)

    def gpu_frame():
        for p, im in zip(pyr, imgs):
            p.build(ctx, im, stream=stream)
        xy = sel.compute_gftt_and_select_features(pyr[0], 0, 0, 0, 0, None, None, 512, stream).cpu().numpy()
        t = make_tracks(xy, None, float(W), 0.8)
        a, b = tracks_to_device(t, dev), tracks_to_device(t, dev)
        lk.track_points(pyr[0], pyr[2], a, stream=stream)
        lkh.track_points(pyr[0], pyr[1], b, stream=stream)
        return xy, tracks_from_device(a)

    for _ in range(3):
        gpu_frame()
    reps = 20
    t0 = time.perf_counter()
    for _ in range(reps):
        xy, out = gpu_frame()
    gpu_ms = (time.perf_counter() - t0) / reps * 1e3
    cl, cn = O.CpuCamera(W, H), O.CpuCamera(W, H)
    t1 = time.perf_counter()
    for _ in range(3):
        cl.build(left)
        cn.build(nxt)
        cxy = cl.select(None, 512)
        cout, cst = cn.track_from(cl, cxy)
    cpu_ms = (time.perf_counter() - t1) / 3 * 1e3
    sxy, sst = cn.track_from(cl, xy)  # the CPU tracker on the GPU's features
    ok = (out["track_status"] == 1) & (sst == 1)
    gt = synthetic.flow_texture(warp, xy.astype(np.float64))
    return {"workload": f"stereo pair + next frame {W}x{H}, 4 levels, 512 features",
            "gpu_plain_ms_per_frame": gpu_ms, "cpu_reference_ms_per_frame": cpu_ms, "cpu_cores": 1,
            "cpu_note": "the CPU arm tracks left->next only (the restated CPU tracker has no horizontal variant)",
            "deviation_gpu_vs_cpu_px": _dev_stats(out["track"], sxy, ok),
            "gpu_error_vs_truth_px": _dev_stats(out["track"], gt.astype(np.float32), out["track_status"] == 1)}


def config_l2r(ctx, dev, stream, npairs=8):
    """Left-to-right stereo matching: npairs rectified 752x480 pairs (seeded scenes, right view at a
    smoothed U(5, 40) px disparity), 4 levels, 512 Shi-Tomasi features per primary, candidates from
    the epipolar table of a pinhole pair (fx 458 px, baseline 0.11 m, auto depth range).  Times the
    folded scan (fe_track_stereo: all pairs, all candidate rounds, one launch) against the reference's
    launch pattern driven with the same horizontal LK kernel (one launch per candidate round, records
    up and down, a stream synchronisation per round, the host loop in Python), and the oracle's CPU
    restatement of the scan on one pair (1 core)."""
    import ctypes

    import torch

    from cuvslam_b200 import _lib, synthetic
    from cuvslam_b200.frontend import ImagePyramid, Selection, _stream_handle
    from cuvslam_b200.stereo import EpipolarCurves, StereoMatcher, StereoPair, cross_cam_search_radius
    from cuvslam_b200.types import TRACK_DTYPE, level_sizes, make_tracks
    from oracle import oracle as O

    W, H, L, NF = 752, 480, 4, 512
    sizes = level_sizes(W, H, L)
    top = len(sizes) - 1
    k = (458.0, 458.0, 367.0, 248.0)
    table = EpipolarCurves.pinhole(k, k, (np.eye(3), (-0.11, 0.0, 0.0)), top, sizes[top][0], sizes[top][1], device=dev)
    lefts = [synthetic.quantise(synthetic.Scene.draw(1000 + c, W, H).render()) for c in range(npairs)]
    rights = [synthetic.stereo_right(c, W, H) for c in range(npairs)]
    pl = [ImagePyramid(W, H, L, device=dev).build(ctx, torch.from_numpy(a).to(dev)) for a in lefts]
    pr = [ImagePyramid(W, H, L, device=dev).build(ctx, torch.from_numpy(a).to(dev)) for a in rights]
    sel = Selection(ctx)
    uvs = [sel.compute_gftt_and_select_features(p, 0, 0, 0, 0, None, None, NF, stream).contiguous() for p in pl]
    pairs = [StereoPair(a, b, uv, curves=table) for a, b, uv in zip(pl, pr, uvs)]
    radius = cross_cam_search_radius(top)
    m = StereoMatcher(ctx)
    outs = m.track_primary_to_secondary(pairs, stream=stream)
    outs1 = m.track_primary_to_secondary(pairs[:1], stream=stream)
    torch.cuda.synchronize()

    def dev_ms(fn, reps=50):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for _ in range(reps):
            fn()
        e.record(stream)
        torch.cuda.synchronize()
        return s.elapsed_time(e) / reps

    folded_ms = dev_ms(lambda: m.track_primary_to_secondary(pairs, outputs=outs, stream=stream))
    folded1_ms = dev_ms(lambda: m.track_primary_to_secondary(pairs[:1], outputs=outs1, stream=stream))
    n_points = sum(int(u.shape[0]) for u in uvs)

    # the reference's launch pattern with the same tracker: candidates on the host, one horizontal LK
    # launch per round over all points, records copied up and down, a synchronisation per round
    cw, ch, inv = table.width, table.height, table.inv_scale
    lib = ctx.lib
    hs = _stream_handle(stream)

    def multi_launch_setup(i):
        uv = uvs[i].cpu().numpy()
        off, cxy = O.epipolar_candidates(cw, ch, inv, table.offsets_host, table.xy_host, uv)
        n = len(uv)
        host = torch.from_numpy(make_tracks(uv, None, radius, 0.8).view(np.uint8).reshape(n, 80).copy()).pin_memory()
        back = torch.empty_like(host).pin_memory()
        d = torch.empty((n, 80), dtype=torch.uint8, device=dev)
        return uv, off, cxy, host, back, d

    setups = [multi_launch_setup(i) for i in range(npairs)]

    def multi_launch(i):
        uv, off, cxy, host, back, d = setups[i]
        n = len(uv)
        lens = np.diff(off)
        rec = host.numpy().view(TRACK_DTYPE).reshape(n)
        out = back.numpy().view(TRACK_DTYPE).reshape(n)
        won = np.zeros(n, bool)
        winner = np.full(n, -1, np.int32)
        tracked = 0
        for kk in range(int(lens.max(initial=0))):
            active = ~won & (kk < lens)
            if not active.any():
                break
            rec["track"] = uv
            rec["track_status"] = 0
            rec["info"] = 0.0
            idx = np.where(active, off[:-1] + kk, 0)
            rec["offset"] = np.where(active[:, None], cxy[np.minimum(idx, max(len(cxy) - 1, 0))] - uv, 0.0)
            d.copy_(host, non_blocking=True)
            _lib.check(lib.fe_track(ctx.handle, ctypes.byref(pl[i].desc), ctypes.byref(pr[i].desc),
                                    ctypes.c_void_p(d.data_ptr()), n, 1, _lib.FE_SAMPLE_TEXTURE, hs), "fe_track")
            back.copy_(d, non_blocking=True)
            stream.synchronize()
            new = active & (out["track_status"] != 0)
            winner[new] = kk
            won |= new
            tracked += int(new.sum())
            if np.float32(tracked) >= np.float32(0.8) * np.float32(n):
                break
        return winner

    wins = [multi_launch(i) for i in range(npairs)]
    same = all(np.array_equal(w, o[1].cpu().numpy()) for w, o in zip(wins, outs))
    reps = 5
    t0 = time.perf_counter()
    for _ in range(reps):
        for i in range(npairs):
            multi_launch(i)
    multi_ms = (time.perf_counter() - t0) / reps * 1e3
    rounds = [int(o[2].cpu().numpy()[1]) for o in outs]
    matched = [int(o[2].cpu().numpy()[0]) for o in outs]
    attempts = [int(o[2].cpu().numpy()[2]) for o in outs]

    # the oracle's CPU restatement of the scan, one pair, 1 core
    opl, opr = O.pyramid(lefts[0], L), O.pyramid(rights[0], L)
    uv0, off0, cxy0 = setups[0][:3]
    t1 = time.perf_counter()
    cpu_reps = 3
    for _ in range(cpu_reps):
        _, cwin, _ = O.stereo_scan(opl, opr, uv0, off0, cxy0, None, radius, 0.8, 0.8)
    cpu_ms = (time.perf_counter() - t1) / cpu_reps * 1e3
    return {"workload": f"{npairs} rectified {W}x{H} stereo pairs, {L} levels, {NF} features per primary, "
                        "epipolar-table candidates (fx 458, baseline 0.11 m)",
            "points": n_points, "matched": matched, "rounds_per_pair": rounds, "attempts_per_pair": attempts,
            "folded_ms_all_pairs": folded_ms, "folded_ms_one_pair": folded1_ms,
            "points_per_s_folded": n_points / (folded_ms / 1e3),
            "multi_launch_ms_all_pairs": multi_ms, "folded_speedup_vs_multi_launch": multi_ms / folded_ms,
            "winners_equal_multi_launch": bool(same),
            "winners_equal_cpu_oracle_pair0": bool(np.array_equal(cwin, outs[0][1].cpu().numpy())),
            "cpu_oracle_ms_one_pair": cpu_ms, "cpu_cores": 1}


def config_affine(ctx, dev, stream, n_tracks=8192):
    """Affine (Shi-Tomasi) tracker: one 1920x1200 frame pair (seeded scene, similarity warp), n_tracks
    Shi-Tomasi features, 0 shift + 20 full-map steps (GPUSTFeatureTracker(0, 20)).  Times fe_track_affine,
    fe_affine_build_cache and fe_track_affine_cached on the device (CUDA events, records reset before
    each call), and the oracle's CPU restatement on a bounded sample (1 core)."""
    import torch

    from cuvslam_b200 import synthetic
    from cuvslam_b200.frontend import (ImagePyramid, Selection, STFeatureTracker, STFeatureTrackerWithCache,
                                       tracks_from_device)
    from cuvslam_b200.types import make_tracks
    from oracle import oracle as O

    W, H = 1920, 1200
    prev, nxt, warp = synthetic.frame_pair(5, W, H)
    pp = ImagePyramid(W, H, 10, device=dev).build(ctx, torch.from_numpy(prev).to(dev))
    cp = ImagePyramid(W, H, 10, device=dev).build(ctx, torch.from_numpy(nxt).to(dev))
    uv = Selection(ctx).compute_gftt_and_select_features(pp, 0, 0, 0, 0, None, None, n_tracks, stream)
    torch.cuda.synchronize()
    pts = uv.cpu().numpy().astype(np.float32)
    gt = synthetic.flow_texture(warp, pts.astype(np.float64)).astype(np.float32)
    rec = make_tracks(pts, (gt - pts) + np.float32(0.5), 64.0, 0.8)
    src = torch.from_numpy(rec.view(np.uint8).reshape(len(rec), 80).copy()).to(dev)
    d = src.clone()
    st = STFeatureTracker(ctx, 0, 20)
    stc = STFeatureTrackerWithCache(ctx, 0, 20)
    cache = stc.build_points_cache(pp, d, stream=stream)
    torch.cuda.synchronize()
    src_cached = d.clone()  # the records with cache_index set by the build

    def dev_ms(fn, reps=20, init=src):
        for _ in range(3):
            d.copy_(init)
            fn()
        torch.cuda.synchronize()
        tot = 0.0
        for _ in range(reps):
            d.copy_(init)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            fn()
            e.record(stream)
            torch.cuda.synchronize()
            tot += s.elapsed_time(e)
        return tot / reps

    with torch.cuda.stream(stream):
        track_ms = dev_ms(lambda: st.track_points(pp, cp, d, stream=stream))
        out = tracks_from_device(d)
        build_ms = dev_ms(lambda: stc.build_points_cache(pp, d, cache, stream=stream))
        cached_ms = dev_ms(lambda: stc.track_points(cp, cache, d, stream=stream), init=src_cached)
        out_cached = tracks_from_device(d)
    ok = out["track_status"] == 1
    err = np.linalg.norm(out["track"][ok] - gt[ok], axis=1)
    opp, ocp = O.pyramid(prev), O.pyramid(nxt)
    ns = min(512, len(rec))
    t0 = time.perf_counter()
    O.st_track(opp, ocp, rec[:ns], 0, 20)
    cpu_s = time.perf_counter() - t0
    n = len(rec)
    return {"workload": f"{W}x{H} frame pair, {n} Shi-Tomasi features, affine tracker 0 shift + 20 full-map steps",
            "tracks": n, "tracked": int(ok.sum()), "tracked_cached": int((out_cached["track_status"] == 1).sum()), "median_err_px_vs_truth": float(np.median(err)) if ok.any() else None,
            "track_ms": track_ms, "build_cache_ms": build_ms, "track_cached_ms": cached_ms,
            "tracks_per_s": n / (track_ms / 1e3), "tracks_per_s_cached": n / (cached_ms / 1e3),
            "cpu_oracle_tracks_per_s": ns / cpu_s, "cpu_sample": f"{ns} tracks, 1 core"}


STREAM_CAMS, STREAM_W, STREAM_H, STREAM_TRACKS, STREAM_FRAMES = 32, 1920, 1200, 8192, 30


def _stream_base(c):
    from cuvslam_b200 import synthetic

    return synthetic.quantise(synthetic.Scene.draw(1000 + c, STREAM_W, STREAM_H).render())


def stream_bases():
    import multiprocessing as mp

    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        return pool.map(_stream_base, range(STREAM_CAMS))


def config_stream(ctx, dev, stream, bases):
    """Forward + backward stream: 16 stereo pairs (32 images) at 1920x1200, 30 consecutive frames, 8192 features
    per image; per frame the forward tracker and the implicit adjoint of the mean squared distance to
    ground truth run in one captured CUDA graph, the pyramids rebuilt for the backward instead of kept.
    Frames: each camera's rendered base frame warped on the GPU by its per-frame similarity (a stand-in
    for 30 rendered frames); features selected on frame 0, tracked from their true positions in frame
    f to frame f + 1."""
    import torch
    import torch.nn.functional as F

    from cuvslam_b200 import synthetic
    from cuvslam_b200.diff import DiffTracker
    from cuvslam_b200.frontend import ImagePyramid, Selection

    B, W, H, N = STREAM_CAMS, STREAM_W, STREAM_H, STREAM_TRACKS
    free0 = torch.cuda.mem_get_info(dev)[0]
    base = torch.from_numpy(np.stack(bases)).to(dev).float()
    poses = [[synthetic.draw_similarity(2000 + f + 7919 * c, W, H) if f else synthetic.Similarity(cx=(W - 1) / 2,
              cy=(H - 1) / 2) for f in range(STREAM_FRAMES + 1)] for c in range(B)]

    def frame(f):
        """(B, H, W) frames in [0, 1]: base sampled at pose_f^-1 (bilinear, border clamp)."""
        ys, xs = torch.meshgrid(torch.arange(H, device=dev, dtype=torch.float64),
                                torch.arange(W, device=dev, dtype=torch.float64), indexing="ij")
        grids = []
        for c in range(B):
            P = poses[c][f]
            m = np.linalg.inv(P._mat())
            xc, yc = xs - P.cx - P.tx, ys - P.cy - P.ty
            bx = m[0, 0] * xc + m[0, 1] * yc + P.cx
            by = m[1, 0] * xc + m[1, 1] * yc + P.cy
            grids.append(torch.stack([bx / (W - 1) * 2 - 1, by / (H - 1) * 2 - 1], -1))
        g = torch.stack(grids).float()
        out = F.grid_sample(base[:, None], g, mode="bilinear", padding_mode="border", align_corners=True)[:, 0]
        return (out.round().clamp(0, 255) / 255.0).contiguous()

    sel = Selection(ctx)
    f0 = frame(0)
    xy0 = []
    for c in range(B):
        pp = ImagePyramid(W, H, device=dev).build(ctx, (f0[c] * 255).round().to(torch.uint8))
        v = sel.compute_gftt_and_select_features(pp, 0, 0, 0, 0, None, None, N).reshape(-1, 2).cpu()
        xy0.append(torch.cat([v] * (N // max(len(v), 1) + 1))[:N].numpy())
    t = DiffTracker(ctx, B, H, W, N, mode="implicit", recompute_pyramids=True)
    xy_buf = torch.zeros((B, N, 2), dtype=torch.float32, device=dev)
    gt_buf = torch.zeros_like(xy_buf)
    n = B * N

    def step():
        t._fields_in[:, :, 0:2].copy_(xy_buf)
        t._fields_in[:, :, 2:4].zero_()
        t.build_pyramids()
        t.forward_step()
        pos, st = t.outputs()
        t.grad_xy.copy_(torch.where(st[..., None], 2.0 * (pos - gt_buf) / n, torch.zeros_like(pos)))
        t.build_pyramids()  # recomputed for the backward
        t.backward_step()

    def load(f):
        t.prev_img.copy_(frame(f))
        t.cur_img.copy_(frame(f + 1))
        a, b = [], []
        for c in range(B):
            pa = synthetic.flow_texture(poses[c][f], xy0[c].astype(np.float64)) if f else xy0[c].astype(np.float64)
            a.append(pa)
            b.append(_gt_between(poses[c][f], poses[c][f + 1], pa))
        xy_buf.copy_(torch.from_numpy(np.stack(a).astype(np.float32)))
        gt_buf.copy_(torch.from_numpy(np.stack(b).astype(np.float32)))

    load(0)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(3):
            step()
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        step()
    used = free0 - torch.cuda.mem_get_info(dev)[0]
    ms, kept = 0.0, 0
    for f in range(STREAM_FRAMES):
        load(f)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g.replay()
        e1.record()
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
        kept += int(t.outputs()[1].sum().item())
    # forward and backward apart (same frame), for their ratio
    fwd_ms = bwd_ms = 0.0
    reps = 5
    for _ in range(reps):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record()
        t.build_pyramids()
        t.forward_step()
        e[1].record()
        t.build_pyramids()
        t.backward_step()
        e[2].record()
        torch.cuda.synchronize()
        fwd_ms += e[0].elapsed_time(e[1]) / reps
        bwd_ms += e[1].elapsed_time(e[2]) / reps
    del g
    deviation = stream_reference_deviation(t, frame, load, xy_buf)
    t.close()
    return {"workload": f"{B} images {W}x{H} (16 stereo pairs), {STREAM_FRAMES} frames, {N} tracks per image, "
                        "forward + implicit adjoint per frame in one CUDA graph, pyramids rebuilt for the backward",
            "value": n * STREAM_FRAMES / (ms / 1e3), "unit": "tracks/s (forward + backward)",
            "ms_per_frame": ms / STREAM_FRAMES, "tracks_kept_per_frame": kept / STREAM_FRAMES,
            "fwd_ms": fwd_ms, "bwd_ms_with_pyramid_rebuild": bwd_ms, "bwd_over_fwd": bwd_ms / fwd_ms,
            "device_memory_bytes": int(used), "deviation_from_reference": deviation}


STREAM_PARITY_CAMS = 4  # cameras of the stream's frame 0 -> 1 compared with the reference's kernel


def stream_reference_deviation(t, frame, load, xy_buf):
    """The differentiable forward (exact bilinear sampling, the reference rule per level, then Newton
    steps to the fixed point at level 0) against the reference's own lk_track_kernel on the same
    uint8 frames and input tracks: frame 0 -> 1 of the first STREAM_PARITY_CAMS cameras, after the
    timed regions.  A deviation, not a parity bar: the two iteration rules stop at different points
    (the reference once its Gauss-Newton update is below 0.12 px, this forward at the fixed point)
    and the forward keeps only tracks whose refinement settles."""
    import torch

    from oracle import ref as R
    from cuvslam_b200.types import TRACK_DTYPE, make_tracks

    if not R.available():
        return {"unavailable": "the reference's kernels (oracle/_ref) were not built"}
    load(0)
    t._fields_in[:, :, 0:2].copy_(xy_buf)
    t._fields_in[:, :, 2:4].zero_()
    t.build_pyramids()
    t.forward_step()
    pos, st = t.outputs()
    pos, st = pos.cpu().numpy(), st.cpu().numpy()
    f0, f1 = frame(0), frame(1)
    d_all, agree, both, n = [], 0, 0, 0
    cams = min(STREAM_PARITY_CAMS, pos.shape[0])
    for c in range(cams):
        prev_u8 = (f0[c] * 255).round().to(torch.uint8).cpu().numpy()
        next_u8 = (f1[c] * 255).round().to(torch.uint8).cpu().numpy()
        xy = xy_buf[c].cpu().numpy()
        want = R.lk(prev_u8, next_u8, make_tracks(xy, None, 2048.0, 0.8))
        got = np.zeros(len(xy), TRACK_DTYPE)
        got["track"] = pos[c]
        got["track_status"] = st[c].astype(np.uint8)
        sg, sw = got["track_status"] != 0, want["track_status"] != 0
        k = sg & sw
        d_all.append(np.linalg.norm(got["track"][k].astype(np.float64) - want["track"][k].astype(np.float64), axis=1))
        agree += int((sg == sw).sum())
        both += int(k.sum())
        n += len(xy)
    d = np.concatenate(d_all) if d_all else np.zeros(0)
    return {"cameras": cams, "tracks": n, "kept_both": both,
            "median_px": float(np.median(d)) if len(d) else 0.0,
            "p99_px": float(np.percentile(d, 99)) if len(d) else 0.0,
            "status_agree": agree / max(n, 1),
            "against": "the reference's own lk_track_kernel (texture sampling) on the same uint8 frames and tracks",
            "note": "different iteration rule by design (fixed point vs converged Gauss-Newton steps)"}


def profile_adjoint(args, local):
    import torch

    from cuvslam_b200.frontend import Context

    global ADJ_CAMS
    if args.adj_cams:
        ADJ_CAMS = int(args.adj_cams)

    torch.cuda.set_device(local)
    ctx = Context(local)
    stream = torch.cuda.current_stream()
    t, _ = adjoint_tracker(ctx, args.profile, adjoint_inputs(ctx, torch.device("cuda", local)), stream)
    for _ in range(args.warmup + args.steps):
        torch.cuda.nvtx.range_push("fwd")
        t.build_pyramids(stream)
        t.forward_step(stream)
        torch.cuda.nvtx.range_pop()
        torch.cuda.nvtx.range_push("bwd")
        t.backward_step(stream)
        torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    print(json.dumps({"profile": args.profile, "fwd_launches": t.kernel_count(2) + t.kernel_count(0),
                      "bwd_launches": t.kernel_count(1)}))
    t.close()
    ctx.close()


def profile_affine(args, local):
    """The affine-tracker workload alone (2048 Shi-Tomasi features of one 1920x1200 pair), for an ncu
    capture of st_track_kernel; prints the config's JSON."""
    import torch

    from cuvslam_b200.frontend import Context

    torch.cuda.set_device(local)
    ctx = Context(local)
    r = config_affine(ctx, torch.device("cuda", local), torch.cuda.Stream(), n_tracks=2048)
    print(json.dumps({"profile": "affine", **r}))
    ctx.close()


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)

    if args.profile in ("implicit", "unrolled"):
        return profile_adjoint(args, local)
    if args.profile == "affine":
        return profile_affine(args, local)
    shapes, counts, prevs, nexts = workload(seed_offset=rank)
    want_configs = rank == 0 and world == 1 and not args.no_configs
    seq_frames = sequence_frames() if want_configs else None
    bases = stream_bases() if want_configs else None
    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from cuvslam_b200 import _lib
    from cuvslam_b200.frontend import Batch, CameraFrame, Context, ImagePyramid, Selection, tracks_to_device
    from cuvslam_b200.types import make_tracks, level_sizes

    # LK samples through the texture unit, as lk_track_kernel does (the emulations of its filtering,
    # bit-identical to the oracle, stay available as FE_SAMPLE_TEXTURE / _WIDE)
    STEP_SAMPLING = _lib.FE_SAMPLE_HARDWARE

    ctx = Context(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()

    # setup (untimed): previous pyramids, the features to track (selected on the previous frames)
    prev_pyr, cur_pyr, frames, pristine, host_tracks = [], [], [], [], []
    img_dev = [torch.from_numpy(n).to(dev) for n in nexts]
    sel = Selection(ctx)
    for (w, h), p, n in zip(shapes, prevs, counts):
        pp = ImagePyramid(w, h, device=dev).build(ctx, torch.from_numpy(p).to(dev))
        xy = sel.compute_gftt_and_select_features(pp, 0, 0, 0, 0, None, None, n).cpu().numpy()
        t = make_tracks(xy, None, float(w), 0.8)
        host_tracks.append(t)
        prev_pyr.append(pp)
        cur_pyr.append(ImagePyramid(w, h, device=dev))
    # every camera's tracks in one device buffer (a view per camera), so that a step's inputs are
    # restored with one copy
    trk_offs = np.concatenate([[0], np.cumsum([len(t) for t in host_tracks])]).astype(np.int64)
    trk_all = torch.empty((int(trk_offs[-1]), 80), dtype=torch.uint8, device=dev)
    for i in range(len(shapes)):
        td = trk_all[trk_offs[i]:trk_offs[i + 1]]
        td.copy_(tracks_to_device(host_tracks[i], dev))
        frames.append(CameraFrame(img_dev[i], cur_pyr[i], prev_pyr[i], td, counts[i], (0, 0, 0, 0)))
    pristine_all = trk_all.clone()
    pristine = [pristine_all[trk_offs[i]:trk_offs[i + 1]] for i in range(len(shapes))]
    batch = Batch(ctx, frames, STEP_SAMPLING)
    tuning = batch.autotune(reps=10, stream=stream)  # restores the tracks it moved
    attempted = sum(len(t) for t in host_tracks)
    if args.profile == "step":
        for _ in range(args.warmup + args.steps):
            torch.cuda.nvtx.range_push("step")
            batch.run(stream)
            torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        print(json.dumps({"profile": "step", "steps": args.warmup + args.steps, "kernels_per_step": batch.kernel_count()}))
        batch.close()
        ctx.close()
        return
    if args.profile:
        part_id = {"pyramid": 0, "lk": 1, "select": 2}[args.profile]
        batch.run_part(0, stream)
        batch.run_part(1, stream)
        for _ in range(args.warmup + args.steps):
            trk_all.copy_(pristine_all)  # every launch of the part on the step's input tracks
            torch.cuda.nvtx.range_push("part")
            batch.run_part(part_id, stream)
            torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        print(json.dumps({"profile": args.profile, "launches": args.warmup + args.steps}))
        batch.close()
        ctx.close()
        return
    kernels_per_step = batch.kernel_count()

    def restore():
        trk_all.copy_(pristine_all, non_blocking=True)

    def step_batched():
        restore()
        batch.run(stream)

    def step_plain():
        restore()
        batch.run_plain(stream)

    def timed(fn, k, w):
        for _ in range(w):
            fn()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for _ in range(k):
            fn()
        e.record(stream)
        torch.cuda.synchronize()
        return reduce_max(s.elapsed_time(e), dist, dev)

    # ---- headline: batched, device-resident inputs.  Clocks are sampled from just before this
    #      timed region through the last GPU measurement below (the window the samples cover).
    clk = ClockSampler(local).__enter__()
    ms = timed(step_batched, args.steps, args.warmup)
    total_units = reduce_sum(attempted, dist, dev)
    value = throughput(total_units, args.steps, ms)

    # ---- the whole MonoSOFGPU frame: the same step plus the retrack pass and the finish filters
    #      (collect, ages, border kill, collapse) between LK and selection
    from cuvslam_b200.frontend import TrackFinish
    fin_frames = []
    fin_trk = pristine_all.clone()
    fin_age0 = torch.ones(int(trk_offs[-1]), dtype=torch.int32, device=dev)
    fin_age = fin_age0.clone()
    for i, f in enumerate(frames):
        fin_frames.append(CameraFrame(f.image, ImagePyramid(f.image.shape[1], f.image.shape[0], device=dev), f.prev,
                                      fin_trk[trk_offs[i]:trk_offs[i + 1]], f.num_desired, f.border,
                                      finish=TrackFinish(fin_age[trk_offs[i]:trk_offs[i + 1]], 0.85)))
    batch_f = Batch(ctx, fin_frames, STEP_SAMPLING)
    batch_f.set_tuning(**tuning)

    def step_finish():
        fin_trk.copy_(pristine_all, non_blocking=True)
        fin_age.copy_(fin_age0, non_blocking=True)
        batch_f.run(stream)

    ms_fin = timed(step_finish, max(3, args.steps // 2), 2)
    fin_value = throughput(total_units, max(3, args.steps // 2), ms_fin)
    fin_alive = sum(int(f.finish.alive_count.item()) for f in fin_frames)

    # ---- plain per-camera launch sequence (same work)
    ms_plain = timed(step_plain, max(3, args.steps // 2), 2)
    plain_value = throughput(total_units, max(3, args.steps // 2), ms_plain)

    # ---- end to end through the public API with host buffers: every camera's frame and tracks in
    #      one pinned host buffer each (as a capture ring would hold them), so that a step's inputs go
    #      up in two copies and its results come back in three
    img_sizes = [n.size for n in nexts]
    img_offs = np.concatenate([[0], np.cumsum(img_sizes)]).astype(np.int64)
    trk_counts = [len(t) for t in host_tracks]
    trk_offs = np.concatenate([[0], np.cumsum(trk_counts)]).astype(np.int64)
    nd_counts = [max(f.num_desired, 1) for f in frames]
    nd_offs = np.concatenate([[0], np.cumsum(nd_counts)]).astype(np.int64)
    pin_img = torch.empty(int(img_offs[-1]), dtype=torch.uint8).pin_memory()
    pin_trk = torch.empty((int(trk_offs[-1]), 80), dtype=torch.uint8).pin_memory()
    for i, n in enumerate(nexts):
        pin_img[img_offs[i]:img_offs[i + 1]].copy_(torch.from_numpy(n.reshape(-1)))
        pin_trk[trk_offs[i]:trk_offs[i + 1]].copy_(
            torch.from_numpy(np.ascontiguousarray(host_tracks[i]).view(np.uint8).reshape(-1, 80)))
    out_trk = torch.empty_like(pin_trk).pin_memory()
    out_new = torch.empty((int(nd_offs[-1]), 2), dtype=torch.float32).pin_memory()
    out_cnt = torch.empty(len(frames), dtype=torch.int32).pin_memory()
    h2d = pin_img.numel() + pin_trk.numel()
    d2h = out_trk.numel() + out_new.numel() * 4 + out_cnt.numel() * 4

    # Two batches over the same cameras (own packed frame, track and output buffers and current
    # pyramids; the previous pyramids shared read-only) in ping-pong: while one computes its step, the
    # other's frames and tracks come in on an upload stream and its results go out on a download stream.
    def packed_set():
        d_img = torch.empty_like(pin_img, device=dev)
        d_trk = torch.empty_like(pin_trk, device=dev)
        d_new = torch.zeros((int(nd_offs[-1]), 2), dtype=torch.float32, device=dev)
        d_cnt = torch.zeros(len(frames), dtype=torch.int32, device=dev)
        fr = []
        for i, f in enumerate(frames):
            h, w = f.image.shape
            cf = CameraFrame(d_img[img_offs[i]:img_offs[i + 1]].view(h, w), ImagePyramid(w, h, device=dev), f.prev,
                             d_trk[trk_offs[i]:trk_offs[i + 1]], f.num_desired, f.border)
            cf.new_xy = d_new[nd_offs[i]:nd_offs[i + 1]]
            cf.new_count = d_cnt[i:i + 1]
            fr.append(cf)
        bt = Batch(ctx, fr, STEP_SAMPLING)
        bt.set_tuning(**tuning)
        return bt, (d_img, d_trk, d_new, d_cnt)

    sets = [packed_set(), packed_set()]
    up, down = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_done = [torch.cuda.Event() for _ in range(2)]
    ev_free = [torch.cuda.Event() for _ in range(2)]
    for e in ev_free:
        e.record(stream)

    def step_e2e(k):
        b, (d_img, d_trk, d_new, d_cnt) = sets[k % 2]
        with torch.cuda.stream(up):
            up.wait_event(ev_free[k % 2])  # this set's previous results are out
            d_img.copy_(pin_img, non_blocking=True)
            d_trk.copy_(pin_trk, non_blocking=True)
            ev_in[k % 2].record(up)
        stream.wait_event(ev_in[k % 2])
        b.run(stream)
        ev_done[k % 2].record(stream)
        with torch.cuda.stream(down):
            down.wait_event(ev_done[k % 2])
            out_trk.copy_(d_trk, non_blocking=True)
            out_new.copy_(d_new, non_blocking=True)
            out_cnt.copy_(d_cnt, non_blocking=True)
            ev_free[k % 2].record(down)

    for k in range(max(args.warmup, 3)):
        step_e2e(k)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for k in range(args.steps):
        step_e2e(k)
    stream.wait_event(ev_free[(args.steps - 1) % 2])  # the last results are on the host
    s1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = reduce_max(s0.elapsed_time(s1), dist, dev)
    e2e_value = throughput(total_units, args.steps, ms_e2e)

    # ---- the parts of the step, each launch timed alone with CUDA events on its stream (the tracks
    #      restored, and for the selection LK run, outside the event pair), and their rooflines
    def part_launch_ms(p, reps, warm=2):
        pairs = []
        for r in range(warm + reps):
            restore()
            if p == 2:
                batch.run_part(1, stream)  # the selection reads LK's survivors
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            batch.run_part(p, stream)
            s1.record(stream)
            if r >= warm:
                pairs.append((s0, s1))
        torch.cuda.synchronize()
        return reduce_max(sum(a.elapsed_time(b) for a, b in pairs) / reps, dist, dev)

    reps = 10
    part_ms = {name: part_launch_ms(p, reps) for name, p in (("pyramid", 0), ("lk", 1), ("select", 2))}
    clk.__exit__()
    clocks = clk.summary()
    if clocks is not None:
        clocks["window"] = ("50 ms samples from just before the headline timed region through the per-part "
                            "timings (all GPU measurements of the step)")
    alg_bytes = 0
    for (w, h) in shapes:
        alg_bytes += w * h + 12 * sum(a * b for a, b in level_sizes(w, h))
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak, peak_src = json.load(open(peaks_path))["hbm_gbs"], "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    achieved = alg_bytes / (part_ms["pyramid"] / 1e3) / 1e9
    traffic, traffic_src = None, None
    prof = os.path.join(ROOT, "profiles", "pyramid_multicam32_traffic.txt")
    if os.path.exists(prof):
        captured_on = None
        for line in open(prof):
            if line.startswith("dram_bytes_per_step:"):
                traffic = int(line.split(":")[1])
            if line.startswith("kernel_source_sha256:"):
                captured_on = line.split(":")[1].strip()
        import hashlib
        current = hashlib.sha256(open(os.path.join(ROOT, "cuvslam_b200", "csrc", "pyramid.cu"), "rb").read()).hexdigest()[:16]
        traffic_src = {"from": "ncu capture of this workload's pyramid launch (profiles/pyramid_multicam32_traffic.txt), "
                               "not measured in this run",
                       "captured_on_pyramid_cu": captured_on, "current_pyramid_cu": current,
                       "current": captured_on == current}
    # LK: algorithmic FLOPs by the convention of the work counters (per level set up 2592, per
    # Gauss-Newton step 1134, per NCC evaluation 200), counted by the kernel itself in one extra run
    restore()
    lk_levels, lk_steps, lk_ncc = batch.lk_work(stream)
    lk_flops = 2592 * lk_levels + 1134 * lk_steps + 200 * lk_ncc
    props = torch.cuda.get_device_properties(dev)
    sm_max = (clocks or {}).get("sm_max_mhz") or 1965.0
    fp32_peak = props.multi_processor_count * 128 * 2 * sm_max * 1e6 / 1e12
    lk_achieved = lk_flops / (part_ms["lk"] / 1e3) / 1e12

    # ---- parity against the reference's own kernels (checker; after every timed region), rank 0
    parity = None
    if rank == 0 and not args.no_parity:
        try:
            parity = reference_parity(prevs, nexts, counts, host_tracks, frames, step_batched)
        except Exception as ex:  # reported, not fatal: the headline line must still print
            parity = {"error": f"{type(ex).__name__}: {ex}"}

    # ---- CPU baseline (restated reference CPU tracker), rank 0 at N=1 only
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        host = host_cpu()
        nrep = 3
        variants, (variant, _, _) = cpu_baseline_variants(shapes, counts, prevs, nexts, host["usable_cores"], nrep)
        cpu = {"value": variants[variant], "unit": UNIT, "cores": host["usable_cores"], "kind": "port",
               "sample": f"full 32-camera frame step x {nrep} per variant, restated reference CPU tracker; "
                         f"value = the faster variant ({variant.replace('_', ' ')})",
               "variants": variants, **host}

    adjoint = None
    if rank == 0 and not args.no_adjoint:
        adjoint = adjoint_bench(ctx, dev, stream, timed)
    workloads = None
    if want_configs:
        workloads = {}
        for name, fn in (("stereo_plain", lambda: config_stereo_plain(ctx, dev, stream)),
                         ("sequence", lambda: config_sequence(ctx, dev, stream, seq_frames)),
                         ("l2r_stereo", lambda: config_l2r(ctx, dev, stream)),
                         ("affine_st", lambda: config_affine(ctx, dev, stream)),
                         ("stream_fwd_bwd", lambda: config_stream(ctx, dev, stream, bases))):
            try:
                workloads[name] = fn()
            except Exception as ex:  # reported, not fatal: the headline line must still print
                workloads[name] = {"error": f"{type(ex).__name__}: {ex}"}
            torch.cuda.synchronize()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "tracks_per_step": total_units, "cameras": len(shapes) * world,
                       "l2": "working set > L2 (~600 MB of pyramids written per step)", "sampling": "texture unit (FE_SAMPLE_HARDWARE)",
                       "tuning": tuning},
            "plain": {"value": plain_value, "unit": UNIT, "ms_per_step": ms_plain / max(3, args.steps // 2)},
            "batched_over_plain": value / plain_value,
            "frame_with_finish": {"value": fin_value, "unit": UNIT, "ms_per_step": ms_fin / max(3, args.steps // 2),
                                  "kernels_per_step": batch_f.kernel_count(), "tracks_alive": fin_alive,
                                  "what": "the step plus the retrack pass (NCC 0.85) and the finish filters"},
            "parts_ms": part_ms,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "pipeline": "two batches in ping-pong, uploads and downloads on their own streams; each step's "
                                "inputs and results in packed pinned buffers (2 copies up, 3 down)"},
            "roofline": {"bound": "hbm", "kernel": "pyramid stages (all cameras)", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "traffic_source": traffic_src, "algorithmic_bytes": alg_bytes, "peak_source": peak_src},
            "roofline_lk": {"bound": "latency of the texture fetches (the texture unit filters; FP32 issue "
                                     "bounds the emulated modes)",
                            "kernel": "LK (all tracks), texture-unit sampling", "achieved": lk_achieved,
                            "peak": fp32_peak, "unit": "TFLOP/s", "frac": lk_achieved / fp32_peak,
                            "flops_per_launch": lk_flops, "ms_per_launch": part_ms["lk"],
                            "work": {"levels_set_up": lk_levels, "gauss_newton_steps": lk_steps, "ncc": lk_ncc},
                            "convention": "2592 per level set up + 1134 per Gauss-Newton step + 200 per NCC "
                                          "evaluation, counted by the kernel",
                            "peak_source": f"nominal: {props.multi_processor_count} SMs x 128 FP32 lanes x 2 x "
                                           f"{sm_max:.0f} MHz (no measured FP32 peak)"},
            "cpu_baseline": cpu,
            "parity": parity,
            "clocks": clocks,
            "gpu_launches": kernels_per_step * args.steps,
            "adjoint": adjoint,
            "other_configs": workloads,
        }
        print(json.dumps(line), flush=True)
    batch.close()
    for bt, _ in sets:
        bt.close()
    batch_f.close()
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
