"""Benchmark: batched multi-camera tracking front-end on B200.

Workload (BASELINE config "batched multicamera"): 32 cameras of uneven resolution (12 x 640x480,
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
    ap.add_argument("--profile", choices=["pyramid", "lk", "select", "step", "implicit", "unrolled"], default=None,
                    help="for an ncu capture: run only this part of the step (inside NVTX ranges named "
                         "'part'), whole batched steps (ranges named 'step'), or the LK adjoint workload's "
                         "forward and backward in one mode (ranges 'fwd', 'bwd'), warmup + steps times")
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
        self.path = os.path.join(ROOT, "gpurun_out" if os.path.isdir(os.path.join(ROOT, "gpurun_out")) else "/tmp",
                                 f"clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
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


def cpu_reference_step_fn(shapes, counts, prevs, nexts, nthreads):
    """A callable running one frame step of the restated reference CPU tracker over all cameras."""
    from oracle import oracle as O

    prev_cams = [O.CpuCamera(w, h).build(p) for (w, h), p in zip(shapes, prevs)]
    cur_cams = [O.CpuCamera(w, h) for (w, h) in shapes]
    feats = [c.select(None, n) for c, n in zip(prev_cams, counts)]
    attempted = sum(len(f) for f in feats)

    def step():
        return O.cpu_frame_step(prev_cams, cur_cams, nexts, feats, None, counts, nthreads)

    return step, attempted


def run_reference(args, rank):
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    shapes, counts, prevs, nexts = workload()
    step, attempted = cpu_reference_step_fn(shapes, counts, prevs, nexts, nthreads)
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
                             "sample": f"full 32-camera frame step x {args.steps} steps, one camera per thread"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


ADJ_CAMS, ADJ_W, ADJ_H, ADJ_TRACKS = 8, 1280, 720, 4096


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


def profile_adjoint(args, local):
    import torch

    from cuvslam_b200.frontend import Context

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


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)

    if args.profile in ("implicit", "unrolled"):
        return profile_adjoint(args, local)
    shapes, counts, prevs, nexts = workload(seed_offset=rank)
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
    for i in range(len(shapes)):
        td = tracks_to_device(host_tracks[i], dev)
        pristine.append(td.clone())
        frames.append(CameraFrame(img_dev[i], cur_pyr[i], prev_pyr[i], td, counts[i], (0, 0, 0, 0)))
    batch = Batch(ctx, frames, _lib.FE_SAMPLE_TEXTURE)
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
        for f, p in zip(frames, pristine):
            f.tracks.copy_(p, non_blocking=True)

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

    # ---- headline: batched, device-resident inputs
    with ClockSampler(local) as clk:
        ms = timed(step_batched, args.steps, args.warmup)
    clocks = clk.summary()
    total_units = reduce_sum(attempted, dist, dev)
    value = throughput(total_units, args.steps, ms)

    # ---- plain per-camera launch sequence (same work)
    ms_plain = timed(step_plain, max(3, args.steps // 2), 2)
    plain_value = throughput(total_units, max(3, args.steps // 2), ms_plain)

    # ---- end to end through the public API with host buffers
    pin_imgs = [torch.from_numpy(n).pin_memory() for n in nexts]
    pin_tracks = [torch.from_numpy(np.ascontiguousarray(t).view(np.uint8).reshape(len(t), 80).copy()).pin_memory()
                  for t in host_tracks]
    out_tracks = [torch.empty_like(t).pin_memory() for t in pin_tracks]
    out_new = [torch.empty((f.new_xy.shape[0], 2), dtype=torch.float32).pin_memory() for f in frames]
    out_cnt = [torch.empty(1, dtype=torch.int32).pin_memory() for _ in frames]
    h2d = sum(i.numel() for i in pin_imgs) + sum(t.numel() for t in pin_tracks)
    d2h = sum(t.numel() for t in out_tracks) + sum(o.numel() * 4 for o in out_new) + 4 * len(out_cnt)

    def step_e2e():
        for f, pi, pt in zip(frames, pin_imgs, pin_tracks):
            f.image.copy_(pi, non_blocking=True)
            f.tracks.copy_(pt, non_blocking=True)
        batch.run(stream)
        for f, ot, on, oc in zip(frames, out_tracks, out_new, out_cnt):
            ot.copy_(f.tracks, non_blocking=True)
            on.copy_(f.new_xy, non_blocking=True)
            oc.copy_(f.new_count, non_blocking=True)

    ms_e2e = timed(step_e2e, args.steps, max(args.warmup, 3))
    e2e_value = throughput(total_units, args.steps, ms_e2e)

    # ---- dominant part and its roofline (pyramid stages: HBM-bound)
    def part(p):
        return lambda: batch.run_part(p, stream)

    reps = 10
    part_ms = {name: timed(part(p), reps, 2) / reps for name, p in (("pyramid", 0), ("lk", 1), ("select", 2))}
    alg_bytes = 0
    for (w, h) in shapes:
        alg_bytes += w * h + 12 * sum(a * b for a, b in level_sizes(w, h))
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak, peak_src = json.load(open(peaks_path))["hbm_gbs"], "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    achieved = alg_bytes / (part_ms["pyramid"] / 1e3) / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "pyramid_multicam32_traffic.txt")
    if os.path.exists(prof):
        for line in open(prof):
            if line.startswith("dram_bytes_per_step:"):
                traffic = int(line.split(":")[1])

    # ---- CPU baseline (restated reference CPU tracker), rank 0 at N=1 only
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        nthreads = os.cpu_count() or 1
        stepc, att = cpu_reference_step_fn(shapes, counts, prevs, nexts, nthreads)
        stepc()
        t0 = time.perf_counter()
        nrep = 3
        for _ in range(nrep):
            stepc()
        dt = time.perf_counter() - t0
        cpu = {"value": att * nrep / dt, "unit": UNIT, "cores": nthreads, "kind": "port",
               "sample": f"full 32-camera frame step x {nrep}, restated reference CPU tracker, one camera per thread"}

    adjoint = None
    if rank == 0 and not args.no_adjoint:
        adjoint = adjoint_bench(ctx, dev, stream, timed)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "tracks_per_step": total_units, "cameras": len(shapes) * world,
                       "l2": "working set > L2 (~600 MB of pyramids written per step)", "sampling": "texture",
                       "tuning": tuning},
            "plain": {"value": plain_value, "unit": UNIT, "ms_per_step": ms_plain / max(3, args.steps // 2)},
            "batched_over_plain": value / plain_value,
            "parts_ms": part_ms,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm", "kernel": "pyramid stages (all cameras)", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "algorithmic_bytes": alg_bytes, "peak_source": peak_src},
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": kernels_per_step * args.steps,
            "adjoint": adjoint,
        }
        print(json.dumps(line), flush=True)
    batch.close()
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
