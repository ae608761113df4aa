#!/usr/bin/env python
"""Benchmark of the B200 cull + meshlet-DAG LOD cut: views/s of the batched launch on the ruins-like scene.

One step = one pass of the hot path over one batch of synthetic input: the 32 poses of the ruins-like scene's
camera spline (113,106 instances of 40 meshes, 1920 x 1080, errorThreshold 1 px, HZB occlusion from each pose's
1920 x 1080 occluder depth image): 32 HZB builds plus one batched cut (CUDA graph) of the 32 views.

Printed (one JSON line on rank 0): views/s with inputs resident in HBM (`value`), the same metric end to end
through the public C ABI with host buffers (`e2e`: depth images + views in, draw lists + counters out), the plain
per-view launch beside it, per-view latency percentiles, the roofline of the dominant kernel, the CPU baseline
(the oracle's double restatement of the reference path on the host cores) and sampled SM clocks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config ruins|plain_small]
"""
from __future__ import annotations

import argparse
import contextlib
import copy
import ctypes
import gc
import json
import math
import os
import re
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "three-virtual-geometry_b200"))

METRIC = "views/sec & p99 ms: served batched cull+LOD cut vs plain per-view, same B200"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="ruins", choices=["ruins", "plain_small"])
    ap.add_argument("--poses", type=int, default=32, help="views per step (the spline's pose count)")
    ap.add_argument("--profile-case", nargs="?", const="cut", default=None,
                    choices=["cut", "occluders", "visibility"],
                    help="small case for an ncu capture (not a bench line): the batched and plain cuts, the "
                         "occluder depth pass over 4 poses, or the closed loop (expand + visibility) over 4 poses")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="bound of the CPU-baseline sample")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batching, occluder, large-world and serving sections")
    ap.add_argument("--extras", default="serve_ruins,batching,occluders,visibility,updates,large_world,serve",
                    help="comma-separated sections to run after the headline line's measurement")
    ap.add_argument("--serve-rate", type=float, default=10_000.0, help="Poisson request rate of the serving section")
    ap.add_argument("--serve-max-meshlets", type=int, default=0,
                    help="draw-list capacity (meshlets per cut) of every serving scene's views (0: by scene size)")
    ap.add_argument("--serve-max-triangles", type=int, default=0,
                    help="triangle capacity (camera cut) of every serving scene's views (0: by scene size)")
    ap.add_argument("--serve-requests", type=int, default=20_000)
    return ap.parse_args()


def read_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def read_traffic(kernel: str):
    """dram read+write bytes per launch from the committed ncu summary of `kernel`, scaled to the full launch."""
    path = os.path.join(ROOT, "profiles", f"{kernel}.md")
    try:
        text = open(path).read()
    except OSError:
        return None
    m = re.search(r"dram_bytes_per_full_launch\s*=\s*([0-9.eE+]+)", text)
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 20 ms while the timed region runs. The sampler is live
    (its first row read) before the region starts, so that a short region still gets samples; the summary uses the
    rows read inside the region, else the last row read before it (`samples_in_region` says which)."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device: int):
        self.device = device
        self.rows = []  # (time, fields)
        self.proc = None
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            deadline = time.perf_counter() + 5.0
            while not self.rows and time.perf_counter() < deadline and self.proc.poll() is None:
                time.sleep(0.005)
        except OSError:
            self.proc = None
        self.t0 = time.perf_counter()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append((time.perf_counter(), [x.strip() for x in line.split(",")]))

    def __exit__(self, *exc):
        self.t1 = time.perf_counter()
        if self.proc:
            time.sleep(0.03)  # the row that covers the region's end
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        inside = [r for t, r in self.rows if self.t0 is not None and self.t0 <= t <= self.t1 + 0.03]
        before = [r for t, r in self.rows if self.t0 is not None and t < self.t0]
        rows = inside or before[-1:]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for i, n in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows), "samples_in_region": len(inside)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        # one process per GPU over NCCL; gloo where no GPU is visible (the host-side logic's tests)
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def build_scene(config: str, poses: int):
    from vgcut import scenes
    threads = os.cpu_count() or 8
    if config == "plain_small":
        return scenes.plain_small(threads=threads), dict(workload="plain_small: 1,048,820-triangle icosphere x 64 instances, 1080p, 1 view, t=1px")
    spec = scenes.ruins(poses=poses, threads=threads)
    return spec, dict(workload=f"ruins-like: {spec.instance_count} instances of {len(spec.meshes)} meshes "
                               f"({spec.notes['meshlets']} meshlets, {spec.full_detail_triangles / 1e9:.2f}B full-detail "
                               f"triangles), 1920x1080, {len(spec.cameras)} spline poses per step, t=1px, HZB 1920x1080")


# ------------------------------------------------------------------ CPU baseline (the oracle, double precision)
class OraclePass:
    """The oracle's double restatement of the reference path (cells, instances, meshlets, prefix, HZB build) over the
    bench scene, set up once (cells, Morton order, pool arrays) so that timing covers the per-view pass only."""

    def __init__(self, spec, occlusion: bool):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        from vgcut import engine
        self.O, self.engine, self.spec, self.occlusion = O, engine, spec, occlusion
        flags = [dict(occlusion=occlusion) for _ in spec.meshes]
        self.scene, _, _ = O.scene_from_spec(spec.meshes, spec.instances, flags)
        self.cores = os.cpu_count() or 1

    def view(self, k: int) -> int:
        """Pose k: HZB build from its depth image, then the full pass on all host cores; returns meshlets selected."""
        O, spec = self.O, self.spec
        hzb = O.hzb_build(spec.depth_images[k]) if (self.occlusion and spec.depth_images) else None
        v = O.make_view(spec.cameras[k], self.engine.ViewParams(error_threshold=1.0), 1 << 20, (30_000_000, 12_000_000),
                        hzb=hzb)
        r = O.cull_pass(self.scene, v, "f64", threads=self.cores, capacity=1 << 18)
        return r["counters"][2]


def cpu_baseline(spec, seconds: float, occlusion: bool, runner=None):
    """Times the oracle pass over a bounded sample of the step's views (poses in order, at least one); returns
    (views/s, cores, sample description)."""
    runner = runner or OraclePass(spec, occlusion)
    done, t0 = 0, time.perf_counter()
    while True:
        runner.view(done % len(spec.cameras))
        done += 1
        if time.perf_counter() - t0 >= seconds or done >= 4 * len(spec.cameras):
            break
    dt = time.perf_counter() - t0
    return done / dt, runner.cores, (f"{done} views of the same workload (oracle f64 full pass incl. HZB build, "
                                     f"{runner.cores} threads, {dt:.1f} s; scene set up outside the timing)")


PARITY_STEPS = list(range(0, 255, 15))  # blend steps of the DAG-cut invariant check


def parity_capture(vg, spec, views, occl, device):
    """GPU outputs the parity check compares with the oracle (after the timed steps, outside any timing): every
    fourth headline view cut once more through the plain launch (its HZB built from its depth image on the device)
    with the controller state it starts from, and one culling-off cut of pose 0 at 2 px (blend band open) from a
    context whose draw list holds it whole."""
    from vgcut import engine
    out = dict(views={}, max_meshlets=1 << 18)
    for k in list(range(0, len(views), 4))[:8]:
        state = list(vg.state(views[k].state_slot))
        vg.cut([views[k]], first_slot=k)
        out["views"][k] = dict(lists=[vg.draw_list(k, 0), vg.draw_list(k, 1)], stats=vg.read_stats(k), state=state)
    big = engine.VirtualGeometry(max_triangles=40_000_000, max_shadow_triangles=4_000_000, max_meshlets=1 << 20,
                                 output_slots=1, device=device)
    from vgcut import scenes
    scenes.load_into(big, spec, occlusion_culling=occl)
    p = engine.ViewParams(error_threshold=2.0, frustum_culling=False, min_pixel_radius=0.0)
    big.update(spec.cameras[0], slot=0, **p.__dict__)
    out["culling_off"] = dict(list=big.draw_list(0, 0), stats=big.read_stats(0), threshold=2.0)
    big.dispose()
    return out


def parity_check(runner, captured) -> dict:
    """The parity counters of the headline views: the GPU against the oracle's float mirror (sets, counters), every
    difference from the double restatement classified by its decision's slack (within the 1e-5 relative margin or
    not), and the DAG-cut invariant (verifyCutCoverage / verifyCutOverlap per instance and blend step) of the
    culling-off cut."""
    import numpy as np
    O, engine, spec = runner.O, runner.engine, runner.spec
    keys = lambda e, cols: set(map(tuple, np.asarray(e)[:, list(cols)].tolist())) if len(e) else set()
    mirror_mismatch = margin = outside = entries = 0
    max_slack = 0.0
    for k, g in captured["views"].items():
        hzb = O.hzb_build(spec.depth_images[k]) if (runner.occlusion and spec.depth_images) else None
        p = engine.ViewParams(error_threshold=1.0, hzb=(k if runner.occlusion else -1))
        caps = (30_000_000, 12_000_000)
        v32 = O.make_view(spec.cameras[k], p, captured["max_meshlets"], caps, hzb=hzb, state=g["state"])
        r32 = O.cull_pass(runner.scene, v32, "f32", threads=runner.cores)
        # the double restatement of each cut at the controller scales of its final computation (pinned rounds)
        r64, v64 = O.pinned_reference(
            runner.scene, lambda st: O.make_view(spec.cameras[k], p, captured["max_meshlets"], caps, hzb=hzb, state=st),
            v32, g["state"], threads=runner.cores)
        s = g["stats"]
        if [s["selected"][0], s["selected"][1], s["visible_cells"]] != [r32["counters"][2], r32["counters"][7],
                                                                          r32["counters"][0]]:
            mirror_mismatch += 1
        seen = set()
        for cut in (0, 1):
            gk = keys(g["lists"][cut], (0, 1, 3))
            if gk != keys(r32["entries"][cut], (0, 1, 2)):
                mirror_mismatch += 1
            entries += len(gk)
            for inst, m, _ in gk ^ keys(r64[cut], (0, 1, 2)):
                if (cut, inst, m) in seen:
                    continue
                seen.add((cut, inst, m))
                slack = O.explain(runner.scene, v64[cut], cut, inst, m)
                if slack <= 1e-5:
                    margin += 1
                else:
                    outside += 1
                    max_slack = max(max_slack, slack)
    off = captured["culling_off"]
    inst_slot = np.concatenate([np.full(len(m), i, np.uint32) for i, m in enumerate(spec.instances)])
    bad, checked = O.cut_invariant(spec.meshes, inst_slot, off["list"][:, [0, 1, 3]], PARITY_STEPS,
                                   threads=runner.cores)
    return dict(views_checked=len(captured["views"]), entries_compared=entries, mirror_mismatches=mirror_mismatch,
                margin_decisions=margin, outside_margin=outside, outside_margin_max_slack=max_slack,
                invariant_instances=checked, invariant_of=spec.instance_count, invariant_violations=bad,
                invariant_steps=len(PARITY_STEPS),
                note="every 4th headline view (HZB on) vs the oracle's float mirror (bit-exact sets and counters) and "
                     "its double restatement at the controller state of the cut's final round (differences classified "
                     "by decision slack, margin 1e-5 relative; a decision just past it comes from float32 positions "
                     "at kilometre world coordinates, ~3e-5 m, near the camera); "
                     "invariant: pose 0 at 2 px with culling off, every instance's cut complete and overlap-free at "
                     "each checked blend step")


def run_reference(args, world, rank):
    """The reference arm: one step = the same views the GPU arm cuts per step (every pose of the spline, each with
    its HZB build), through the oracle's double restatement on all host cores. Scene set-up is outside the timing."""
    if rank != 0:
        return
    spec, cfg = build_scene(args.config, args.poses)
    occl = args.config == "ruins"
    runner = OraclePass(spec, occl)
    P = len(spec.cameras)

    def step():
        for k in range(P):
            runner.view(k)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    value = P * args.steps / dt
    cfg.update(bench_config(P, occl))
    line = dict(metric=METRIC, value=value, unit="views/s", n_gpus=args.gpus, steps=args.steps, warmup=args.warmup,
                ms_per_step=dt / args.steps * 1e3, higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f64",
                data="synthetic (seeded ruins-like scene; the reference's WebGPU scenes cannot run here)", config=cfg,
                impl="reference", ms_per_view=dt / (P * args.steps) * 1e3,
                cpu_baseline=dict(value=value, unit="views/s", cores=runner.cores, kind="port",
                                  sample=f"{P} views per step (every pose, HZB build included), {args.steps} steps: the "
                                         f"oracle's f64 restatement of the reference passes on {runner.cores} threads "
                                         f"(the TypeScript reference cannot run here)"),
                e2e=dict(value=value, unit="views/s", h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)


def bench_config(views_per_step: int, occlusion: bool) -> dict:
    """The config keys both arms report (the workload's own key comes from build_scene)."""
    return dict(views_per_step=views_per_step,
                flush="GPU arm: 256 MB L2 flush before every timed step (outside the events); host arm: none",
                max_meshlets_per_cut=1 << 18, threshold_px=1.0, occlusion=occlusion)


# ------------------------------------------------------------------ our arm
def run_ours(args, world, rank, local):
    import numpy as np
    import torch
    from vgcut import engine, scenes

    torch.cuda.set_device(local)
    spec, cfg = build_scene(args.config, args.poses)
    if args.profile_case in ("occluders", "visibility"):
        small = copy.copy(spec)
        small.cameras = spec.cameras[:4]
        run = run_occluders if args.profile_case == "occluders" else run_visibility
        res = run(small, args, torch.empty(256 << 20, dtype=torch.uint8, device="cuda"), torch.cuda.Stream())
        print(json.dumps(dict(profile_case="ok", **{args.profile_case: res})), flush=True)
        return
    P = len(spec.cameras)
    occl = args.config == "ruins" and len(spec.depth_images) > 0
    vg = engine.VirtualGeometry(max_triangles=10_000_000, max_shadow_triangles=4_000_000, max_meshlets=1 << 18,
                                output_slots=P, device=local)
    scenes.load_into(vg, spec, occlusion_culling=occl)
    stream = torch.cuda.Stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    L = engine.lib()
    d_depth = [torch.from_numpy(d).cuda() for d in spec.depth_images] if occl else []
    h_depth = [torch.from_numpy(d).pin_memory() for d in spec.depth_images] if occl else []
    H, W = (spec.depth_images[0].shape if occl else (0, 0))
    # each view carries its occluder depth: the cut builds its HZB in the same launch sequence, reading mip 0 from the
    # depth image (VGC_VIEW_DEPTH_AS_MIP0: the HZB is rebuilt every step, so mip 0 need not be copied into the slot)
    views = [engine.make_view(c, engine.ViewParams(error_threshold=1.0, hzb=(k if occl else -1), state_slot=k,
                                                   depth_as_mip0=occl),
                              depth=((d_depth[k].data_ptr(), W, H) if occl else None))
             for k, c in enumerate(spec.cameras)]
    views_host = [engine.make_view(c, engine.ViewParams(error_threshold=1.0, hzb=(k if occl else -1), state_slot=k))
                  for k, c in enumerate(spec.cameras)]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    def hzb_step(host: bool):
        for k in range(P if occl else 0):
            src = h_depth[k] if host else d_depth[k]
            engine.check(L.vgc_hzb_build(vg.handle, k, src.data_ptr(), W, H, 0 if host else 1, sp))

    def step_resident():
        vg.cut(views, first_slot=0, stream=sp, graph=True)

    host_ms = []  # host time of each timed step's call (view constants, plan, graph launch)

    def timed(fn, steps):
        out = []
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            t0 = time.perf_counter()
            fn()
            host_ms.append((time.perf_counter() - t0) * 1e3)
            b.record(stream)
            b.synchronize()
            out.append(a.elapsed_time(b))
        return out

    # warm-up (graph capture happens in the first step)
    for _ in range(max(3, args.warmup)):
        step_resident()
    torch.cuda.synchronize()
    # The views' capacity controllers start from their initial state; with the poses the same from step to step they
    # settle within a few tens of steps, after which no view redoes its cut. Steps until then run retry rounds (a view
    # near its draw capacity is cut again at a coarser threshold, as the reference does); they are timed here and
    # reported as `controller`, and the timed steps below are the settled frames.
    settle_ms, quiet = [], 0
    while len(settle_ms) < 60 and quiet < 8 and not args.profile_case:
        with torch.cuda.stream(stream):
            flush.fill_(1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        step_resident()
        b.record(stream)
        b.synchronize()
        settle_ms.append(a.elapsed_time(b))
        quiet = quiet + 1 if sum(vg.read_stats(k)["rounds"] for k in range(P)) == P else 0
    if args.profile_case:
        # a small, fixed case for profilers: two more batched steps, then four plain per-view cuts
        for _ in range(2):
            step_resident()
        for k in range(min(4, P)):
            arr = (engine.View * 1)(views[k])
            engine.check(L.vgc_cut(vg.handle, arr, 1, k, sp))
        torch.cuda.synchronize()
        print(json.dumps(dict(profile_case="ok", views=P, work=vg.read_stats(0))), flush=True)
        vg.dispose()
        return
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        t_wall = time.perf_counter()
        step_ms = timed(step_resident, args.steps)
        t_wall = time.perf_counter() - t_wall
    torch.cuda.synchronize()
    barrier(world)
    total_ms = max_over_ranks(sum(step_ms), world)
    value = world * P * args.steps / (total_ms / 1e3)

    # per-view work counters of the last step (algorithmic bytes of the dominant kernel, k_chunks: the meshlet
    # tests read 64 B of bounds per tested meshlet and write 16 B per drawn entry; a span record is 16 B plus its
    # instance matrix 64 B, one per item and 512-meshlet window crossed; a chunk record is 16 B per window)
    st = [vg.read_stats(k) for k in range(P)]
    b_select = 0.0
    for s in st:
        sel = s["selected"][0] + s["selected"][1]
        spans = s["work"][0] + s["work"][1] + s["meshlets_tested"] / 512.0
        b_select += 64 * s["meshlets_tested"] + 16 * (sel - s["fast_emitted"]) + 80 * spans + 16 * s["meshlets_tested"] / 512.0
    # read mip 0, write mips 1 and up (a third of mip 0's texels): mip 0 is read from the depth image, not copied
    b_hzb = (4 * W * H + 4 * W * H / 3) * (P if occl else 0)
    work = {k: statistics.mean(float(s[k] if not isinstance(s[k], list) else s[k][0]) for s in st)
            for k in ("visible_cells", "instances_tested", "meshlets_tested", "meshlets_queued", "fast_emitted",
                      "selected", "survived",
                      "occluded_instances", "requested_indices", "rounds")}

    # plain per-view launches, timed per kernel kind on the launching stream
    vg.set_profiling(True)
    vg.kernel_times(reset=True)
    plain_ms = []
    for i in range(max(1, args.steps // 2)):
        for k in range(P):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            arr = (engine.View * 1)(views[k])
            engine.check(L.vgc_cut(vg.handle, arr, 1, k, sp))
            b.record(stream)
            b.synchronize()
            plain_ms.append(a.elapsed_time(b))
    kt = vg.kernel_times(reset=True)
    # the batched kernels with events around each launch: the same launch sequence as the graph, 32 views each
    for i in range(max(1, args.steps // 2)):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        vg.cut(views, first_slot=0, stream=sp, graph=False)
    kb = vg.kernel_times(reset=True)
    vg.set_profiling(False)
    plain_vps = 1e3 / statistics.mean(plain_ms)
    sel_ms, sel_n = kb["chunks0"]
    select_avg_ms = sel_ms / max(1, sel_n)
    # one k_chunks launch covers the step's P views
    achieved_select = b_select / (select_avg_ms / 1e3) / 1e9
    hzb_ms, hzb_n = kt["hzb"]
    peak, peak_kind = read_peaks()
    traffic = read_traffic("k_chunks") if args.config == "ruins" else None  # the capture is of the ruins workload

    # end to end through the C ABI with host buffers: depth images + views in, draw lists + counters out
    rt = ctypes.CDLL("libcudart.so.12")
    rt.cudaMemcpyAsync.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_void_p]
    out0 = vg.output(0)
    cw = engine.COUNTER_HEADER + out0.mesh_slots * 8
    h_counters = torch.empty(P * cw, dtype=torch.int32).pin_memory()
    cap = 1 << 18
    h_lists = torch.empty((P, cap, 4), dtype=torch.int32).pin_memory()
    outs = [vg.output(k) for k in range(P)]
    d2h_bytes = [0]

    # Each step uploads its depth images on a copy stream and waits for them before its cut; the next step's upload
    # starts once this step's cut has been queued (double-buffered images), so it overlaps this step's cut and
    # read-back. All of it lies between the two events on the timed stream.
    cs = torch.cuda.Stream()
    d_depth2 = [torch.empty_like(x) for x in d_depth]
    bufs = [d_depth, d_depth2]
    vsets = [views, [engine.make_view(c, engine.ViewParams(error_threshold=1.0, hzb=(k if occl else -1), state_slot=k,
                                                           depth_as_mip0=occl),
                                      depth=((d_depth2[k].data_ptr(), W, H) if occl else None))
                     for k, c in enumerate(spec.cameras)]]
    ev_in = [torch.cuda.Event(), torch.cuda.Event()]
    ev_used = [torch.cuda.Event(), torch.cuda.Event()]

    def upload(b):
        with torch.cuda.stream(cs):
            cs.wait_event(ev_used[b])  # the cut that read these buffers last has run
            for k in range(P if occl else 0):  # the step's occluder depth from pinned host memory
                bufs[b][k].copy_(h_depth[k], non_blocking=True)
            ev_in[b].record(cs)

    def step_e2e(i, last):
        b = i % 2
        stream.wait_event(ev_in[b])
        vg.cut(vsets[b], first_slot=0, stream=sp, graph=True)
        ev_used[b].record(stream)
        if not last:
            upload(1 - b)
        rt.cudaMemcpyAsync(h_counters.data_ptr(), out0.counters, P * cw * 4, 2, sp)
        stream.synchronize()
        c = h_counters.numpy().reshape(P, cw)
        nbytes = P * cw * 4
        for k in range(P):
            n = min(int(c[k, 2]), cap)
            if n:
                rt.cudaMemcpyAsync(h_lists[k].data_ptr(), outs[k].draw_list[0], n * 16, 2, sp)
                nbytes += n * 16
        d2h_bytes[0] = nbytes

    def run_e2e(steps):
        a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for e in ev_used:
            e.record(stream)
        a.record(stream)
        cs.wait_event(a)
        upload(0)
        for i in range(steps):
            step_e2e(i, i == steps - 1)
        z.record(stream)
        z.synchronize()
        return a.elapsed_time(z)

    run_e2e(2)
    torch.cuda.synchronize()
    e2e_total = max_over_ranks(run_e2e(args.steps), world)
    e2e_vps = world * P * args.steps / (e2e_total / 1e3)
    h2d_bytes = (P * W * H * 4 if occl else 0) + P * ctypes.sizeof(engine.View)

    clk = clocks.summary()
    cfg.update(bench_config(P, occl))
    lat = sorted(plain_ms)
    line = dict(
        metric=METRIC, value=value, unit="views/s", n_gpus=world, steps=args.steps, warmup=max(3, args.warmup),
        ms_per_step=statistics.mean(step_ms), higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f32",
        data="synthetic (seeded ruins-like scene; the reference's WebGPU scenes cannot run here)", config=cfg,
        batched_ms_per_view=statistics.mean(step_ms) / P,
        step_ms=[round(x, 4) for x in step_ms], host_ms_per_step=statistics.mean(host_ms[:len(step_ms)]),
        controller=dict(settle_steps=len(settle_ms), settle_ms=[round(x, 4) for x in settle_ms],
                        settled=quiet >= 8,
                        note="steps after the warm-up until no view redid its cut in eight consecutive steps (retry "
                             "rounds while the capacity controllers settle); the timed steps follow them"),
        plain_views_per_sec=plain_vps, batched_over_plain=value / world / plain_vps,
        p50_ms=lat[len(lat) // 2], p99_ms=lat[min(len(lat) - 1, int(math.ceil(0.99 * len(lat))) - 1)],
        latency_note="p50/p99: one view through the plain launch (HZB build + cut), CUDA events",
        e2e=dict(value=e2e_vps, unit="views/s", h2d_bytes_per_step=int(h2d_bytes), d2h_bytes_per_step=int(d2h_bytes[0]),
                 note="depth uploads on a copy stream, double-buffered: step i+1's upload overlaps step i's cut and "
                      "read-back; one event pair around all steps (inputs > L2, no flush)"),
        roofline=dict(bound="hbm", achieved=achieved_select, peak=peak, unit="GB/s", frac=achieved_select / peak,
                      traffic=traffic, kernel="k_chunks", peak_source=f"{peak_kind} hbm_gbs",
                      algorithmic_bytes_per_launch=b_select, avg_launch_ms=select_avg_ms,
                      note="k_chunks algorithmic bytes per view = 64 M (bounds of tested meshlets) + 16 (S - F) (drawn "
                           "entries) + 80 (items + M/512) (span records + instance matrices) + 16 M/512 (chunk records); "
                           "the scene's bounds sit in L2, so algorithmic GB/s can exceed DRAM GB/s"),
        kernels_plain={k: dict(ms=v[0], launches=v[1]) for k, v in kt.items() if v[1]},
        kernels_batched={k: dict(ms=v[0], launches=v[1]) for k, v in kb.items() if v[1]},
        work_per_view=work,
        hzb_achieved_gbs=b_hzb / (kb["hzb"][0] / max(1, kb["hzb"][1]) / 1e3) / 1e9 if (occl and kb["hzb"][1]) else None,
        hzb_mode=("each view's HZB is built from its depth image in the cut's launch sequence with mip 0 read from the "
                  "image (VGC_VIEW_DEPTH_AS_MIP0; the reference copies the depth texture into the HZB's first level: "
                  "about 30 us more per 32-view step here); draw lists identical (tested)") if occl else None,
        # per step: HZB strip stream + tail (with occlusion), reset, cells, and per capacity round k_instances,
        # k_chunks, k_instances_redo, k_finish (rounds 1-2 return at once when no view redoes)
        gpu_launches=args.steps * ((2 if occl else 0) + 2 + 3 * 4),
        clocks=clk,
    )
    line["autotune"] = autotune_report(vg, views, sp, stream, flush, args.steps)
    captured = parity_capture(vg, spec, views, occl, local) if rank == 0 else None
    vg.dispose()
    if world == 1 and args.config == "ruins" and not args.no_extras:
        extras = set(args.extras.split(","))
        if "serve_ruins" in extras:
            line["serve_ruins"] = run_serve_ruins(spec, args, plain_vps)
            line["served_views_per_sec"] = line["serve_ruins"]["saturated"]["views_per_sec"]
            line["served_over_plain"] = line["serve_ruins"]["served_over_plain"]
            rates = line["serve_ruins"]["poisson"]
            top = max(rates, key=float, default=None)  # p99 at the highest Poisson rate measured
            line["served_p99_ms"] = rates[top]["p99_ms"] if top else None
            line["served_p99_rate"] = float(top) if top else None
        if "batching" in extras:
            line["batching"] = run_batching(spec, args, flush, stream)
        if "occluders" in extras:
            line["occluders"] = run_occluders(spec, args, flush, stream)
        if "visibility" in extras:
            line["visibility"] = run_visibility(spec, args, flush, stream)
        if "updates" in extras:
            line["updates"] = run_updates(spec, args, flush, stream)
        if "large_world" in extras:
            line["large_world"] = run_large_world(spec, args, flush, stream)
        if "serve" in extras:
            line["serve"] = run_serve(spec, args)
    if rank == 0:
        runner = OraclePass(spec, occl)
        vps, cores, sample = cpu_baseline(spec, args.cpu_seconds, occl, runner)
        line["cpu_baseline"] = dict(value=vps, unit="views/s", cores=cores, kind="port", sample=sample)
        line["parity"] = parity_check(runner, captured)
        print(json.dumps(tail_order(line)), flush=True)


def autotune_report(vg, views, sp, stream, flush, steps: int) -> dict:
    """vgc_batch_autotune on a batched launch, after the figures that use the default shapes: the shapes it picks
    (meshlets per chunk, blocks per SM of the instance and meshlet kernels) and the device time per step before and
    after (L2 flushed before each step)."""
    import torch

    def step_ms():
        for _ in range(3):
            vg.cut(views, first_slot=0, stream=sp, graph=True)
        ms = []
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            vg.cut(views, first_slot=0, stream=sp, graph=True)
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        return statistics.mean(ms)

    default_ms = step_ms()
    tuned = vg.autotune(views, stream=sp, reps=3)
    tuned_ms = step_ms()
    return dict(chunk_meshlets=tuned["chunk_meshlets"], instances_blocks_per_sm=tuned["instances_blocks_per_sm"],
                chunks_blocks_per_sm=tuned["chunks_blocks_per_sm"], default_ms_per_step=default_ms,
                tuned_ms_per_step=tuned_ms, gain=default_ms / tuned_ms - 1.0,
                note="default shapes: 512 meshlets per chunk, the kernels' occupancy limits; `value` uses the defaults")


TAIL_KEYS = ("cpu_baseline", "parity", "roofline", "e2e", "plain_views_per_sec", "batched_over_plain", "p50_ms",
             "p99_ms", "served_views_per_sec", "served_over_plain", "served_p99_ms", "clocks", "value", "ms_per_step")


def tail_order(line: dict) -> dict:
    """The line with the figures a reader checks first moved to its end, where a truncated log still shows them
    (key order does not change the parsed line)."""
    head = {k: v for k, v in line.items() if k not in TAIL_KEYS}
    head.update({k: line[k] for k in TAIL_KEYS if k in line})
    return head


def percentile(sorted_values, q: float) -> float:
    return sorted_values[min(len(sorted_values) - 1, max(0, int(math.ceil(q * len(sorted_values))) - 1))]


def run_batching(ruins, args, flush, stream):
    """64 cameras over the ruins-like scene at 1280x720 / 1920x1080 / 3840x2160 with thresholds 0.5 / 1 / 2 px, each
    with 4 orthographic shadow cascades: 320 views in one CUDA-graph launch, grid sizes picked by the autotuner."""
    import torch
    from vgcut import engine, scenes
    # draw lists of 2^19 entries: at 2^17, 141 of the 320 views overflowed in a round (4K views at 0.5 px select
    # up to 1.9M meshlets), and their retried rounds coarsened the cuts
    vg = engine.VirtualGeometry(max_triangles=40_000_000, max_shadow_triangles=16_000_000, max_meshlets=1 << 19,
                                output_slots=320)
    for data, mats in zip(ruins.meshes, ruins.instances):
        vg.create_mesh(data, mats, cast_shadow=True)
    views = [engine.make_view(cam, engine.ViewParams(state_slot=k, fresh_state=True, **levers))
             for k, (cam, levers) in enumerate(scenes.batching_views(ruins))]
    sp = ctypes.c_void_p(stream.cuda_stream)

    def timed_steps():
        for _ in range(max(3, args.warmup)):
            vg.cut(views, first_slot=0, stream=sp, graph=True)
        torch.cuda.synchronize()
        ms = []
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            vg.cut(views, first_slot=0, stream=sp, graph=True)
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        return statistics.mean(ms)

    default_ms = timed_steps()
    tuned = vg.autotune(views, stream=sp, reps=3)
    tuned_ms = timed_steps()
    st = [vg.read_stats(k) for k in range(len(views))]
    overflow_share = statistics.mean(1.0 if s["overflow"] else 0.0 for s in st)
    rounds_mean = statistics.mean(s["rounds"] for s in st)
    cam_tris = statistics.mean(s["requested_indices"][0] / 3 for k, s in enumerate(st) if k % 5 == 0)
    casc_tris = statistics.mean(s["requested_indices"][1] / 3 for k, s in enumerate(st) if k % 5 != 0)
    vg.dispose()
    n = len(views)
    return dict(workload="batching: ruins-like scene, 64 cameras at 1280x720 / 1920x1080 / 3840x2160 with thresholds "
                         "0.5 / 1 / 2 px, each with 4 orthographic shadow cascades (splits 0.1-10-40-150-600 m): 320 "
                         "views in one CUDA-graph launch (64 camera cuts + 256 cascade cuts; 64 x (1 + 4) = 320, not "
                         "256)",
                views_per_sec=n / (tuned_ms / 1e3), ms_per_step=tuned_ms, views_per_step=n,
                camera_views_per_sec=64 / (tuned_ms / 1e3), cascade_views_per_sec=256 / (tuned_ms / 1e3),
                untuned_ms_per_step=default_ms, autotune=tuned,
                camera_cut_triangles_mean=cam_tris, cascade_cut_triangles_mean=casc_tris,
                overflow_share=overflow_share, rounds_mean=rounds_mean,
                capacity=dict(max_meshlets=1 << 19, max_triangles=40_000_000, max_shadow_triangles=16_000_000),
                note="cascades: no occlusion (the reference never occlusion-culls shadow cuts)")


def run_occluders(ruins, args, flush, stream):
    """Two-pass occlusion on the ruins-like scene, every mesh an occluder: per pose, the previous frame's camera cut is
    drawn depth-only with the current camera at 960x540 (the reference's half-resolution target), and the 32-view
    batched cut builds its HZB from those images in its own launch sequence."""
    import torch
    from vgcut import engine
    vg = engine.VirtualGeometry(max_triangles=10_000_000, max_shadow_triangles=4_000_000, max_meshlets=1 << 18,
                                output_slots=2 * len(ruins.cameras))
    for data, mats in zip(ruins.meshes, ruins.instances):
        vg.create_mesh(data, mats, occlusion_culling=True, occluder=True)
    P, W, H = len(ruins.cameras), 960, 540
    sp = ctypes.c_void_p(stream.cuda_stream)
    prev = [engine.make_view(c, engine.ViewParams(error_threshold=1.0, state_slot=k)) for k, c in enumerate(ruins.cameras)]
    # this frame's poses: the next pose of the spline (the last one repeats)
    cams = [ruins.cameras[min(k + 1, P - 1)] for k in range(P)]
    depth = [torch.empty((H, W), dtype=torch.float32, device="cuda") for _ in range(P)]
    views = [engine.make_view(c, engine.ViewParams(error_threshold=1.0, hzb=k, state_slot=P + k, fresh_state=True,
                                                   depth_as_mip0=True),
                              depth=(depth[k].data_ptr(), W, H)) for k, c in enumerate(cams)]
    open_views = [engine.make_view(c, engine.ViewParams(error_threshold=1.0, state_slot=P + k, fresh_state=True))
                  for k, c in enumerate(cams)]
    vg.cut(prev, first_slot=0, stream=sp, graph=True)  # the previous frame's cuts in slots 0..P-1

    # the 32 images in one call (vgc_occluder_depth_batch), its arguments packed once
    first_frame = engine.OccluderBatch(vg, list(range(P)), cams, [d.data_ptr() for d in depth])

    def occluder_pass():
        first_frame.run(W, H, stream=sp)

    def timed(fn):
        for _ in range(max(3, args.warmup)):
            fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        return statistics.mean(ms)

    occ_ms = timed(occluder_pass)
    both_ms = timed(lambda: (occluder_pass(), vg.cut(views, first_slot=P, stream=sp, graph=True)))
    drawn_hzb = [vg.read_stats(P + k)["drawn"][0] for k in range(P)]
    occluded = [vg.read_stats(P + k)["occluded_instances"] for k in range(P)]
    vg.cut(open_views, first_slot=P, stream=sp, graph=True)
    torch.cuda.synchronize()
    drawn_open = [vg.read_stats(P + k)["drawn"][0] for k in range(P)]
    covered = statistics.mean(float((d < 1).float().mean()) for d in depth)

    # End to end, the loop as a renderer runs it through the C ABI: each step uploads the views (host structs), draws
    # every view's previous cut as occluders with its camera, cuts with the HZB built from those images, and reads
    # the counters and draw lists back into pinned host memory; cuts alternate between two slot sets, so each step's
    # occluders are the previous step's cuts. No depth image crosses PCIe.
    rt = ctypes.CDLL("libcudart.so.12")
    rt.cudaMemcpyAsync.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_void_p]
    cw = engine.COUNTER_HEADER + vg.output(0).mesh_slots * 8
    cap = 1 << 18
    h_counters = torch.empty(2 * P * cw, dtype=torch.int32).pin_memory()
    h_lists = torch.empty((P, cap, 4), dtype=torch.int32).pin_memory()
    loop_views = [[engine.make_view(c, engine.ViewParams(error_threshold=1.0, hzb=k, state_slot=s * P + k,
                                                         depth_as_mip0=True),
                                    depth=(depth[k].data_ptr(), W, H)) for k, c in enumerate(cams)] for s in (0, 1)]
    d2h = [0]
    outs = [vg.output(k) for k in range(2 * P)]

    occl = [engine.OccluderBatch(vg, [src * P + k for k in range(P)], cams, [d.data_ptr() for d in depth])
            for src in (0, 1)]

    def loop_device(i):
        src, dst = (i + 1) % 2, i % 2
        occl[src].run(W, H, stream=sp)
        vg.cut(loop_views[dst], first_slot=dst * P, stream=sp, graph=True)
        return dst

    def loop_step(i):
        dst = loop_device(i)
        rt.cudaMemcpyAsync(h_counters.data_ptr(), outs[dst * P].counters, P * cw * 4, 2, sp)
        stream.synchronize()
        c = h_counters.numpy()[:P * cw].reshape(P, cw)
        nbytes = P * cw * 4
        for k in range(P):
            n = min(int(c[k, 2]), cap)
            if n:
                rt.cudaMemcpyAsync(h_lists[k].data_ptr(), outs[dst * P + k].draw_list[0], n * 16, 2, sp)
                nbytes += n * 16
        d2h[0] = nbytes

    vg.cut(prev, first_slot=P, stream=sp, graph=True)  # slot set 1 holds "the previous frame" for step 0
    for i in range(max(3, args.warmup)):
        loop_step(i)
    torch.cuda.synchronize()
    a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for i in range(args.steps):
        loop_step(i)
    z.record(stream)
    z.synchronize()
    loop_ms = a.elapsed_time(z)
    # the same loop on the device alone (L2 flushed before each step), and its occluder pass alone: the steady state,
    # where each view's occluders are its previous occlusion-culled cut
    steady_ms, steady_occ = [], []
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        a, m, z = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        a.record(stream)
        src, dst = (i + 1) % 2, i % 2
        occl[src].run(W, H, stream=sp)
        m.record(stream)
        vg.cut(loop_views[dst], first_slot=dst * P, stream=sp, graph=True)
        z.record(stream)
        z.synchronize()
        steady_ms.append(a.elapsed_time(z))
        steady_occ.append(a.elapsed_time(m))
    steady_drawn = statistics.mean(vg.read_stats(((args.steps - 1) % 2) * P + k)["drawn"][0] for k in range(P))
    vg.dispose()
    return dict(workload=f"two-pass occlusion, ruins-like scene, {P} poses: previous camera cut drawn depth-only with "
                         f"the next pose at {W}x{H}, HZB built in the batched cut's launch sequence",
                occluder_pass_ms_per_view=occ_ms / P, two_pass_ms_per_step=both_ms, views_per_sec=P / (both_ms / 1e3),
                occluder_coverage=covered, occluded_instances_mean=statistics.mean(occluded),
                drawn_meshlets_with_hzb=statistics.mean(drawn_hzb), drawn_meshlets_without=statistics.mean(drawn_open),
                steady=dict(occluder_pass_ms_per_view=statistics.mean(steady_occ) / P,
                            ms_per_step=statistics.mean(steady_ms), views_per_sec=P / (statistics.mean(steady_ms) / 1e3),
                            occluder_meshlets_mean=steady_drawn,
                            note="each view's occluders are its previous occlusion-culled cut (a renderer's steady "
                                 "state); the figures above draw an unculled previous cut"),
                e2e=dict(value=P * args.steps / (loop_ms / 1e3), unit="views/s",
                         h2d_bytes_per_step=P * ctypes.sizeof(engine.View), d2h_bytes_per_step=int(d2h[0]),
                         note="two-pass loop through the C ABI: views up, occluder pass from the previous step's cuts, "
                              "cut with the HZB built from them, counters and draw lists back to pinned host memory; "
                              "no depth upload; one event pair around all steps"))


def run_visibility(ruins, args, flush, stream):
    """The loop closed headlessly: per pose, the camera cut (batched, 32 views per launch), its index expansion and
    the visibility buffer drawn from the expanded indices at 1920x1080 (vertex pulling, draw-distance fade, LOD blend
    mask), one view after the other through one index buffer."""
    import torch
    from vgcut import engine
    vg = engine.VirtualGeometry(max_triangles=10_000_000, max_shadow_triangles=4_000_000, max_meshlets=1 << 18,
                                output_slots=len(ruins.cameras))
    for data, mats in zip(ruins.meshes, ruins.instances):
        vg.create_mesh(data, mats, vertex_data=True)
    P, W, H = len(ruins.cameras), 1920, 1080
    sp = ctypes.c_void_p(stream.cuda_stream)
    views = [engine.make_view(c, engine.ViewParams(error_threshold=1.0, state_slot=k, fresh_state=True))
             for k, c in enumerate(ruins.cameras)]
    cap = 10_000_000 * 3
    idx = torch.empty(cap, dtype=torch.int32, device="cuda")
    vis = torch.empty((H, W), dtype=torch.int64, device="cuda")

    def draw_all():
        for k in range(P):
            vg.expand(k, 0, idx.data_ptr(), cap, stream=sp)
            vg.visibility(k, 0, ruins.cameras[k], idx.data_ptr(), cap, vis.data_ptr(), W, H, stream=sp)

    def timed(fn):
        for _ in range(max(3, args.warmup)):
            fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        return statistics.mean(ms)

    vg.cut(views, first_slot=0, stream=sp, graph=True)
    torch.cuda.synchronize()
    draw_ms = timed(draw_all)
    loop_ms = timed(lambda: (vg.cut(views, first_slot=0, stream=sp, graph=True), draw_all()))
    torch.cuda.synchronize()
    tris = statistics.mean(vg.read_stats(k)["requested_indices"][0] / 3 for k in range(P))
    covered = float((vis != engine.VIS_EMPTY).float().mean())
    vg.dispose()
    return dict(workload=f"closed loop, ruins-like scene, {P} poses: batched camera cut, index expansion and a "
                         f"{W}x{H} visibility buffer from the expanded indices, per view",
                expand_and_visibility_ms_per_view=draw_ms / P, loop_ms_per_step=loop_ms,
                views_per_sec=P / (loop_ms / 1e3), triangles_per_view=tris,
                triangles_per_sec=tris * P / (draw_ms / 1e3), coverage_last_view=covered)


def run_updates(ruins, args, flush, stream):
    """Instance updates and the Morton re-sort on the ruins-like scene: every instance of every mesh moves to another
    instance's place (commitInstances on the device), which leaves the 128-instance cells spread over the whole
    world; vgc_instances_resort then restores compact cells. Batched views/s of the 32 poses before, after the move
    and after the re-sort (no occlusion)."""
    import numpy as np
    import torch
    from vgcut import engine, scenes
    vg = engine.VirtualGeometry(max_triangles=10_000_000, max_shadow_triangles=4_000_000, max_meshlets=1 << 18,
                                output_slots=len(ruins.cameras))
    meshes = scenes.load_into(vg, ruins)
    P = len(ruins.cameras)
    sp = ctypes.c_void_p(stream.cuda_stream)
    views = [engine.make_view(c, engine.ViewParams(error_threshold=1.0, state_slot=k, fresh_state=True))
             for k, c in enumerate(ruins.cameras)]

    def views_per_sec():
        for _ in range(max(3, args.warmup)):
            vg.cut(views, first_slot=0, stream=sp, graph=True)
        torch.cuda.synchronize()
        ms = []
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            vg.cut(views, first_slot=0, stream=sp, graph=True)
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        return P / (statistics.mean(ms) / 1e3)

    def cell_radius():
        cells, _ = vg.debug_scene()
        return float(cells[:, 3].mean())

    before, r_before = views_per_sec(), cell_radius()
    rng = np.random.default_rng(31)
    moved = []
    for mats in ruins.instances:
        m = np.array(mats, np.float32).reshape(-1, 16)
        perm = rng.permutation(len(m))
        m[:, 12:15] = m[perm, 12:15]
        moved.append(m)
    torch.cuda.synchronize()
    t = time.perf_counter()
    for mesh, m in zip(meshes, moved):
        mesh.set_matrices(m)
        mesh.commit_instances()  # synchronous: upload + cells on the device
    commit_ms = (time.perf_counter() - t) * 1e3
    scattered, r_scattered = views_per_sec(), cell_radius()
    torch.cuda.synchronize()
    t = time.perf_counter()
    for mesh in meshes:
        mesh.resort()  # synchronous: codes, sort, permutation, cells on the device; host mirror follows
    resort_ms = (time.perf_counter() - t) * 1e3
    resorted, r_resorted = views_per_sec(), cell_radius()
    n = sum(len(m) for m in moved)
    vg.dispose()
    return dict(workload=f"ruins-like scene, {n} instances: every instance moved to another's place, then re-sorted; "
                         f"{P} poses, batched, no occlusion",
                commit_ms=commit_ms, resort_ms=resort_ms, instances=n,
                views_per_sec_before=before, views_per_sec_moved=scattered, views_per_sec_resorted=resorted,
                mean_cell_radius_before=r_before, mean_cell_radius_moved=r_scattered,
                mean_cell_radius_resorted=r_resorted,
                note="commit and re-sort times are host wall clock around the synchronous calls (all meshes)")


def run_large_world(ruins, args, flush, stream):
    """3M instances over 6 km x 6 km, 16 poses at 3840 x 2160, triangleBudget 6M by the device histogram search,
    maxDrawDistance 400 m on the small-mesh bucket: batched views/s and how the search met the budget."""
    import torch
    from vgcut import engine, scenes
    spec = scenes.large_world(ruins.meshes, ruins.mesh_triangles, ruins.notes["weight_exponent"])
    small = set(spec.notes["small_meshes"])
    vg = engine.VirtualGeometry(max_triangles=12_000_000, max_shadow_triangles=4_000_000, max_meshlets=1 << 18,
                                output_slots=len(spec.cameras))
    for i, (data, mats) in enumerate(zip(spec.meshes, spec.instances)):
        vg.create_mesh(data, mats, max_draw_distance=(400.0 if i in small else float("inf")))
    budget = spec.notes["triangle_budget"]
    # the search range reaches 24 px: at 3840 x 2160 over 3M instances no threshold in the reference's default
    # [0.5, 3] brings the camera cut down to 6M triangles
    trange = (0.5, 24.0)
    views = [engine.make_view(c, engine.ViewParams(triangle_budget=budget, threshold_range=trange, state_slot=k,
                                                   fresh_state=True))
             for k, c in enumerate(spec.cameras)]
    sp = ctypes.c_void_p(stream.cuda_stream)
    for _ in range(max(3, args.warmup)):
        vg.cut(views, first_slot=0, stream=sp, graph=True)
    torch.cuda.synchronize()
    ms = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        vg.cut(views, first_slot=0, stream=sp, graph=True)
        b.record(stream)
        b.synchronize()
        ms.append(a.elapsed_time(b))
    st = [vg.read_stats(k) for k in range(len(views))]
    tune = autotune_report(vg, views, sp, stream, flush, args.steps)
    drawn = [s["requested_indices"][0] // 3 for s in st]
    pred = [s["predicted_triangles"] for s in st]
    out = dict(workload=f"large world: {spec.instance_count} instances of {len(spec.meshes)} meshes over 6x6 km "
                        f"({spec.notes['placement']}), {len(views)} poses at 3840x2160, triangleBudget 6M, "
                        f"maxDrawDistance 400 m on the 10 smallest meshes",
               views_per_sec=len(views) * len(ms) / (sum(ms) / 1e3), ms_per_step=statistics.mean(ms),
               budget=budget, predicted_triangles_mean=statistics.mean(pred), predicted_over_budget=max(pred) / budget,
               camera_cut_triangles_mean=statistics.mean(drawn),
               threshold_range=list(trange),
               thresholds=[min(s["effective_threshold"] for s in st), max(s["effective_threshold"] for s in st)],
               autotune=tune,
               note="predicted = the histogram's plain-cut triangles at the chosen threshold; the drawn camera cut adds "
                    "the LOD-blend band's overlap")
    vg.dispose()
    return out


class ServeDriver:
    """Drives a server with a request list: submits (arrival s, request index) items - at their arrival times when
    paced - from a submitter thread, waits for and releases each, and summarises latency (submit -> completion seen
    by the server, host steady clock) and throughput."""

    def __init__(self, server, scene_of, views):
        self.server, self.scene_of, self.views = server, scene_of, views

    def run(self, items, paced: bool):
        base = self.server.stats()
        tickets = [0] * len(items)
        ready = threading.Semaphore(0)

        def submitter():
            t0 = time.perf_counter()
            for j, (at, i) in enumerate(items):
                while paced:
                    dt = t0 + at - time.perf_counter()
                    if dt <= 0:
                        break
                    # a sleep, even of 0, lets the waiting thread take the interpreter lock: a spin without one
                    # keeps it for the interpreter's whole switch interval and starves the releases
                    time.sleep(dt - 2e-4 if dt > 3e-4 else 0)
                tickets[j] = self.server.submit(self.scene_of[i], self.views[i])
                ready.release()

        th = threading.Thread(target=submitter)
        th.start()
        from vgcut import engine
        raw = [engine.ServeResult() for _ in items]  # filled as results come, read after the run
        for j in range(len(items)):
            ready.acquire()
            self.server.wait_into(tickets[j], raw[j])
            self.server.release(tickets[j])
        th.join()
        results = [self.server.result_dict(r) for r in raw]
        st = self.server.stats()
        delta = {k: st[k] - base[k] for k in ("batches", "views_launched", "multi_scene_batches")}
        return results, delta, st

    @staticmethod
    def summary(results, delta):
        lat = sorted((r["done_us"] - r["submit_us"]) / 1e3 for r in results)
        span_s = (max(r["done_us"] for r in results) - min(r["submit_us"] for r in results)) / 1e6
        return dict(views_per_sec=len(results) / span_s, p50_ms=percentile(lat, 0.5), p99_ms=percentile(lat, 0.99),
                    p999_ms=percentile(lat, 0.999), mean_batch=delta["views_launched"] / max(1, delta["batches"]),
                    batches=delta["batches"], multi_scene_batches=delta["multi_scene_batches"],
                    batch_gpu_ms_mean=statistics.mean(r["batch_gpu_ms"] for r in results),
                    rounds_mean=statistics.mean(r["stats"]["rounds"] for r in results),
                    overflow_share=statistics.mean(1.0 if r["stats"]["overflow"] else 0.0 for r in results))

    def poisson(self, rate: float, n: int, n_requests: int, seed: int = 17, warmup: int = 200):
        """Poisson arrivals at `rate`: `warmup` requests at the same rate first (not summarised), then `n`."""
        import numpy as np
        rng = np.random.default_rng(seed)
        if warmup:
            w = np.cumsum(rng.exponential(1.0 / rate, warmup))
            self.run([(float(w[j]), (n + j) % n_requests) for j in range(warmup)], True)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
        res, delta, st = self.run([(float(arrivals[j]), j % n_requests) for j in range(n)], True)
        out = self.summary(res, delta)
        slow = sorted(range(n), key=lambda j: res[j]["done_us"] - res[j]["submit_us"])[-max(1, n // 100):]
        out.update(offered_per_sec=n / float(arrivals[-1]), requests=n, warmup_requests=warmup,
                   slowest_percent_at=[round(float(arrivals[j]) / float(arrivals[-1]), 3) for j in sorted(slow)][:20])
        return out, st


# Serving on one scene: output slots enough that admission does not cut batches short while results wait to be read
# and released, and a linger that lets a short batch fill while another one runs (none when the GPU is idle).
SERVE_SLOTS = 1024
SERVE_LINGER_US = 800


@contextlib.contextmanager
def driver_without_gc():
    """Python's garbage collector paused while the serving driver paces requests and reads results, so that no
    collection pass delays a submission or a read-out (the server itself is native)."""
    gc.collect()
    gc.disable()
    try:
        yield
    finally:
        gc.enable()


def run_serve_ruins(ruins, args, plain_vps: float):
    """Serving on the ruins-like scene (113,106 instances) at 1920 x 1080: requests (spline pose with its prebuilt
    HZB, threshold U[0.5, 2] px), continuous batching on 4 streams; a saturated burst and Poisson arrivals at
    2k-20k requests/s, beside the plain per-view launch."""
    import numpy as np
    from vgcut import engine, scenes
    P = len(ruins.cameras)
    # output capacity for the finest request: at 0.5 px a 1080p view of this scene selects up to 334k meshlets and
    # 33.8M triangles (oracle, all poses), so a fresh request's cut fits in its first round
    cap_meshlets, cap_triangles = 1 << 19, 40_000_000
    vg = engine.VirtualGeometry(max_triangles=cap_triangles, max_shadow_triangles=4_000_000, max_meshlets=cap_meshlets,
                                output_slots=1)
    scenes.load_into(vg, ruins, occlusion_culling=True)
    for k in range(P):
        vg.build_hzb(k, ruins.depth_images[k])
    rng = np.random.default_rng(23)
    n_req = 4096
    poses = rng.integers(P, size=n_req)
    thresholds = rng.uniform(0.5, 2.0, n_req)
    views = [engine.make_view(ruins.cameras[int(k)], engine.ViewParams(error_threshold=float(t), hzb=int(k)))
             for k, t in zip(poses, thresholds)]
    server = engine.Server([vg], streams=4, max_batch=64, slots_per_scene=SERVE_SLOTS, linger_us=SERVE_LINGER_US)
    drv = ServeDriver(server, [0] * n_req, views)
    rates = {}
    try:
        with driver_without_gc():
            drv.run([(0.0, i) for i in range(512)], False)  # warm-up
            res, delta, _ = drv.run([(0.0, i) for i in range(n_req)], False)
            saturated = drv.summary(res, delta)
            for rate in (2_000.0, 5_000.0, 10_000.0, 20_000.0):
                if rate > 0.9 * saturated["views_per_sec"]:
                    continue
                rates[f"{int(rate)}"], _ = drv.poisson(rate, int(min(40_000, rate * 2.0)), n_req)
    finally:
        server.close()
        vg.dispose()
    return dict(workload=f"serving, ruins-like scene: {ruins.instance_count} instances, 1920x1080 requests (one of "
                         f"{P} spline poses with its prebuilt HZB, threshold U[0.5, 2] px), 4 streams, batches <= 64",
                saturated=dict(saturated, requests=n_req, note="burst submitted at once: the server's capacity"),
                poisson=rates, plain_views_per_sec=plain_vps,
                served_over_plain=saturated["views_per_sec"] / plain_vps if plain_vps else None,
                capacity=dict(max_meshlets=cap_meshlets, max_triangles=cap_triangles, slots=SERVE_SLOTS),
                linger_us=SERVE_LINGER_US,
                latency_note="submit -> completion seen by the server (host steady clock); Poisson arrivals, about "
                             "2 s of requests per rate, after 200 warm-up requests at the same rate")


def serve_capacity(instances: int) -> tuple:
    """Output capacity of a serving scene's views, by its size: draw-list meshlets and camera-cut triangles grow with
    the instances a 4K view can see, so that a fresh request's cut fits after its capacity rounds."""
    meshlets = 1 << max(17, min(20, (max(1, instances) - 1).bit_length()))
    triangles = int(min(48_000_000, max(10_000_000, 16 * instances)))
    return meshlets, triangles


def run_serve(ruins, args):
    """The serving loop: 16 resident scenes of 10k-3M instances, a seeded Poisson request stream (pose, 720p / 1080p
    / 4K, threshold U[0.5, 2], budget on a quarter), admission by output slots and HBM budget, 4 streams, batches
    across scenes."""
    from vgcut import engine, scenes
    specs = scenes.serving_scenes(ruins.meshes, ruins.mesh_triangles, ruins.notes["weight_exponent"])
    vgs, caps = [], []
    for sp in specs:
        meshlets, triangles = serve_capacity(sp.instance_count)
        if args.serve_max_meshlets:
            meshlets = args.serve_max_meshlets
        if args.serve_max_triangles:
            triangles = args.serve_max_triangles
        vg = engine.VirtualGeometry(max_triangles=triangles, max_shadow_triangles=2_000_000, max_meshlets=meshlets,
                                    output_slots=1)
        scenes.load_into(vg, sp)
        vgs.append(vg)
        caps.append((sp.instance_count, meshlets, triangles))
    reqs = scenes.request_stream(specs, args.serve_requests, args.serve_rate)
    views = [engine.make_view(cam, engine.ViewParams(error_threshold=t, triangle_budget=b, threshold_range=(0.5, 3.0)))
             for _, _, cam, t, b in reqs]
    budget = 16 << 30
    server = engine.Server(vgs, streams=4, max_batch=64, slots_per_scene=64, hbm_budget_bytes=budget,
                           linger_us=SERVE_LINGER_US)
    drv = ServeDriver(server, [r[1] for r in reqs], views)
    try:
        with driver_without_gc():
            drv.run([(0.0, i) for i in range(256)], False)  # warm-up
            # capacity: the whole burst submitted at once
            n_sat = min(len(reqs), 4096)
            res, delta, _ = drv.run([(0.0, i) for i in range(n_sat)], False)
            saturated = drv.summary(res, delta)
            # latency under a Poisson stream at 70% of that capacity (or the requested rate, if lower)
            rate = min(args.serve_rate, 0.7 * saturated["views_per_sec"])
            paced, st = drv.poisson(rate, min(len(reqs), max(1000, int(rate * 4.0))), len(reqs))
    finally:
        server.close()
        for vg in vgs:
            vg.dispose()
    return dict(workload=f"serving: {len(specs)} resident scenes of {min(s.instance_count for s in specs)}-"
                         f"{max(s.instance_count for s in specs)} instances ({sum(s.instance_count for s in specs)} total) "
                         f"of the ruins meshes; seeded requests (scene, ground pose, 720p/1080p/4K, threshold U[0.5,2], "
                         f"triangleBudget 2M/4M/8M on ~25%)",
                saturated=dict(saturated, requests=n_sat, note="burst submitted at once: the server's capacity"),
                poisson=dict(paced, note="Poisson arrivals at min(requested rate, 70% of capacity)"),
                max_in_flight=st["max_in_flight"], hbm_budget_bytes=budget, max_bytes_in_use=st["max_bytes_in_use"],
                latency_note="submit -> completion seen by the server, host steady clock",
                config=dict(streams=4, max_batch=64, slots_per_scene=64, cross_scene=True, linger_us=SERVE_LINGER_US,
                            capacity_by_scene=[dict(instances=i, max_meshlets=m, max_triangles=t) for i, m, t in caps]))


def main():
    args = parse()
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            barrier(world)
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
