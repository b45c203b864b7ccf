"""Benchmark: primary visibility + shading of a stereo VR frame on one B200 per rank.

Workload (the configuration the headline metric is quoted on): a 995,072-triangle seeded
procedural scene (256x256-quad heightfield + 72,000 boxes), two eyes of 1080x1200 with a
64 mm IPD, per-pixel sample positions warped by barrel distortion
r' = r (1 + 0.22 r^2 + 0.24 r^4), 8x MSAA, GGX shading with 1 directional + 4 point lights.

One step = one stereo frame through the full path on the GPU: block cull, tile cull,
intersect + G-buffer compression + shade + resolve, remap to the eye images.

value  : Gsamples/s with everything resident in HBM (device images), device-timed with
         CUDA events per frame; an L2 flush (a 256 MiB write) separates frames and is not timed.
e2e    : the same metric through the C ABI with CPU_MEMORY render targets: the per-frame
         camera transforms go in, both RGBA8 images come back to host memory inside the timing.
Multi-GPU (torchrun): replicas - each rank renders its own stereo frame; no collective on
the data path. value = frames of all ranks / max-over-ranks time.

--impl reference runs the reference's own traversal + intersect/shade code, compiled from the
reference sources into oracle/_ref (else the oracle port), on the host cores, one full stereo
frame per step, without loading this repository's CUDA library.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W, H, MSAA, IPD = 1080, 1200, 8, 0.064


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="hvvr_b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="stereo", choices=["stereo", "batched", "served", "foveated", "c1"],
                    help="stereo: the headline 2x1080x1200 frame; c1: one 640x480 1xMSAA grid view of the 57k-triangle "
                         "scene; batched: 64 views over 4 scenes, batched vs plain; "
                         "served: Poisson request arrivals against the render server; foveated: polar foveated "
                         "stereo, 16xMSAA, resolved to 1440x1600 per eye, gaze in a 10-degree saccade")
    ap.add_argument("--rates", default="100,250,500,1000,2000,5000,10000,20000", help="served: arrival rates, req/s")
    ap.add_argument("--seconds", type=float, default=1.0, help="served: arrival window per rate")
    ap.add_argument("--views", type=int, default=64)
    ap.add_argument("--max-batch-views", type=int, default=64, help="served: views per throughput batch")
    ap.add_argument("--throughput-slots", type=int, default=3, help="served: throughput batches in flight")
    ap.add_argument("--latency-slots", type=int, default=1, help="served: latency-class slots")
    ap.add_argument("--served-cull-cap", type=int, default=3,
                    help="served: throughput batches' tile-cull CTAs per SM (0 = no cap)")
    ap.add_argument("--latency-frames", type=int, default=500,
                    help="stereo: frames of the p50/p99 latency run after the timed steps")
    ap.add_argument("--profile", action="store_true",
                    help="case for ncu: the stereo frame (or with --workload foveated the foveated frame), 3 frames")
    ap.add_argument("--visit-clocks", action="store_true",
                    help="per-visit phase cycles of the tile cull on the stereo frame, from the profiling build "
                         "(make -C hvvr_b200/csrc visit-clocks); not a benchmark line")
    return ap.parse_args()


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # nvidia-smi takes a moment to start: begin the timed region once it samples
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < 5.0 and self.proc.poll() is None:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.02)

    def stop(self):
        """The samples' summary, or {} when nvidia-smi gave none."""
        if not self.proc:
            return {}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        for r in rows:
            for name, v in zip(["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"], r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": float(rows[0][2]),
                "reasons": sorted(reasons), "samples": len(rows)}


def max_over_ranks(x, dist, device):
    """Max of a float over all ranks (identity without a process group)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(samples_per_frame, frames, seconds, world):
    """Whole-job Gsamples/s for replicas: every rank renders `frames` frames; seconds is the max over ranks."""
    return world * samples_per_frame * frames / seconds / 1e9


import numpy as np  # noqa: E402


def stereo_setup(hv, scenes, sc, target_cuda, torch):
    rc = hv.Raycaster(tri_index_capacity=128 << 20)
    rc.create_model(sc)
    for l in sc.lights:
        rc.create_light(l)
    smp = scenes.barrel_samples(W, H)
    eyes = scenes.stereo_eyes(IPD)
    cams, images = [], []
    for xf in eyes:
        cam = rc.create_camera(scenes.viewport_for(W, H))
        if target_cuda:
            img = torch.zeros((H, W), dtype=torch.int32, device="cuda")
            cam.set_render_target(W, H, device_ptr=img.data_ptr())
            images.append(img)
        else:
            cam.set_render_target(W, H)
        cam.set_samples(smp)
        cam.set_camera_to_world(xf)
        cam.set_msaa(MSAA)
        cams.append(cam)
    return rc, cams, images, smp, eyes


def sample_setup_ms(hv, scenes):
    """Wall time of one eye's sample hierarchy (SampleData: clustering, tile and block frusta,
    beams, image remap; 1,296,000 barrel-distorted samples), built on the device and on the host
    (Camera.prepare, which returns once the setup is on the device)."""
    smp = scenes.barrel_samples(W, H)
    out = {"samples": int(len(smp))}
    for name, mode in (("device", hv.HVVR_SETUP_DEVICE), ("host", hv.HVVR_SETUP_HOST)):
        best = None
        for _ in range(2 if name == "device" else 1):
            rc = hv.Raycaster(sample_setup=mode)
            cam = rc.create_camera(scenes.viewport_for(W, H))
            cam.set_render_target(W, H)
            cam.set_samples(smp)
            t0 = time.perf_counter()
            cam.prepare()
            dt = (time.perf_counter() - t0) * 1e3
            rc.close()
            best = dt if best is None else min(best, dt)
        out[name] = best
    return out


def frame_counts(hv, scenes, sc):
    """Counts of one captured stereo frame (both eyes) that define the algorithmic bytes."""
    rc, cams, _, _, _ = stereo_setup(hv, scenes, sc, False, None)
    for c in cams:
        c.set_capture(hv.HVVR_CAPTURE_HITS)
    rc.render()
    rc.render()
    ctr = rc.counters()
    out = {"padded_samples": 0, "tiles": 0, "list_entries": 0, "unique_hits": 0, "node_visits": 0,
           "tested_entries": int(ctr[4]), "tested_warp_entries": int(ctr[5]), "longest_tile_node_visits": 0}
    for cam in cams:
        blocks, tiles, padded, msaa = cam.layout()
        n, tri, mask = cam.gbuffer()
        out["padded_samples"] += padded
        out["tiles"] += tiles
        out["list_entries"] += cam.list_total()
        out["unique_hits"] += int(((tri != 0xFFFFFFFF) & (mask != 0)).sum())
        costs = cam.tile_costs().astype(np.int64)
        out["node_visits"] += int(costs.sum())
        out["longest_tile_node_visits"] = max(out["longest_tile_node_visits"], int(costs.max()))
    rc.close()
    return out


def intersect_bytes(c):
    """Compulsory HBM bytes of a frame's intersect+shade launches: per sample 48 B beam + 4 B RGBA8
    written; per list entry 4 B index + 48 B triangle; per unique (sample, triangle) hit 16 B shade
    record + 3 x 32 B vertices + 64 B material + 48 B triangle."""
    return c["padded_samples"] * (48 + 4) + c["list_entries"] * (4 + 48) + c["unique_hits"] * (16 + 96 + 64 + 48)


def intersect_flops(c, msaa):
    """FP32 operations of a frame's executed intersect tests: every (warp of 32 samples, surviving
    list entry) pair whose tests ran (counted on the device; pairs the per-warp depth bound skips are
    not counted), 72 flops of per-(sample, triangle) setup (IntersectTriangleThread +
    GetDifferentials) and 16 per subsample test (7 FMA + 2 adds) per sample."""
    return c["tested_warp_entries"] * 32 * (72 + 16 * msaa)


def fp32_line(c, msaa, launch_ms, sm_mhz):
    """achieved FP32 rate of the intersect launch (timed alone) against the FP32 peak at the sampled
    SM clock (148 SMs x 128 FP32 lanes x 2 flops per FMA: a nominal figure; no FP32 peak is measured)"""
    flops = intersect_flops(c, msaa)
    peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
    achieved = flops / (launch_ms * 1e-3) / 1e12
    return {"flops_per_launch": flops, "launch_ms": launch_ms, "achieved_tflops": achieved, "peak_tflops": peak,
            "frac": achieved / peak, "peak_source": "nominal at %.0f MHz" % sm_mhz,
            "counted": "executed subsample tests only (device counter)"}


def cull_bytes(c):
    """Compulsory HBM bytes of a frame's tile-cull launches: one 128 B BVH node per visit, 4 B per
    list entry written, 96 B of corner rays per tile."""
    return c["node_visits"] * 128 + c["list_entries"] * 4 + c["tiles"] * 96


def stereo_config(world):
    """The workload's description, shared by both arms so that their lines name the same config."""
    return {"workload": "stereo 2x1080x1200 8xMSAA barrel-distorted samples, 995,072-triangle scene, "
                        "one frame (both eyes) per step", "samples_per_frame": 2 * W * H,
            "parallelism": "replicas x%d" % world,
            "l2": "GPU arm: flushed between frames (256 MiB write, untimed); CPU arm: n/a"}


def library_free_imports():
    """The scene generator, the ABI structs and the reference bindings without loading
    libhvvr_b200.so: the package is registered as a bare namespace, so its __init__ (which loads the
    CUDA library) does not run. The reference arm uses nothing of this repository's product."""
    import types
    if "hvvr_b200" not in sys.modules:
        pkg = types.ModuleType("hvvr_b200")
        pkg.__path__ = [os.path.join(ROOT, "hvvr_b200")]
        sys.modules["hvvr_b200"] = pkg
    from hvvr_b200 import _abi, scenes
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    return _abi, scenes, pyoracle


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return ""


def reference_stereo(scenes, pyoracle, sc=None):
    """The reference's own code (oracle/_ref, else the oracle port) set up for the stereo frame:
    the scene with the reference's GenerateTopology, uploaded and refit, and one camera per eye
    with its SampleData, kept across frames as the reference's Raycaster keeps them."""
    kind = "reference" if pyoracle.Reference.available() else "port"
    if sc is None:
        sc = scenes.scene_c2()
    ref = pyoracle.Reference() if kind == "reference" else None
    if sc.nodes is None:
        if ref is None:
            raise RuntimeError("no reference build to run GenerateTopology")
        sc.verts, sc.tri_shade, sc.nodes = ref.generate_topology(sc)
    smp = scenes.barrel_samples(W, H)
    vp = scenes.viewport_for(W, H)
    if ref is not None:
        sessions = [ref.session(sc, smp, vp, W, H, MSAA) for _ in range(2)]
    else:
        sessions = None
    return kind, sc, smp, sessions


def reference_frame(kind, sessions, sc, smp, eyes, threads, pyoracle, scenes, rows=None):
    """One stereo frame (or, with rows, a band of rows of both eyes) through the reference's path."""
    if kind == "reference" and rows is None:
        for s, xf in zip(sessions, eyes):
            s.frame(xf, threads)
        return 2 * len(smp)
    crop = smp if rows is None else smp[(smp["pixel"][:, 1] >= rows[0]) & (smp["pixel"][:, 1] < rows[1])]
    impl = pyoracle.Reference() if kind == "reference" else pyoracle.Oracle()
    for xf in eyes:
        impl.render(sc, crop, xf, scenes.viewport_for(W, H), W, H, MSAA, fp_mode=pyoracle._abi.HVVR_FP_STRICT,
                    threads=threads,
                    want=("colors",))
    return 2 * len(crop)


def run_reference_arm(args, rank):
    """The reference's own path on the host cores, on this arm's config: the full stereo frame of
    the benchmark (995,072 triangles, 2x1080x1200 barrel samples, 8xMSAA) per step, with the
    reference's GenerateTopology, SampleData, frustum transform, two-level AVX traversal run like
    cullThread on all host threads, and its intersect/shade code per tile on the same threads.
    Scene upload and sample setup happen once, before the steps, as in the reference's Raycaster.
    Nothing of this repository's product is loaded (see library_free_imports)."""
    if rank != 0:
        return
    _abi, scenes, pyoracle = library_free_imports()
    kind, sc, smp, sessions = reference_stereo(scenes, pyoracle)
    eyes = scenes.stereo_eyes(IPD)
    cores = os.cpu_count() or 1
    times, samples = [], 0
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        n = reference_frame(kind, sessions, sc, smp, eyes, cores, pyoracle, scenes)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
            samples += n
    total = sum(times)
    value = samples / total / 1e9
    ms = 1e3 * total / len(times)
    sample = ("the full stereo frame per step (2 x 1,296,000 samples, both eyes), traversal + intersect + shade + "
              "remap; scene and sample setup once before the steps; the reference's host code computes without "
              "contraction (its STRICT arithmetic)")
    line = {"metric": "vis+shade Gsamples/s", "impl": "reference", "value": value, "unit": "Gsamples/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "p50_frame_ms": 1e3 * statistics.median(times), "p99_frame_ms": 1e3 * float(np.percentile(times, 99)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural 995k-triangle scene, barrel-distorted sample set)",
            "config": stereo_config(args.gpus),
            "cpu_baseline": {"value": value, "unit": "Gsamples/s", "cores": cores, "kind": kind, "sample": sample,
                             "cpu_model": cpu_model()},
            "e2e": {"value": value, "unit": "Gsamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    for s in sessions or []:
        s.close()
    print(json.dumps(line), flush=True)


def cpu_baseline(scenes):
    """The reference's own path (oracle/_ref, else the oracle port) on this host: two full stereo
    frames on all cores, and one core over a 60-row band of both eyes."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    kind, sc, smp, sessions = reference_stereo(scenes, pyoracle)
    eyes = scenes.stereo_eyes(IPD)
    cores = os.cpu_count() or 1
    reference_frame(kind, sessions, sc, smp, eyes, cores, pyoracle, scenes)
    t0 = time.perf_counter()
    n = sum(reference_frame(kind, sessions, sc, smp, eyes, cores, pyoracle, scenes) for _ in range(2))
    dt = time.perf_counter() - t0
    rows1 = (570, 630)
    t1 = time.perf_counter()
    n1 = reference_frame(kind, sessions, sc, smp, eyes, 1, pyoracle, scenes, rows=rows1)
    dt1 = time.perf_counter() - t1
    for s in sessions or []:
        s.close()
    return {"value": n / dt / 1e9, "unit": "Gsamples/s", "cores": cores, "kind": kind,
            "sample": "2 full stereo frames (2 x 2,592,000 samples), traversal + intersect + shade + remap, %.1f s" % dt,
            "one_core": {"value": n1 / dt1 / 1e9, "unit": "Gsamples/s",
                         "sample": "%d samples (rows %d-%d of both eyes, sample setup included), %.1f s" %
                                   (n1, rows1[0], rows1[1], dt1)},
            "cpu_model": cpu_model()}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank)
        return
    if args.profile:
        if args.workload == "foveated":
            run_profile_case_foveated()
        else:
            run_profile_case()
        return
    if args.visit_clocks:
        run_visit_clocks()
        return
    if args.workload == "batched":
        run_batched(args)
        return
    if args.workload == "served":
        # a latency slot's launches must not share a hardware work queue with the throughput slots'
        # (8 queues by default); read by CUDA when the process first uses the device, which happens
        # in run_served
        os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
        run_served(args)
        return
    if args.workload == "foveated":
        run_foveated(args)
        return
    if args.workload == "c1":
        run_c1(args)
        return
    import numpy as np
    import torch
    import hvvr_b200 as hv
    from hvvr_b200 import scenes
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    sc = scenes.scene_c2()
    hv.generate_topology(sc)
    counts = frame_counts(hv, scenes, sc)

    rc, cams, images, smp, eyes = stereo_setup(hv, scenes, sc, True, torch)
    samples_per_frame = 2 * len(smp)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sp = ctypes_stream(stream)
    for _ in range(args.warmup):
        rc.render(stream=sp)
    torch.cuda.synchronize()
    rc.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = Clocks(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    for i in range(args.steps):
        flush.fill_(i & 0xff)
        starts[i].record(stream)
        rc.render(stream=sp)
        ends[i].record(stream)
        torch.cuda.synchronize()
    torch.cuda.synchronize()
    frame_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    # frame latency over a longer run of the same frames (p50/p99 over args.latency_frames), still
    # inside the clock sampling window
    lat_ms = frame_latencies(rc, sp, stream, flush, args.latency_frames)
    ck = clocks.stop()
    rc.synchronize()
    # the pipeline's span and the stages, from frames with per-launch events
    _, stage_ms = launch_times(rc, cams[0], lambda k: rc.render(stream=sp), flush)
    parts = rc.part_times()
    span = parts[2 * 3 + 1]  # rate class 3 (8x MSAA), the pipelined part
    # each kernel alone: one launch over all tiles of the frame, serial on one stream
    kernel_ms, _ = launch_times(rc, cams[0], lambda k: rc.render(stream=sp), flush, pipeline=0, heavy_divisor=0)
    total_ms = max_over_ranks(sum(frame_ms), dist, "cuda")
    ms_per_step = total_ms / args.steps
    value = replica_throughput(samples_per_frame, args.steps, total_ms * 1e-3, world)

    # end to end through the C ABI: CPU_MEMORY targets, images copied to host every frame
    rc.close()
    setup_ms = sample_setup_ms(hv, scenes)
    rc2, cams2, _, _, _ = stereo_setup(hv, scenes, sc, False, torch)
    for _ in range(max(2, args.warmup)):
        for c, xf in zip(cams2, eyes):
            c.set_camera_to_world(xf)
        rc2.render()
    e2e_steps = max(3, args.steps // 2)
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        for c, xf in zip(cams2, eyes):
            c.set_camera_to_world(xf)
        rc2.render()
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, "cuda")
    e2e_value = replica_throughput(samples_per_frame, e2e_steps, e2e_s, world)
    rc2.close()

    peak, peak_kind = load_peaks()
    cull_ms = statistics.mean(k[0] for k in kernel_ms)
    isect_ms = statistics.mean(k[1] for k in kernel_ms)
    kernels = {
        "tileCullKernel": {"algorithmic_bytes": cull_bytes(counts), "launch_ms": cull_ms},
        "intersectShadeKernel<8,FMA>": {"algorithmic_bytes": intersect_bytes(counts), "launch_ms": isect_ms},
    }
    for name, k in kernels.items():
        k["achieved_gbs"] = k["algorithmic_bytes"] / (k["launch_ms"] * 1e-3) / 1e9
        k["frac"] = k["achieved_gbs"] / peak
    dom = max(kernels, key=lambda n: kernels[n]["launch_ms"])
    fp32 = fp32_line(counts, MSAA, isect_ms, ck.get("sm_mhz") or 1965.0)
    line = {
        "metric": "vis+shade Gsamples/s", "value": value, "unit": "Gsamples/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "p50_frame_ms": float(np.percentile(lat_ms, 50)), "p99_frame_ms": float(np.percentile(lat_ms, 99)),
        "latency_frames": len(lat_ms),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded procedural 995k-triangle scene, barrel-distorted sample set)",
        "config": stereo_config(world),
        "e2e": {"value": e2e_value, "unit": "Gsamples/s", "h2d_bytes_per_step": 2 * 32,
                "d2h_bytes_per_step": 2 * W * H * 4},
        "roofline": {"bound": "hbm", "achieved": kernels[dom]["achieved_gbs"], "peak": peak, "unit": "GB/s",
                     "frac": kernels[dom]["frac"], "traffic": None, "kernel": dom,
                     "launch_ms": kernels[dom]["launch_ms"],
                     "timed": "each kernel alone: one launch over all 20,352 tiles of the stereo frame, serial on one "
                              "stream (pipeline off, no heavy split), per-launch CUDA events on that stream, mean of "
                              "5 frames after the timed ones",
                     "traffic_source": "null here: DRAM bytes per launch are in the committed ncu summaries under "
                                       "profiles/ (the BVH and the shared list triangles stay in L2, so DRAM traffic is "
                                       "far below the algorithmic bytes)",
                     "binding_bound": "neither kernel is HBM-bound: the tile cull is latency-bound (dependent node "
                                      "visits, see critical_path) and the intersect FP32-issue-bound (see fp32)",
                     "peak_source": peak_kind, "kernels": kernels, "counts": counts},
        "fp32": fp32,
        "critical_path": {"pipeline_span_ms": float(span[2] - span[0]) if span[0] >= 0 else None,
                          "longest_tile_node_visits": counts["longest_tile_node_visits"],
                          "note": "the frame ends when the longest tiles' dependent node visits and their shading "
                                  "end; span measured with per-launch events (which cost device time)"},
        "stage_ms_per_frame": {k: statistics.mean(s[i] for s in stage_ms) for i, k in
                               [(1, "block_cull"), (2, "first_tile_cull"), (3, "rest_of_cull_and_intersect_shade"),
                                (4, "remap"), (5, "total")]},
        # per frame: block cull, tile order, tile cull, pipelined intersect/shade, retry cull, retry-list
        # shade, remap per eye
        "gpu_launches": args.steps * 8,
        "sample_setup_ms": setup_ms,
        "clocks": ck,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(scenes)
        except Exception as e:  # reported, not fatal
            line["cpu_baseline"] = {"error": str(e)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def run_c1(args):
    """The small configuration: one 640x480 grid view (1xMSAA) of the 57,344-triangle scene,
    rendered into device memory; one step = one frame. Single GPU."""
    import numpy as np
    import torch
    import hvvr_b200 as hv
    from hvvr_b200 import scenes
    torch.cuda.set_device(0)
    sc = scenes.scene_c1()
    hv.generate_topology(sc)
    w, h = 640, 480
    rc = hv.Raycaster()
    rc.create_model(sc)
    for light in sc.lights:
        rc.create_light(light)
    img = torch.zeros((h, w), dtype=torch.int32, device="cuda")
    cam = rc.create_camera(scenes.viewport_for(w, h))
    cam.set_render_target(w, h, device_ptr=img.data_ptr())
    cam.set_samples(scenes.grid_samples(w, h))
    cam.set_camera_to_world(scenes.camera_transform())
    cam.set_msaa(1)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sp = ctypes_stream(stream)
    for _ in range(args.warmup):
        rc.render(stream=sp)
    torch.cuda.synchronize()
    clocks = Clocks(0)
    clocks.start()
    frame_ms = []
    for i in range(args.steps):
        flush.fill_(i & 0xff)
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        rc.render(stream=sp)
        s1.record(stream)
        torch.cuda.synchronize()
        frame_ms.append(s0.elapsed_time(s1))
    ck = clocks.stop()
    rc.close()
    ms = statistics.mean(frame_ms)
    print(json.dumps({
        "metric": "vis+shade Gsamples/s", "value": w * h / (ms * 1e-3) / 1e9, "unit": "Gsamples/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "p50_frame_ms": statistics.median(frame_ms),
        "p99_frame_ms": float(np.percentile(frame_ms, 99)), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural 57,344-triangle scene, grid samples)",
        "config": {"workload": "640x480 grid 1xMSAA, 57,344-triangle scene, one frame per step",
                   "l2": "flushed between frames (256 MiB write, untimed)"},
        "gpu_launches": args.steps * 9, "clocks": ck}))


def run_batched(args):
    """Batched form vs plain form on one GPU: the same views (uneven sizes and MSAA rates over 4
    resident scenes, 10% of each scene's vertices animated and refit every frame) rendered as one
    batch replayed from a CUDA graph, and one view per launch. Device-timed per frame (animation,
    refit, traversal, intersect/shade, remap; device images). Then one captured frame of each
    form checks that every view's hit IDs and depth are identical."""
    import hashlib
    import torch
    import hvvr_b200 as hv
    from hvvr_b200 import scenes, workloads
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    scs = workloads.make_scenes()
    views = workloads.make_views(args.views)
    setup_s = time.perf_counter() - t0
    rcs, anims = [], []
    for sc in scs:
        rc = hv.Raycaster()
        m = rc.create_model(sc)
        for l in sc.lights:
            rc.create_light(l)
        rcs.append(rc)
        anims.append(m)
    cams, images = [], []
    for v in views:
        cam = rcs[v.scene].create_camera(v.viewport)
        img = torch.zeros((v.height, v.width), dtype=torch.int32, device="cuda")
        cam.set_render_target(v.width, v.height, device_ptr=img.data_ptr())
        cam.set_samples(v.samples)
        cam.set_msaa(v.msaa)
        cam.set_camera_to_world(scenes.camera_transform(v.eye, v.target))
        cams.append(cam)
        images.append(img)
    for rc in rcs:  # scene upload and per-camera setup
        rc.render()
    animators = [workloads.Animator(torch, m, sc) for m, sc in zip(anims, scs)]
    samples_per_frame = sum(v.sample_count for v in views)
    subsamples_per_frame = sum(v.sample_count * v.msaa for v in views)
    batched = hv.Batch(cameras=cams, config=hv.batch_config(tri_index_capacity=768 << 20))
    tuned = batched.autotune(frames=3)
    plain = [hv.Batch(cameras=[c], config=hv.batch_config(tile_cull_warps=tuned.tile_cull_warps,
                                                          heavy_divisor=tuned.heavy_divisor,
                                                          tri_index_capacity=48 << 20)) for c in cams]
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sp = ctypes_stream(stream)

    def frame(form, t):
        for a in animators:
            a.step(t, sp)
        if form == "batched":
            batched.render(stream=sp)
        else:
            for b in plain:
                b.render(stream=sp)

    result = {}
    clocks = Clocks(0)
    for form in ("plain", "batched"):
        for i in range(args.warmup):
            frame(form, 0.1 * i)
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        if form == "batched":
            clocks.start()
        for i in range(args.steps):
            ev[i][0].record(stream)
            frame(form, 0.1 * (args.warmup + i))
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        if form == "batched":
            ck = clocks.stop()
        ms = [a.elapsed_time(b) for a, b in ev]
        result[form] = {"value": samples_per_frame * len(ms) / (sum(ms) * 1e-3) / 1e9, "ms_per_frame": sum(ms) / len(ms),
                        "p50_frame_ms": statistics.median(ms), "p99_frame_ms": float(np.percentile(ms, 99)),
                        "launches_per_frame": (3 + 8) if form == "batched" else 8 * len(views)}
    # identical hit IDs: one captured frame of each form at the same animation time
    digests = {}
    for form in ("plain", "batched"):
        for c in cams:
            c.set_capture(hv.HVVR_CAPTURE_HITS)
        frame(form, 123.0)
        torch.cuda.synchronize()
        dl = []
        for c in cams:
            ids, depth = c.hits()
            dl.append(hashlib.sha1(ids.tobytes() + depth.tobytes()).hexdigest())
        digests[form] = dl
        for c in cams:
            c.set_capture(0)
    match = sum(a == b for a, b in zip(digests["plain"], digests["batched"]))
    stats = batched.stats()
    line = {
        "metric": "vis+shade Gsamples/s, batched vs plain (one view per launch), same GPU",
        "value": result["batched"]["value"], "unit": "Gsamples/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": result["batched"]["ms_per_frame"],
        "p50_frame_ms": result["batched"]["p50_frame_ms"], "p99_frame_ms": result["batched"]["p99_frame_ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (4 seeded procedural scenes, grid/barrel/foveated sample sets)",
        "config": {"workload": "%d views over 4 resident scenes (100k/500k/1M/2M tris), sizes from {256x256, "
                               "640x480, 1080x1200 barrel, foveated 300k-1.2M}, MSAA {1,4,8,16}, 10%% of vertices "
                               "animated + GPU refit per frame" % len(views),
                   "samples_per_frame": samples_per_frame, "subsamples_per_frame": subsamples_per_frame,
                   "views": {k: sum(1 for v in views if v.kind == k) for k in workloads.KINDS},
                   "l2": "inputs larger than L2 (%d MB of beams per frame)" % (samples_per_frame * 48 >> 20),
                   "autotuned": {"tile_cull_warps": tuned.tile_cull_warps, "heavy_divisor": tuned.heavy_divisor,
                                 "tri_index_capacity": tuned.tri_index_capacity, "frame_ms": tuned.frame_ms}},
        "plain": result["plain"], "batched": result["batched"],
        "batched_over_plain": result["batched"]["value"] / result["plain"]["value"],
        "hit_id_match_views": "%d/%d" % (match, len(views)), "last_frame_stats": stats,
        "host_setup_s": setup_s, "clocks": ck,
    }
    print(json.dumps(line), flush=True)
    for b in plain:
        b.close()
    batched.close()
    for rc in rcs:
        rc.close()


BACKLOG = 64  # served: arrivals that find this many requests waiting are shed


def run_served(args):
    """Render server under open-loop Poisson arrivals. Six resident scenes (about 100k to 4M
    triangles); request mix: view templates per scene drawn from {256x256, 640x480,
    1080x1200 barrel, foveated 300k-1.2M} with MSAA {1,4,8,16}, plus 5% stereo requests (two
    1080x1200 barrel 8xMSAA eyes on the 1M scene, 64 mm IPD) submitted as the latency class.
    HBM budget 120 GiB. Arrivals that find BACKLOG requests already waiting are shed (counted).
    Latency = output ready - submit, on the server's clock (a stereo pair: both eyes), reported
    over all requests and per class. Then a sample of requests is rendered again by the plain
    path (a single-view batch) and compared image for image."""
    import torch
    import hvvr_b200 as hv
    from hvvr_b200 import scenes, workloads
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    tris = (100_000, 500_000, 1_000_000, 2_000_000, 3_000_000, 4_100_000)
    scs = workloads.make_scenes(tris, seed=20)
    rcs = []
    for sc in scs:
        rc = hv.Raycaster()
        rc.create_model(sc)
        for l in sc.lights:
            rc.create_light(l)
        rcs.append(rc)
    srv = hv.Server(rcs, hv.server_config(slots=args.throughput_slots, max_batch_views=args.max_batch_views,
                                          slot_list_capacity=512 << 20, hbm_budget_bytes=120 << 30,
                                          latency_slots=args.latency_slots, tile_cull_ctas_per_sm=args.served_cull_cap))
    rng = np.random.default_rng(5)
    tmpl = []  # (view id, width, height, samples, scene, spec)
    for si in range(len(scs)):
        for v in workloads.make_views(4, seed=100 + si, scene_count=1):
            vid = srv.add_view(si, v.viewport, v.samples, v.width, v.height)
            tmpl.append((vid, v.width, v.height, v.sample_count, si, v))
    stereo_smp = scenes.barrel_samples(W, H)
    stereo_vid = srv.add_view(2, scenes.viewport_for(W, H), stereo_smp, W, H)
    eyes = scenes.stereo_eyes(IPD)
    ring = {}

    def out_ptr(vid, w, h):
        r = ring.setdefault(vid, [torch.zeros((h, w), dtype=torch.int32, device="cuda") for _ in range(4)])
        r.append(r.pop(0))
        return r[0].data_ptr()

    # instances for the in-flight slots ahead of the traffic (a cold server allocates on admission)
    for vid, w, h, n, si, v in tmpl:
        srv.prewarm(vid, 8)
    srv.prewarm(stereo_vid, 16)
    # a warm server: every template and MSAA rate, and a stereo pair, rendered once before the sweep
    # (a first launch of each kernel variant and the slots' first streams cost milliseconds)
    warm = 0
    for vid, w, h, n, si, v in tmpl:
        for msaa in workloads.RATES:
            srv.submit(vid, int(msaa), scenes.camera_transform(), device_ptr=out_ptr(vid, w, h))
            warm += 1
    for _ in range(2):
        srv.submit_group([(stereo_vid, 8, xf, None, out_ptr(stereo_vid, W, H), 0) for xf in eyes], priority=1)
        warm += 2
    while warm:
        warm -= len(srv.poll(capacity=1024, wait_ms=50.0))
    setup_s = time.perf_counter() - t0

    def random_pose():
        ang = rng.uniform(0, 2 * np.pi)
        rad = rng.uniform(7.0, 13.0)
        return scenes.camera_transform((rad * np.sin(ang), rng.uniform(1.5, 5.0), rad * np.cos(ang)),
                                       (rng.uniform(-3, 3), 0.0, rng.uniform(-3, 3)))

    rates = [float(r) for r in args.rates.split(",")]
    sweep = []
    prev_stats = srv.stats()
    clocks = Clocks(0)
    clocks.start()
    for rate in rates:
        info = {}
        groups = {}  # request id -> group (stereo pairs share one)
        submitted_samples = {}
        shed = 0
        arrivals = 0
        start = time.perf_counter()
        next_t = start + rng.exponential(1.0 / rate)
        lat, qwait, service = [], [], []
        lat_class = {"stereo": [], "other": []}
        q_class = {"stereo": [], "other": []}
        s_class = {"stereo": [], "other": []}
        done_samples = 0
        group_done = {}
        end_arrivals = start + args.seconds
        pending = 0
        while True:
            now = time.perf_counter()
            while next_t <= now and next_t < end_arrivals:
                arrivals += 1
                if srv.stats()["queued"] >= BACKLOG:
                    shed += 1
                else:
                    if rng.uniform() < 0.05:
                        g = ("s", arrivals)
                        pair = [(stereo_vid, 8, xf, None, out_ptr(stereo_vid, W, H), 0) for xf in eyes]
                        for rid in srv.submit_group(pair, priority=1):
                            groups[rid] = g
                            submitted_samples[rid] = W * H
                        group_done[g] = [2, 0.0]
                        pending += 2
                    else:
                        vid, w, h, n, si, v = tmpl[int(rng.integers(len(tmpl)))]
                        msaa = int(workloads.RATES[int(rng.integers(4))])
                        rid = srv.submit(vid, msaa, random_pose(), device_ptr=out_ptr(vid, w, h))
                        groups[rid] = ("r", rid)
                        group_done[("r", rid)] = [1, 0.0]
                        submitted_samples[rid] = n
                        pending += 1
                next_t += rng.exponential(1.0 / rate)
            for c in srv.poll(capacity=1024, wait_ms=0.2):
                pending -= 1
                qwait.append(c.dispatch_ms - c.submit_ms)
                service.append(c.done_ms - c.dispatch_ms)
                g = groups.pop(c.id)
                cls = "stereo" if g[0] == "s" else "other"
                q_class[cls].append(c.dispatch_ms - c.submit_ms)
                s_class[cls].append(c.done_ms - c.dispatch_ms)
                done_samples += submitted_samples.pop(c.id)
                gd = group_done[g]
                gd[0] -= 1
                gd[1] = max(gd[1], c.done_ms - c.submit_ms)
                if gd[0] == 0:
                    lat.append(gd[1])
                    lat_class["stereo" if g[0] == "s" else "other"].append(gd[1])
                    del group_done[g]
            if now >= end_arrivals and pending == 0:
                break
        wall = time.perf_counter() - start
        st0 = prev_stats
        st = srv.stats()
        prev_stats = st
        nb = max(1, st["batches"] - st0["batches"])
        info = {"rate_req_s": rate, "arrivals": arrivals, "shed": shed, "completed_requests": len(lat),
                "throughput_gsamples_s": done_samples / wall / 1e9,
                "throughput_req_s": len(lat) / wall,
                "p50_latency_ms": float(np.percentile(lat, 50)) if lat else None,
                "p99_latency_ms": float(np.percentile(lat, 99)) if lat else None,
                "per_class": {k: {"requests": len(v), "p50_latency_ms": float(np.percentile(v, 50)) if v else None,
                                  "p99_latency_ms": float(np.percentile(v, 99)) if v else None,
                                  "max_latency_ms": float(max(v)) if v else None,
                                  # per eye / per request: host queue (submit -> dispatch) and service
                                  # (dispatch -> output ready)
                                  "p50_queue_ms": float(np.percentile(q_class[k], 50)) if q_class[k] else None,
                                  "p99_queue_ms": float(np.percentile(q_class[k], 99)) if q_class[k] else None,
                                  "p50_service_ms": float(np.percentile(s_class[k], 50)) if s_class[k] else None,
                                  "p99_service_ms": float(np.percentile(s_class[k], 99)) if s_class[k] else None}
                              for k, v in lat_class.items()},
                "p50_queue_ms": float(np.percentile(qwait, 50)) if qwait else None,
                "p50_service_ms": float(np.percentile(service, 50)) if service else None,
                "p99_service_ms": float(np.percentile(service, 99)) if service else None,
                "mean_batch_views": st["mean_batch_views"], "instances": st["instances"],
                "mean_batch_gpu_ms": (st["batch_gpu_ms"] - st0["batch_gpu_ms"]) / nb,
                "mean_dispatch_host_ms": (st["dispatch_host_ms"] - st0["dispatch_host_ms"]) / nb,
                "hbm_peak_gb": st["hbm_peak"] / 1e9, "wall_s": wall}
        sweep.append(info)
    ck = clocks.stop()
    # served vs plain: the same (template, msaa, pose) rendered by a single-view batch after the
    # server has released the scenes
    served = []
    for k in range(12):
        vid, w, h, n, si, v = tmpl[(k * 5) % len(tmpl)]
        msaa = int(workloads.RATES[k % 4])
        xf = random_pose()
        out = np.zeros((h, w), dtype=np.uint32)
        rid = srv.submit(vid, msaa, xf, output=out)
        while not any(c.id == rid for c in srv.poll(wait_ms=50.0)):
            pass
        served.append((si, v, msaa, xf, out))
    srv.close()
    matches = 0
    for si, v, msaa, xf, out in served:
        cam = rcs[si].create_camera(v.viewport)
        cam.set_render_target(v.width, v.height)
        cam.set_samples(v.samples)
        cam.set_msaa(msaa)
        cam.set_camera_to_world(xf)
        b = hv.Batch(cameras=[cam], config=hv.batch_config(use_graph=0, tri_index_capacity=64 << 20))
        b.render()
        matches += int(np.array_equal(cam.image, out))
        b.close()
        rcs[si].destroy_camera(cam)
    checks = len(served)
    best = max(sweep, key=lambda x: x["throughput_gsamples_s"])
    line = {
        "metric": "served vis+shade Gsamples/s under Poisson arrivals, p50/p99 request latency",
        "value": best["throughput_gsamples_s"], "unit": "Gsamples/s", "n_gpus": 1, "steps": len(rates),
        "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (6 seeded procedural scenes, grid/barrel/foveated sample sets)",
        "config": {"workload": "render server: 6 resident scenes (0.1M-4.1M tris), %d view templates + stereo "
                               "2x1080x1200 8xMSAA (5%% of requests, each pair submitted as one group), Poisson arrivals %s req/s for %.1f s each, "
                               "120 GiB HBM budget, %d throughput slots x %d views + %d latency slot(s) (stereo pairs as "
                               "the latency class; latency isolation: the throughput slots cull a tile per warp "
                               "without the cull -> shade pipeline; CUDA_DEVICE_MAX_CONNECTIONS=32), backlog limit %d, instances "
                               "pre-warmed" % (len(tmpl), args.rates, args.seconds, args.throughput_slots,
                                               args.max_batch_views, args.latency_slots, BACKLOG),
                   "l2": "inputs larger than L2"},
        "sweep": sweep, "served_vs_plain_image_match": "%d/%d" % (matches, checks),
        "host_setup_s": setup_s, "clocks": ck,
    }
    print(json.dumps(line), flush=True)
    for rc in rcs:
        rc.close()


# polar foveated stereo: the reference's polar sample set with its foveal MAR (1/60 degree) and a
# slope of 1/300 (MAR(e) = w0 (1 + e / 5 deg) past 0.5 degrees of tracking error, density
# ~ 1 / (1 + e / 5 deg)^2) out to 50 degrees of eccentricity: 1,173,612 samples per eye
FOV_PATTERN = (0.5, 50.0, 1.0 / 300.0, 1.0 / 60.0)
FOV_W, FOV_H, FOV_MSAA, FOV_FIELD = 1440, 1600, 16, 100.0


def saccade(frame):
    """Gaze of frame k of the 8-frame saccade: 10 degrees of azimuth, left to right."""
    a = math.radians(-5.0 + 10.0 * (frame % 8) / 7.0)
    return (math.sin(a), 0.0, -math.cos(a))


def foveated_setup(hv, scenes, sc, target_cuda, torch):
    from hvvr_b200 import _abi
    spec = hv.foveated_spec(*FOV_PATTERN, mode=_abi.HVVR_MODE_FOVEATED_POLAR)
    rc = hv.Raycaster(spec=spec, tri_index_capacity=256 << 20)
    rc.create_model(sc)
    for l in sc.lights:
        rc.create_light(l)
    smp = scenes.grid_samples(FOV_W, FOV_H)
    cams, images = [], []
    for xf in scenes.stereo_eyes(IPD):
        cam = rc.create_camera(scenes.viewport_fov(FOV_W, FOV_H, FOV_FIELD))
        if target_cuda:
            img = torch.zeros((FOV_H, FOV_W), dtype=torch.int32, device="cuda")
            cam.set_render_target(FOV_W, FOV_H, device_ptr=img.data_ptr())
            images.append(img)
        else:
            cam.set_render_target(FOV_W, FOV_H)
        cam.set_samples(smp)
        cam.set_camera_to_world(xf)
        cam.set_msaa(FOV_MSAA)
        cam.set_eye_dir(saccade(0))
        cams.append(cam)
    return rc, cams, images


def resolve_bytes(polar, pixels):
    """Compulsory HBM bytes of a frame's foveated resolve launches, per eye summed: per polar
    sample 4 B colour + 4 B depth + 8 B remap read and 8 B written to the polar textures; per
    polar texel the moments pass reads 4 B and writes 16 B, the polar -> screen pass reads 24 B
    (colour, depth, moments); per pixel the polar -> screen pass reads 4 B of history and writes
    4 B of result, each filter pass reads 4 B and writes 4 B, and the contrast enhancement reads
    8 B and writes 4 B of image."""
    texels = polar["samples_per_ring"] * polar["ring_count"]
    return polar["valid"] * 24 + texels * (4 + 16 + 24) + pixels * (4 + 4 + 8 + 8 + 8 + 4)


def run_foveated(args):
    """Polar foveated stereo on the 995k-triangle scene: both eyes in one batch, 16xMSAA, eye-space
    traversal with the per-frame gaze, the foveated resolve (temporal reprojection, eccentricity
    filters, contrast enhancement) to 1440x1600 per eye; the gaze cycles through an 8-frame
    10-degree saccade. One step = one stereo frame."""
    import numpy as np
    import torch
    import hvvr_b200 as hv
    from hvvr_b200 import scenes
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    sc = scenes.scene_c2()
    hv.generate_topology(sc)
    polar = hv.polar_foveated_samples(hv.foveated_spec(*FOV_PATTERN))
    # counts of one frame (both eyes) for the algorithmic bytes
    rc, cams, _ = foveated_setup(hv, scenes, sc, False, torch)
    for c in cams:
        c.set_capture(hv.HVVR_CAPTURE_HITS)
    rc.render()
    rc.render()
    ctr = rc.counters()
    counts = {"padded_samples": 0, "tiles": 0, "list_entries": 0, "unique_hits": 0, "node_visits": 0,
              "tested_entries": int(ctr[4]), "tested_warp_entries": int(ctr[5])}
    for cam in cams:
        blocks, tiles, padded, msaa = cam.layout()
        n, tri, mask = cam.gbuffer()
        counts["padded_samples"] += padded
        counts["tiles"] += tiles
        counts["list_entries"] += cam.list_total()
        counts["unique_hits"] += int(((tri != 0xFFFFFFFF) & (mask != 0)).sum())
        counts["node_visits"] += int(cam.tile_costs().astype(np.int64).sum())
    rc.close()

    rc, cams, images = foveated_setup(hv, scenes, sc, True, torch)
    samples_per_frame = 2 * polar["valid"]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sp = ctypes_stream(stream)
    frame = 0
    for _ in range(args.warmup):
        for c in cams:
            c.set_eye_dir(saccade(frame))
        rc.render(stream=sp)
        frame += 1
    torch.cuda.synchronize()
    rc.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = Clocks(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    for i in range(args.steps):
        flush.fill_(i & 0xff)
        for c in cams:
            c.set_eye_dir(saccade(frame))
        frame += 1
        starts[i].record(stream)
        rc.render(stream=sp)
        ends[i].record(stream)
        torch.cuda.synchronize()
    torch.cuda.synchronize()
    ck = clocks.stop()
    rc.synchronize()

    def fov_frame(k):
        for c in cams:
            c.set_eye_dir(saccade(frame + k))
        rc.render(stream=sp)
    _, stage_ms = launch_times(rc, cams[0], fov_frame, flush)
    # each kernel alone: one launch over all tiles, serial on one stream
    kernel_ms, _ = launch_times(rc, cams[0], fov_frame, flush, pipeline=0, heavy_divisor=0)
    frame_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = max_over_ranks(sum(frame_ms), dist, "cuda")
    value = replica_throughput(samples_per_frame, args.steps, total_ms * 1e-3, world)
    rc.close()

    # end to end through the C ABI: CPU_MEMORY targets, both resolved images copied to host
    rc2, cams2, _ = foveated_setup(hv, scenes, sc, False, torch)
    for k in range(max(3, args.warmup)):
        for c in cams2:
            c.set_eye_dir(saccade(k))
        rc2.render()
    e2e_steps = max(3, args.steps // 2)
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        for c in cams2:
            c.set_eye_dir(saccade(k))
        rc2.render()
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, "cuda")
    e2e_value = replica_throughput(samples_per_frame, e2e_steps, e2e_s, world)
    rc2.close()

    peak, peak_kind = load_peaks()
    resolve_ms = statistics.mean(s[4] for s in stage_ms)
    kernels = {
        "tileCullKernel": {"algorithmic_bytes": cull_bytes(counts),
                           "launch_ms_per_frame": statistics.mean(k[0] for k in kernel_ms)},
        "intersectShadeKernel<16,FMA>": {"algorithmic_bytes": intersect_bytes(counts),
                                         "launch_ms_per_frame": statistics.mean(k[1] for k in kernel_ms)},
        "foveated resolve (6 kernels per eye)": {"algorithmic_bytes": 2 * resolve_bytes(polar, FOV_W * FOV_H),
                                                 "launch_ms_per_frame": resolve_ms},
    }
    for name, k in kernels.items():
        k["achieved_gbs"] = k["algorithmic_bytes"] / (k["launch_ms_per_frame"] * 1e-3) / 1e9
        k["frac"] = k["achieved_gbs"] / peak
        k["traffic"] = None
    dom = max(kernels, key=lambda n: kernels[n]["launch_ms_per_frame"])
    line = {
        "metric": "vis+shade+resolve Gsamples/s", "value": value, "unit": "Gsamples/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "p50_frame_ms": statistics.median(frame_ms), "p99_frame_ms": float(np.percentile(frame_ms, 99)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded procedural 995k-triangle scene, polar foveated sample set)",
        "config": {"workload": "polar foveated stereo, %d samples per eye (pattern %s), 16xMSAA, resolved to "
                               "1440x1600 per eye over a 100-degree field, gaze in an 8-frame 10-degree saccade, "
                               "995,072-triangle scene; one frame (both eyes) per step" % (polar["valid"], FOV_PATTERN),
                   "samples_per_frame": samples_per_frame, "parallelism": "replicas x%d" % world,
                   "l2": "flushed between frames (256 MiB write, untimed)"},
        "e2e": {"value": e2e_value, "unit": "Gsamples/s", "h2d_bytes_per_step": 2 * 12,
                "d2h_bytes_per_step": 2 * FOV_W * FOV_H * 4},
        "roofline": {"bound": "hbm", "achieved": kernels[dom]["achieved_gbs"], "peak": peak, "unit": "GB/s",
                     "frac": kernels[dom]["frac"], "traffic": None, "kernel": dom,
                     "per_frame": "launches of one stereo frame; bytes and times summed over them",
                     "peak_source": peak_kind, "kernels": kernels, "counts": counts},
        "fp32": fp32_line(counts, FOV_MSAA, kernels["intersectShadeKernel<16,FMA>"]["launch_ms_per_frame"],
                          ck.get("sm_mhz") or 1965.0),
        "stage_ms_per_frame": {k: statistics.mean(s[i] for s in stage_ms) for i, k in
                               [(1, "block_cull"), (2, "first_tile_cull"), (3, "rest_of_cull_and_intersect_shade"),
                                (4, "resolve"), (5, "total")]},
        # per frame (ncu launch list): block cull, tile order, tile cull + retry pass + intersect
        # (2 parts), 6 resolve kernels per eye
        "gpu_launches": args.steps * 20,
        "clocks": ck,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def run_profile_case():
    """The benchmark's stereo frame (both eyes, one batch), 3 frames, 32M-entry list pool: the
    case the ncu launch list and captures run on (a few GB on the device)."""
    import hvvr_b200 as hv
    from hvvr_b200 import scenes
    sc = scenes.scene_c2()
    hv.generate_topology(sc)
    with hv.Raycaster(tri_index_capacity=32 << 20) as rc:
        rc.set_batch_config(timing=1)
        rc.create_model(sc)
        for l in sc.lights:
            rc.create_light(l)
        cams = []
        for xf in scenes.stereo_eyes(IPD):
            cam = rc.create_camera(scenes.viewport_for(W, H))
            cam.set_render_target(W, H)
            cam.set_samples(scenes.barrel_samples(W, H))
            cam.set_camera_to_world(xf)
            cam.set_msaa(MSAA)
            cams.append(cam)
        for _ in range(3):
            rc.render()
        rc.synchronize()
        print(json.dumps({"profile_case": "stereo 2x1080x1200 8xMSAA, 995k tris, frame 3",
                          "stage_ms": [float(x) for x in cams[0].timings()],
                          "kernel_ms": [float(x) for x in rc.kernel_times()],
                          "list_entries": sum(c.list_total() for c in cams)}))


VISIT_PHASES = ("row wait", "child test", "leaf refine + ranges", "multi-child insert", "next node", "list tail")
SHADE_PHASES = ("setup", "chunk: staged triangles, tile tests, compaction", "chunk: depth skip, subsample tests",
                "outputs, G-buffer, shading")


def run_visit_clocks():
    """The stereo frame rendered by the profiling build of the library, whose tile cull sums the SM
    cycles of each tile's node visits per phase (clock64 reads that wait for each phase's result)
    and whose intersect/shade sums its CTA's cycles per phase. Prints one JSON line: cycles per
    visit by phase for all tiles, for the slowest eighth (the heavy part) and for the 16 longest
    tiles, and the intersect/shade cycles per tile by phase for the same sets, each from the third
    frame after an L2 flush."""
    import ctypes as C
    lib_path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "hvvr_b200", "_lib", "visit_clocks",
                            "libhvvr_b200.so")
    if not os.path.exists(lib_path):
        sys.exit("bench.py --visit-clocks: build the profiling library first (make -C hvvr_b200/csrc visit-clocks)")
    os.environ["HVVR_B200_LIB"] = lib_path
    import torch
    import hvvr_b200 as hv
    from hvvr_b200 import scenes
    lib = hv.lib()
    lib.hvvr_dbg_visit_clocks.argtypes = [C.c_void_p, C.c_uint32]
    lib.hvvr_dbg_shade_clocks.argtypes = [C.c_void_p, C.c_uint32]
    sc = scenes.scene_c2()
    hv.generate_topology(sc)
    flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
    with hv.Raycaster(tri_index_capacity=128 << 20) as rc:
        rc.create_model(sc)
        for l in sc.lights:
            rc.create_light(l)
        cams = []
        for xf in scenes.stereo_eyes(IPD):
            cam = rc.create_camera(scenes.viewport_for(W, H))
            cam.set_render_target(W, H)
            cam.set_samples(scenes.barrel_samples(W, H))
            cam.set_camera_to_world(xf)
            cam.set_msaa(MSAA)
            cams.append(cam)
        for _ in range(3):
            flush.fill_(1.0)
            rc.render()
        rc.synchronize()
        tiles = sum(len(c.tile_lists()[0]) for c in cams)
        raw = np.zeros((tiles, len(VISIT_PHASES) + 1), np.uint64)
        assert lib.hvvr_dbg_visit_clocks(raw.ctypes.data, tiles) == 0
        sraw = np.zeros((tiles, len(SHADE_PHASES) + 2), np.uint64)
        assert lib.hvvr_dbg_shade_clocks(sraw.ctypes.data, tiles) == 0
    cyc, visits = raw[:, :-1].astype(np.float64), raw[:, -1].astype(np.int64)
    scyc, entries = sraw[:, :len(SHADE_PHASES)].astype(np.float64), sraw[:, -1].astype(np.int64)

    def table(sel):
        v = max(int(visits[sel].sum()), 1)
        per = cyc[sel].sum(axis=0) / v
        return {"tiles": int(sel.sum()), "visits": int(visits[sel].sum()),
                "cycles_per_visit": round(float(per.sum()), 1),
                "phases": {name: {"cycles_per_visit": round(float(x), 1), "share": round(float(x / per.sum()), 3)}
                           for name, x in zip(VISIT_PHASES, per)}}

    def shade_table(sel):
        sel = sel & (entries > 0)
        n = max(int(sel.sum()), 1)
        per = scyc[sel].sum(axis=0) / n
        return {"tiles": int(sel.sum()), "list_entries_per_tile": round(float(entries[sel].sum()) / n, 1),
                "cycles_per_tile": round(float(per.sum()), 1),
                "phases": {name: {"cycles_per_tile": round(float(x), 1), "share": round(float(x / per.sum()), 3)}
                           for name, x in zip(SHADE_PHASES, per)}}

    order = np.argsort(-visits)
    heavy = np.zeros(tiles, bool)
    heavy[order[: max(1, tiles // 8)]] = True
    top = np.zeros(tiles, bool)
    top[order[:16]] = True
    stop = np.zeros(tiles, bool)
    stop[np.argsort(-scyc.sum(axis=1))[:16]] = True
    print(json.dumps({"visit_clocks": "tile cull, stereo 2x1080x1200 8xMSAA, 995,072 triangles, frame 3 after an L2 "
                                      "flush, profiling build (counters add registers and spills)",
                      "all": table(visits > 0), "slowest_eighth": table(heavy), "longest_16": table(top),
                      "longest_tile_visits": int(visits.max()),
                      "shade_clocks": {"all": shade_table(np.ones(tiles, bool)), "slowest_eighth": shade_table(heavy),
                                       "longest_16_shades": shade_table(stop),
                                       "longest_shade_cycles": round(float(scyc.sum(axis=1).max()), 1)}}))


def run_profile_case_foveated():
    """The foveated benchmark frame (both eyes, resolve to 1440x1600 each), 3 frames of the
    saccade, 64M-entry list pool: the case the foveated launch list and captures run on."""
    import torch
    import hvvr_b200 as hv
    from hvvr_b200 import scenes
    sc = scenes.scene_c2()
    hv.generate_topology(sc)
    rc, cams, _ = foveated_setup(hv, scenes, sc, False, torch)
    rc.set_batch_config(timing=1)
    for k in range(3):
        for c in cams:
            c.set_eye_dir(saccade(k))
        rc.render()
    rc.synchronize()
    print(json.dumps({"profile_case": "polar foveated stereo 16xMSAA, resolve 2x1440x1600, 995k tris, frame 3",
                      "stage_ms": [float(x) for x in cams[0].timings()],
                      "kernel_ms": [float(x) for x in rc.kernel_times()],
                      "list_entries": sum(c.list_total() for c in cams)}))
    rc.close()


def launch_times(rc, cam, render, flush, frames=5, **cfg):
    """Per-launch device times of the workload's frames: the timed frames run without per-launch
    events (they cost device time), so these come from `frames` more frames of the same workload
    rendered right after them with config.timing = 1 and the given config changes (L2 flushed
    before each, as in the timed loop; one untimed frame first when the config changes). Returns
    ([cull, intersect, block cull, remap/resolve] ms, camera stage ms) per frame."""
    import torch
    saved = rc.batch_config()
    rc.set_batch_config(timing=1, **cfg)
    if cfg:
        render(0)
        torch.cuda.synchronize()
    kernel_ms, stage_ms = [], []
    for k in range(frames):
        flush.fill_(k & 0xff)
        render(k)
        torch.cuda.synchronize()
        kernel_ms.append([float(x) for x in rc.kernel_times()])
        stage_ms.append([float(x) for x in cam.timings()])
    rc.set_batch_config(saved)
    return kernel_ms, stage_ms


def frame_latencies(rc, sp, stream, flush, frames):
    """Device times of `frames` consecutive frames (L2 flushed before each, untimed), in ms."""
    import torch
    if frames <= 0:
        return []
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(frames)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(frames)]
    for i in range(frames):
        flush.fill_(i & 0xff)
        starts[i].record(stream)
        rc.render(stream=sp)
        ends[i].record(stream)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in zip(starts, ends)]


def ctypes_stream(stream):
    import ctypes
    return ctypes.c_void_p(stream.cuda_stream)


if __name__ == "__main__":
    main()
