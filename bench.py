"""Benchmark of the structured-volume path (one JSON line on rank 0).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--config 2|1|3]

Step = one frame: bnAccumReset + bnRender (pathsPerPixel waves of ray
generation, macrocell DDA, Woodcock tracking, shading, shadow rays,
accumulation) + resolve, through the bn* C ABI of libbarney_b200.so.

Default workload (the large single-GPU case): 512^3 float32 6-octave value
noise (seed 0), 8^3-voxel macrocells, 256-entry knot transfer function
(seed 1, density 50), 1920x1080, 64 spp, isotropic HG single scatter with
albedo 0.8, one directional light + ambient 0.25.  Seeded synthetic inputs
stand in for user data.  value = volume samples per second (whole job);
frames/s and rays/s are reported beside it.

Multi-GPU (torchrun): every rank renders its own frame of the same workload
(replicas, weak scaling; the path needs no exchange), timed on the device
with CUDA events and reduced by MAX over ranks.

--impl reference: the CPU oracle (a restatement of the reference's own
CPU/embree-backend algorithm; the reference itself cannot be built here) on
all host cores, each step a bounded crop of the same frame.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Msamples/s & frames/s, p99 latency: served/FP16 vs plain FP32 at equal RMSE"
FALLBACK_HBM_GBS = 6650.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--config", default="2", choices=["1", "2", "3", "4", "5"])
    p.add_argument("--requests", type=int, default=None, help="config 5: requests per arrival rate")
    p.add_argument("--rates", default="50,200,500,1000,2000", help="config 5: arrival rates (req/s)")
    p.add_argument("--dtype", default=None, help="storage type for config 3 (f32, f16, u8, bf16)")
    p.add_argument("--spp", type=int, default=None)
    p.add_argument("--phase", default="hg", choices=["hg", "simple"],
                   help="configs 2/3: hg = the multi-scatter build's HGPhase (albedo 0.8); "
                        "simple = Barney's default build, SimplePhase (0.7 x TF colour)")
    p.add_argument("--max-volume-bounces", type=int, default=0,
                   help="configs 2/3: multi-scatter build with up to this many volume bounces")
    p.add_argument("--iso", type=float, default=None,
                   help="configs 2/3: add an iso_surface at this value (matte, colour .8) on the volume's field")
    p.add_argument("--e2e-steps", type=int, default=None)
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-serving", action="store_true",
                   help="skip the served-vs-plain measurement that the default run adds")
    p.add_argument("--tile-dp", action="store_true",
                   help="configs 1-3 on N GPUs: split each frame's pixel tiles across the ranks and gather "
                        "the frame over NCCL every step (strong scaling) instead of one frame per rank")
    p.add_argument("--kernel", default="per-lane", choices=["per-lane", "regrouped"],
                   help="render kernel of plain jobs: one pixel per lane (default) or regrouped pixel slots")
    p.add_argument("--rmse", action="store_true", help="image RMSE of every storage form vs the FP64 oracle")
    p.add_argument("--rmse-size", default="96x54", help="image size of the RMSE frames")
    p.add_argument("--rmse-spp", type=int, default=4096)
    return p.parse_args()


def workload(args, xp, device):
    """Scene dict + JSON description of the benchmarked configuration."""
    from barney_b200 import synth
    if args.config == "1":
        d = synth.config1(reference_semantics=True, spp=args.spp or 16)
        if xp is not None and xp.__name__ == "torch":
            import torch
            d["voxels"] = torch.from_numpy(d["voxels"]).to(device)
        desc = {"workload": "64^3 f32 Gaussian blobs (seed 0), 256x256, 16 spp, 128-entry linear TF, density 50, "
                            "ambient 1, default-build single scatter",
                "volume": "64^3 f32", "image": [256, 256], "spp": d["spp"]}
        return d, desc
    n = 512 if args.config == "2" else 1024
    dtype = args.dtype or "f32"
    vol = synth.to_storage(synth.value_noise(n, 0, xp=xp, device=device), dtype)
    d = synth.config2(vol=vol, dtype=dtype, spp=args.spp or (64 if args.config == "2" else 256))
    scatter = "HG single scatter"
    if args.phase == "simple":
        d["phase"] = "simple"
        scatter = "SimplePhase single scatter (default build)"
    if args.max_volume_bounces > 0:
        d["max_volume_bounces"] = args.max_volume_bounces
        scatter = f"HG multi-scatter (up to {args.max_volume_bounces} volume bounces)"
    if args.iso is not None:
        d["iso"] = {"value": args.iso}
        scatter += f", matte isosurface at {args.iso:g} (one diffuse bounce)"
    desc = {"workload": f"{n}^3 {dtype} 6-octave value noise (seed 0), 8^3 macrocells, 1920x1080, {d['spp']} spp, "
                        f"256-entry knot TF (seed 1) density 50, {scatter}"
                        f"{'' if args.phase == 'simple' else ' albedo 0.8'}, "
                        "dir light + ambient 0.25",
            "volume": f"{n}^3 {dtype}", "image": [1920, 1080], "spp": d["spp"]}
    return d, desc


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_uuid):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if gpu_uuid:
            cmd += ["-i", gpu_uuid]
        try:
            self.p = subprocess.Popen(cmd, stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [l.split(",") for l in open(self.f.name).read().splitlines() if l.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[0]))
                mx = float(r[1])
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, r[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic(key):
    """DRAM bytes per render launch from the committed ncu summary (or None)."""
    path = os.path.join(ROOT, "profiles", "render_traffic.json")
    try:
        with open(path) as f:
            v = json.load(f).get(key)
        return float(v) if v is not None else None
    except Exception:
        return None


def cpu_baseline(desc_scene, seconds):
    """Time the CPU oracle on a centred crop of the frame, all host cores."""
    import numpy as np
    import oracle
    sc = oracle.Scene(desc_scene)
    W, H = desc_scene["width"], desc_scene["height"]
    threads = os.cpu_count() or 1
    # calibrate on a small crop, then size the sample to ~`seconds`
    cw = ch = 32
    spp = 1
    while True:
        x0, y0 = (W - cw) // 2, (H - ch) // 2
        _, secs, st = oracle.render(sc, 1, spp, accum=np.zeros((H, W, 4), np.float32),
                                    rect=(x0, y0, x0 + cw, y0 + ch), threads=threads)
        if secs > seconds / 4 or (cw >= W and ch >= H and spp >= desc_scene.get("spp", 1)):
            break
        grow = max(1.5, min(4.0, (seconds / max(secs, 1e-3)) ** 0.5))
        if spp < desc_scene.get("spp", 1) and cw * ch >= 128 * 128:
            spp = min(desc_scene.get("spp", 1), int(spp * grow * grow) + 1)
        else:
            cw, ch = min(W, int(cw * grow)), min(H, int(ch * grow))
    # a whole frame that is shorter than the sample: render it again until the
    # sample lasts about seconds/4
    reps, samples = 1, st["samples"]
    while secs < seconds / 4 and reps < 10000:
        _, s2, st2 = oracle.render(sc, 1, spp, accum=np.zeros((H, W, 4), np.float32),
                                   rect=(x0, y0, x0 + cw, y0 + ch), threads=threads)
        secs += s2
        samples += st2["samples"]
        reps += 1
    rep = f" x {reps} renders" if reps > 1 else ""
    return {"value": samples / secs / 1e6, "unit": "Msamples/s", "cores": threads, "kind": "port",
            "sample": f"{cw}x{ch} centred crop x {spp} waves of the frame{rep} ({samples} volume samples, "
                      f"{secs:.1f} s)", "seconds": secs}


def run_reference(args):
    """CPU oracle arm: rank 0 only, all host cores, bounded crop per step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    try:
        import torch
        xp, dev = torch, "cpu"
    except Exception:
        import numpy as np
        xp, dev = np, None
    d, desc = workload(args, xp, dev)
    if hasattr(d["voxels"], "numpy"):
        d["voxels"] = d["voxels"].numpy()
    per_step = max(2.0, min(20.0, 120.0 / max(1, args.steps + args.warmup)))
    vals = []
    base = None
    for i in range(args.warmup + args.steps):
        b = cpu_baseline(d, per_step)
        if i >= args.warmup:
            vals.append(b["value"])
            base = b
    value = statistics.mean(vals)
    frame_samples = None
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Msamples/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": base["seconds"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)", "config": desc,
            "cpu_baseline": {"value": value, "unit": "Msamples/s", "cores": base["cores"], "kind": "port",
                             "sample": base["sample"]},
            "e2e": {"value": value, "unit": "Msamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference not buildable here (empty owl/cuBQL/embree/optix submodules, no ANARI SDK); "
                    "CPU restatement of its CPU-backend algorithm timed instead"}
    del frame_samples
    print(json.dumps(line), flush=True)
    return 0


def l2_flush_buffer(d, torch):
    """A 256 MB device buffer to overwrite between timed steps when the
    volume fits in the B200's 126 MB L2 (config 1), else None."""
    vox = d["voxels"]
    nbytes = vox.numel() * vox.element_size() if hasattr(vox, "numel") else vox.nbytes
    if nbytes > 2 * 126 * 2 ** 20:
        return None
    return torch.zeros(64 * 2 ** 20, dtype=torch.float32, device="cuda")


def gather_partitions(frame, owners):
    """Pixel-tile data parallelism: every rank's frame (only its own tiles
    rendered) is all-gathered and the owned pixels are merged into the full
    frame on every rank (TiledFB.cu:230-261 deals tiles the same way)."""
    import torch.distributed as dist
    import barney_b200 as bn
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return frame
    import torch
    frames = [torch.empty_like(frame) for _ in range(dist.get_world_size())]
    dist.all_gather(frames, frame)
    return bn.merge_partitions(frames, owners)


def reduce_over_ranks(ms, samples, rays, device=None):
    """Whole-job figures of a replicated run: the slowest rank's device time
    (MAX) and the work of all ranks (SUM).  Every rank calls this, in the same
    order, with its own figures; single-process runs return them unchanged."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms, float(samples), float(rays)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        tmax = t[:1].clone()
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
        tsum = t[1:].clone()
        dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
        t = torch.cat([tmax, tsum])
    return float(t[0]), float(t[1]), float(t[2])


def run_ours(args):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    import barney_b200 as bn

    d, desc = workload(args, torch, "cuda")
    r = bn.VolumeRenderer(d, color_format="rgba8", gpu=local)
    r.set_regrouping(args.kernel == "regrouped")
    stream = torch.cuda.current_stream()
    r.L.bnxSetStream(r.ctx, stream.cuda_stream)
    bn.check()
    tile_dp = args.tile_dp and world > 1
    if tile_dp:  # this rank renders its tiles; the frame is gathered every step
        r.set_partition(rank, world)
        owners = torch.from_numpy(bn.partition_owners(d["width"], d["height"], world)).cuda()
        device_frame = torch.empty((d["height"], d["width"]), dtype=torch.int32, device="cuda")

    def frame():
        r.accum_reset()
        r.render()
        st = r.stats()
        if tile_dp:
            r.read(device_frame)
            gather_partitions(device_frame, owners)
        return st

    for _ in range(args.warmup):
        frame()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(local).uuid)
        uuid = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
    except Exception:
        pass
    sampler = ClockSampler(uuid) if rank == 0 else None
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    flush = l2_flush_buffer(d, torch)
    if flush is None:  # inputs larger than L2: time the steps back to back
        e0.record(stream)
        for _ in range(args.steps):
            stats.append(frame())
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
    else:  # inputs inside L2: flush it before every step, outside the timed region
        ms = 0.0
        for _ in range(args.steps):
            flush.add_(1)
            e0.record(stream)
            stats.append(frame())
            e1.record(stream)
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
    torch.cuda.synchronize()
    if world > 1:  # the timed region is bracketed by a barrier on both sides
        dist.barrier()
    clocks = sampler.stop() if sampler else None
    samples = sum(s["samples"] for s in stats)
    rays = sum(s["rays"] for s in stats)
    ms_max, samples_all, rays_all = reduce_over_ranks(ms, samples, rays, device="cuda")
    secs = ms_max / 1e3

    # roofline of the render kernel: algorithmic bytes per launch / its mean duration
    es = {"f32": 4, "f16": 2, "bf16": 2, "u8": 1}[d["dtype"]]
    alg = [8 * es * s["samples"] + 4 * s["mc_visits"] + 16 * s["pixel_samples"] for s in stats]
    kms = [s["render_ms"] for s in stats]
    achieved = statistics.mean(a / (k * 1e-3) for a, k in zip(alg, kms)) / 1e9
    peak, peak_kind = measured_peak()
    # the committed capture applies to the same workload only: same config,
    # storage, spp, phase, bounces and isosurface
    tkey = f"config{args.config}_{d['dtype']}_spp{d['spp']}"
    tkey += ("_simple" if d.get("phase") == "simple" else "") + \
        (f"_msc{d['max_volume_bounces']}" if d.get("max_volume_bounces") else "") + \
        (f"_iso{d['iso']['value']:g}" if d.get("iso") else "")
    traffic = profiled_traffic(tkey)

    # end to end through the C ABI with host buffers: per step the camera is
    # set from host memory (kernel parameters) and the rgba8 frame is read
    # into pinned host memory
    e2e_steps = args.e2e_steps or max(1, args.steps)
    host = torch.empty((d["height"], d["width"]), dtype=torch.int32, pin_memory=True)
    cam = d["camera"]
    e2e_samples = 0
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0.record(stream)
    for _ in range(e2e_steps):
        r.set_camera(cam)
        r.accum_reset()
        r.render()
        if tile_dp:  # the frame is assembled on the devices, then read to host memory
            r.read(device_frame)
            host.copy_(gather_partitions(device_frame, owners), non_blocking=True)
        else:
            r.read(host)
        e2e_samples += r.stats()["samples"]
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    e2e_ms_max, e2e_samples_all, _ = reduce_over_ranks(e2e_ms, e2e_samples, 0, device="cuda")
    e2e_value = e2e_samples_all / (e2e_ms_max / 1e3) / 1e6
    h2d = 3 * 3 * 4 + 4 + 8  # position, direction, up, fovy, accumID/spp words
    d2h = d["width"] * d["height"] * 4

    # the fast-math form (bnx.fastMath: FMA contraction, approximate division;
    # within 2 ulp per sample and 3 standard errors per pixel of the exact
    # path) on the same workload, timed the same way
    fast = None
    plain_kernels = not d.get("max_volume_bounces") and not d.get("iso")
    if plain_kernels and not tile_dp:
        r.L.bnSet1i(r.renderer, b"bnx.fastMath", 1)
        r.L.bnCommit(r.renderer)
        bn.check()
        for _ in range(args.warmup):
            frame()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        fstats, fms = [], 0.0
        if flush is None:
            e0.record(stream)
            for _ in range(args.steps):
                fstats.append(frame())
            e1.record(stream)
            torch.cuda.synchronize()
            fms = e0.elapsed_time(e1)
        else:
            for _ in range(args.steps):
                flush.add_(1)
                e0.record(stream)
                fstats.append(frame())
                e1.record(stream)
                torch.cuda.synchronize()
                fms += e0.elapsed_time(e1)
        if world > 1:
            dist.barrier()
        fms_max, fsamples_all, _ = reduce_over_ranks(fms, sum(s["samples"] for s in fstats), 0, device="cuda")
        falg = [8 * es * s["samples"] + 4 * s["mc_visits"] + 16 * s["pixel_samples"] for s in fstats]
        fkms = [s["render_ms"] for s in fstats]
        fach = statistics.mean(a / (k * 1e-3) for a, k in zip(falg, fkms)) / 1e9
        fast = {"value": fsamples_all / (fms_max / 1e3) / 1e6, "unit": "Msamples/s",
                "ms_per_step": fms_max / args.steps, "frames_per_s": world * args.steps / (fms_max / 1e3),
                "kernel_ms": statistics.mean(fkms), "roofline_frac": fach / peak,
                "form": "bnx.fastMath: FMA contraction, approximate division and square root outside the "
                        "texel and TF coordinates"}
        r.L.bnSet1i(r.renderer, b"bnx.fastMath", 0)
        r.L.bnCommit(r.renderer)

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        dh = dict(d)
        dh["voxels"] = d["voxels"].cpu().numpy()
        cpu = cpu_baseline(dh, args.cpu_seconds)
        cpu.pop("seconds", None)
    r.close()

    serving = None
    if world == 1 and args.config == "2" and not args.no_serving and d["spp"] == 64 and d["dtype"] == "f32" \
            and not d.get("max_volume_bounces") and not d.get("iso") and d.get("phase") != "simple":
        torch.cuda.empty_cache()
        # served f16 vs plain f32 on one request stream, bounded for the
        # default run (--config 5 runs it at 10 000 requests per rate)
        serving = serving_arms(n_sat=400, rates=[200.0, 1000.0], n_rate=400)
        serving["reduced"] = "400 requests at saturation and per rate (the full sweep: bench.py --config 5)"

    if rank == 0:
        n_frames = (1 if tile_dp else world) * args.steps
        line = {
            "metric": METRIC, "value": samples_all / secs / 1e6, "unit": "Msamples/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "strong" if tile_dp else "weak", "vs_baseline": None,
            "dtype": d["dtype"],
            "data": "synthetic (seeded value noise / Gaussian blobs generated on device)",
            "config": dict(desc, kernel=args.kernel,
                           parallelism=(f"pixel tiles x{world}, NCCL all-gather per frame" if tile_dp
                                              else f"replicas x{world}" if world > 1 else "single GPU"),
                           l2="inputs larger than L2" if flush is None
                           else "L2 flushed before every timed step (256 MB write, untimed)"),
            "frames_per_s": n_frames / secs, "rays_per_s": rays_all / secs,
            "gpu_launches": 2 * args.steps,
            "clocks": clocks,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": traffic,
                         "algorithmic_bytes_per_launch": statistics.mean(alg),
                         "kernel_ms": statistics.mean(kms)},
            "e2e": {"value": e2e_value, "unit": "Msamples/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "frames_per_s": (1 if tile_dp else world) * e2e_steps / (e2e_ms_max / 1e3)},
            "cpu_baseline": cpu,
        }
        if fast is not None:
            line["fast_math"] = fast
            line["gpu_launches"] += 2 * args.steps
        if serving is not None:
            line["serving"] = serving
            line["served_over_plain"] = serving["served_over_plain"]
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_batch(args):
    """Config 4: 64 mixed jobs rendered as one persistent launch per frame
    (bnxRenderBatch, CUDA graph replay, launch shape and scheduling from the
    autotuner), against the same jobs rendered one bnRender at a time."""
    import torch
    import barney_b200 as bn
    from barney_b200 import synth
    torch.cuda.set_device(0)
    jobs = synth.config4_jobs(64, xp=torch, device="cuda")
    ctx = bn.Context(stream=torch.cuda.current_stream().cuda_stream)
    rs = [bn.VolumeRenderer(j, context=ctx, color_format="rgba8") for j in jobs]
    for r, j in zip(rs, jobs):
        r.set_spp(j["spp"])
    tuned = ctx.autotune_batch(rs)

    def frame():
        for r in rs:
            r.accum_reset()
        ctx.render_batch(rs)
        return ctx.stats()

    for _ in range(args.warmup):
        frame()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    st = [frame() for _ in range(args.steps)]
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    samples = sum(x["samples"] for x in st)
    # the same 64 jobs, one bnRender each (still the v2 megakernel per job)
    e0.record(stream)
    seq_samples = 0
    for r in rs:
        r.accum_reset()
        r.render()
        seq_samples += r.stats()["samples"]
    e1.record(stream)
    torch.cuda.synchronize()
    seq_ms = e0.elapsed_time(e1)
    line = {"metric": METRIC, "value": samples / (ms / 1e3) / 1e6, "unit": "Msamples/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "mixed u8/f16/f32",
            "data": "synthetic (64 seeded jobs)",
            "config": {"workload": "64 jobs: edge log-U[32,256] blobs/noise, u8/f16/f32, side log-U[128,1024], "
                                   "spp {1,4,16,32}, orbit cameras; one persistent batch launch per frame",
                       "autotuned": tuned},
            "frames_per_s": 64 * args.steps / (ms / 1e3),
            "sequential_bnRender": {"frames_per_s": 64 / (seq_ms / 1e3),
                                    "Msamples_per_s": seq_samples / (seq_ms / 1e3) / 1e6},
            "gpu_launches": 2 * args.steps}
    print(json.dumps(line), flush=True)
    for r in rs:
        r.close()
    ctx.close()
    return 0


def serving_volumes(xp, device):
    """16 resident float32 volumes, seeds 100-115: edge log-U[128, 1024] and
    the field (Gaussian blobs or value noise) drawn per seed."""
    import math
    import numpy as np
    from barney_b200 import synth
    out = []
    for seed in range(100, 116):
        rng = np.random.default_rng(seed)
        edge = int(round(math.exp(rng.uniform(math.log(128), math.log(1024)))))
        field = "blobs" if rng.integers(2) == 0 else "noise"
        f = synth.blobs(edge, seed, xp=xp, device=device) if field == "blobs" else \
            synth.value_noise(edge, seed, xp=xp, device=device)
        if field == "blobs":
            d = synth.scene(f, "f32", 256, 256, synth.tf_linear_ramp(128), 50.0, synth.DEFAULT_CAMERA, ambient=1.0)
        else:
            d = synth.config2(vol=f, dtype="f32", width=256, height=256)
        d["seed"], d["edge"], d["field"] = seed, edge, field
        out.append(d)
    return out


def request_stream(n, seed=7):
    """n requests: a volume of the 16, side {256, 512, 1024}, spp {1, 4, 16},
    a camera on an orbit about the volume."""
    import numpy as np
    from barney_b200 import synth
    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(n):
        v = int(rng.integers(16))
        side = [256, 512, 1024][int(rng.integers(3))]
        spp = [1, 4, 16][int(rng.integers(3))]
        reqs.append((v, side, spp, synth.orbit_camera(rng)))
    return reqs


def poisson_arrivals(n, rate, seed):
    import numpy as np
    return np.cumsum(np.random.default_rng(seed).exponential(1.0 / rate, n))


def percentile(xs, q):
    xs = sorted(xs)
    return xs[min(len(xs) - 1, int(q * (len(xs) - 1) + 0.5))] if xs else None


def serving_arms(n_sat, rates, n_rate, fast_math=True):
    """Both forms of the serving workload on ONE request stream (seed 7):

    served  f16 storage (majorants from the stored values, rounded up),
            compensated accumulation (and the fast-math kernels if fast_math),
            continuous batching by the render server under a 150 GB budget;
    plain   the float32 volumes, exact kernels, one bnRender + read-back per
            request, back to back.

    Throughput: the first n_sat requests submitted at once (served) and
    rendered back to back (plain).  Latency at each rate: the first n_rate
    requests arriving as a Poisson process; the served arm is measured live,
    the plain arm's latencies follow from its measured per-request service
    times by the FIFO queue recursion (one request at a time, in arrival
    order)."""
    import numpy as np
    import torch
    import barney_b200 as bn
    from barney_b200 import synth
    torch.cuda.set_device(0)
    n_all = max(n_sat, n_rate)
    reqs = request_stream(n_all, seed=7)
    vols = serving_volumes(torch, "cuda")
    # plain arm first: float32 volumes, one frame buffer per (volume, size)
    ctx2 = bn.Context()
    plain = [bn.VolumeRenderer(d, context=ctx2, color_format="rgba8") for d in vols]
    L = bn.lib()
    fbs = {}
    for i in range(len(plain)):
        for side in (256, 512, 1024):
            fb = L.bnFrameBufferCreate(ctx2.ctx, 0)
            L.bnFrameBufferResize(fb, bn.BN_UFIXED8_RGBA, side, side, bn.BN_FB_COLOR)
            fbs[i, side] = fb
    bn.check()
    host = np.zeros((1024 * 1024,), np.uint32)

    def plain_one(v, side, spp, cam):
        r = plain[v]
        r.set_camera(cam)
        r.set_spp(spp)
        fb = fbs[v, side]
        L.bnAccumReset(fb)
        L.bnRender(r.renderer, r.model, r.camera, fb)
        L.bnFrameBufferRead(fb, bn.BN_FB_COLOR, host.ctypes.data, bn.BN_UFIXED8_RGBA)
        return r.stats()["samples"]

    for q in reqs[:16]:  # warm-up: load the kernels
        plain_one(*q)
    torch.cuda.synchronize()
    service, plain_samples = [], 0
    t0 = time.perf_counter()
    for q in reqs:
        ts = time.perf_counter()
        smp = plain_one(*q)
        service.append(time.perf_counter() - ts)
        if len(service) <= n_sat:
            plain_samples += smp
        if len(service) == n_sat:
            plain_wall = time.perf_counter() - t0
    bn.check()
    plain_fps = n_sat / plain_wall
    for r in plain:
        r.close()
    ctx2.close()
    # served arm: f16 copies of the same volumes
    ctx = bn.Context()
    served = []
    for d in vols:
        ds = dict(d, voxels=synth.to_storage(d["voxels"], "f16"), dtype="f16", majorant_round_up=True,
                  compensated_accum=True, fast_math=fast_math)
        served.append(bn.VolumeRenderer(ds, context=ctx, color_format="rgba8"))
    del vols
    torch.cuda.empty_cache()
    # slices of at most 16 waves and 64 M pixel-waves: on this stream 1168
    # served frames/s against 1064 with 4 waves and 16 M, and a lower p99 at
    # 1000 req/s (31.7 against 36.5 ms); the longest launch grows to ~18 ms
    server = bn.Server(ctx, hbm_budget_bytes=150 << 30, max_slots=256, slice_waves=16,
                       slice_pixel_waves=64 << 20)
    server.reserve(8 << 30)

    def serve(sub, arrivals):
        server.reset_stats()
        ids = []
        t_start = time.perf_counter()
        for (v, side, spp, cam), ta in zip(sub, arrivals):
            delay = t_start + ta - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            ids.append(server.submit(served[v], cam, side, side, spp, "rgba8"))
        for rid in ids:
            server.wait(rid, host)
        return server.stats()

    serve(reqs[:16], [0.0] * 16)  # warm-up
    st = serve(reqs[:n_sat], [0.0] * n_sat)
    sat = {"frames_per_s": st["completed"] / st["wallSeconds"],
           "Msamples_per_s": st["samples"] / st["wallSeconds"] / 1e6, "requests": n_sat}
    rate_rows = []
    for rate in rates:
        arr = poisson_arrivals(n_rate, rate, seed=int(rate) + 1)
        st = serve(reqs[:n_rate], arr)
        # the plain arm on the same arrivals: FIFO, its measured service times
        free, lat = 0.0, []
        for ta, sv in zip(arr, service[:n_rate]):
            start = max(ta, free)
            free = start + sv
            lat.append((free - ta) * 1e3)
        plain_span = max(free, float(arr[-1]))
        rate_rows.append({"rate_req_s": rate, "requests": n_rate,
                          "served": {"frames_per_s": st["completed"] / st["wallSeconds"],
                                     "p50_ms": st["p50Ms"], "p99_ms": st["p99Ms"], "max_launch_ms": st["maxSliceMs"],
                                     "gpu_busy_frac": st["busySeconds"] / st["wallSeconds"]},
                          "plain": {"frames_per_s": n_rate / plain_span, "p50_ms": percentile(lat, 0.5),
                                    "p99_ms": percentile(lat, 0.99)}})
        print(json.dumps({"partial": rate_rows[-1]}), file=sys.stderr, flush=True)
    server.close()
    for r in served:
        r.close()
    ctx.close()
    torch.cuda.empty_cache()
    svc_ms = [x * 1e3 for x in service[:n_sat]]
    return {"served_over_plain": sat["frames_per_s"] / plain_fps,
            "served": sat,
            "plain": {"frames_per_s": plain_fps, "Msamples_per_s": plain_samples / plain_wall / 1e6,
                      "service_p50_ms": percentile(svc_ms, 0.5), "service_p99_ms": percentile(svc_ms, 0.99)},
            "rates": rate_rows,
            "stream": "one request stream (seed 7) for both arms: volume of 16, side {256,512,1024}, "
                      "spp {1,4,16}, orbit camera",
            "served_form": "f16 storage, majorants rounded up, compensated accumulation" +
                           (", fast-math kernels" if fast_math else "") +
                           ", continuous batching (16 waves and at most 64M pixel-waves per launch), 150 GB budget",
            "plain_form": "f32 storage, exact kernels, one bnRender + read-back per request"}


def run_serving(args):
    """Config 5: the served and plain forms on one Poisson request stream over
    16 resident volumes (10 000 requests per rate unless --requests)."""
    rates = [float(x) for x in args.rates.split(",")]
    n = args.requests or 10000
    res = serving_arms(n_sat=min(n, 2000), rates=rates, n_rate=n)
    line = {"metric": METRIC, "value": res["served"]["frames_per_s"], "unit": "frames/s", "n_gpus": 1,
            "steps": len(rates), "warmup": 1, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f16 storage, f32 arithmetic", "data": "synthetic (16 seeded volumes)",
            "config": {"workload": "Poisson request stream over 16 resident volumes (seeds 100-115, edges "
                                   "log-U[128,1024]); side {256,512,1024}, spp {1,4,16}; HBM budget 150 GB",
                       "requests_per_rate": n, "rates": rates},
            "serving": res, "served_over_plain": res["served_over_plain"]}
    print(json.dumps(line), flush=True)
    return 0


def run_rmse(args):
    """Image RMSE against the FP64 expectation (oracle/bn_fp64.cpp, exact
    -log, off the hot path) for the plain FP32 path and every storage /
    precision form, on a reduced frame of the configured workload at high
    spp.  The FP64 reference is computed from the float32 field, so storage
    error shows up in the forms' RMSE."""
    import numpy as np
    import torch
    import barney_b200 as bn
    import oracle
    from barney_b200 import synth
    torch.cuda.set_device(0)
    w, h = (int(x) for x in args.rmse_size.split("x"))
    if args.config == "1":
        base = synth.config1(reference_semantics=True)
        f32 = base["voxels"]
        n = 64
    else:
        n = 512 if args.config == "2" else 1024
        f32d = synth.value_noise(n, 0, xp=torch, device="cuda")
        f32 = f32d.cpu().numpy()
        base = synth.config2(vol=f32, dtype="f32")
    base = dict(base, width=w, height=h)
    t0 = time.time()
    step = 1.0 / (n - 1)
    truth = oracle.render_expected_fp64(oracle.Scene(base), step=step, subpix=2, env_dirs=64)
    fp64_s = time.time() - t0
    forms = [("plain f32 (fastLog)", "f32", {}), ("f32 exact -log", "f32", {"exact_log": True}),
             ("f16 storage", "f16", {"majorant_round_up": True, "compensated_accum": True}),
             ("bf16 storage", "bf16", {"majorant_round_up": True, "compensated_accum": True}),
             ("u8 storage", "u8", {"majorant_round_up": True, "compensated_accum": True}),
             ("f32 fast math", "f32", {"fast_math": True}),
             ("f16 storage, fast math", "f16", {"majorant_round_up": True, "compensated_accum": True,
                                               "fast_math": True})]
    out = []
    for name, dtype, kw in forms:
        d = dict(base, voxels=synth.to_storage(f32, dtype), dtype=dtype, **kw)
        r = bn.VolumeRenderer(d, color_format="float4")
        r.set_spp(args.rmse_spp)
        r.render()
        img = r.read().astype(np.float64)
        st = r.stats()
        r.close()
        err = img[..., :3] - truth[..., :3]
        out.append({"form": name, "rmse": float(np.sqrt((err ** 2).mean())),
                    "mean_abs": float(np.abs(err).mean()), "render_ms": st["render_ms"],
                    "Msamples_per_s": st["samples"] / st["render_ms"] / 1e3})
    plain = out[0]["rmse"]
    for o in out:
        o["rmse_over_plain"] = o["rmse"] / plain
    line = {"rmse_vs_fp64": out, "config": args.config, "image": [w, h], "spp": args.rmse_spp,
            "fp64_oracle": {"step": step, "subpix": 2, "env_dirs": 64, "seconds": fp64_s, "threads": os.cpu_count()}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.rmse:
        return run_rmse(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.config == "4":
        return run_batch(args)
    if args.config == "5":
        return run_serving(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
