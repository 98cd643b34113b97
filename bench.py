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
    p.add_argument("--config", default="2", choices=["1", "2", "3"])
    p.add_argument("--dtype", default=None, help="storage type for config 3 (f32, f16, u8, bf16)")
    p.add_argument("--spp", type=int, default=None)
    p.add_argument("--e2e-steps", type=int, default=None)
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
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
    desc = {"workload": f"{n}^3 {dtype} 6-octave value noise (seed 0), 8^3 macrocells, 1920x1080, {d['spp']} spp, "
                        "256-entry knot TF (seed 1) density 50, HG single scatter albedo 0.8, "
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
    return {"value": st["samples"] / secs / 1e6, "unit": "Msamples/s", "cores": threads, "kind": "port",
            "sample": f"{cw}x{ch} centred crop x {spp} waves of the frame ({st['samples']} volume samples, "
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
    stream = torch.cuda.current_stream()
    r.L.bnxSetStream(r.ctx, stream.cuda_stream)
    bn.check()

    def frame():
        r.accum_reset()
        r.render()
        return r.stats()

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
    e0.record(stream)
    for _ in range(args.steps):
        stats.append(frame())
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop() if sampler else None
    ms = e0.elapsed_time(e1)
    samples = sum(s["samples"] for s in stats)
    rays = sum(s["rays"] for s in stats)
    t = torch.tensor([ms, float(samples), float(rays)], dtype=torch.float64, device="cuda")
    if world > 1:
        tmax = t.clone()
        dist.all_reduce(tmax[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
        t[0] = tmax[0]
    ms_max, samples_all, rays_all = float(t[0]), float(t[1]), float(t[2])
    secs = ms_max / 1e3

    # roofline of the render kernel: algorithmic bytes per launch / its mean duration
    es = {"f32": 4, "f16": 2, "bf16": 2, "u8": 1}[d["dtype"]]
    alg = [8 * es * s["samples"] + 4 * s["mc_visits"] + 16 * s["pixel_samples"] for s in stats]
    kms = [s["render_ms"] for s in stats]
    achieved = statistics.mean(a / (k * 1e-3) for a, k in zip(alg, kms)) / 1e9
    peak, peak_kind = measured_peak()
    traffic = profiled_traffic(f"config{args.config}_{d['dtype']}")

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
        r.read(host)
        e2e_samples += r.stats()["samples"]
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    t2 = torch.tensor([e2e_ms, float(e2e_samples)], dtype=torch.float64, device="cuda")
    if world > 1:
        m = t2.clone()
        dist.all_reduce(m[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t2[1:], op=dist.ReduceOp.SUM)
        t2[0] = m[0]
    e2e_value = float(t2[1]) / (float(t2[0]) / 1e3) / 1e6
    h2d = 3 * 3 * 4 + 4 + 8  # position, direction, up, fovy, accumID/spp words
    d2h = d["width"] * d["height"] * 4

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        dh = dict(d)
        dh["voxels"] = d["voxels"].cpu().numpy()
        cpu = cpu_baseline(dh, args.cpu_seconds)
        cpu.pop("seconds", None)
    r.close()

    if rank == 0:
        n_frames = world * args.steps
        line = {
            "metric": METRIC, "value": samples_all / secs / 1e6, "unit": "Msamples/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": d["dtype"],
            "data": "synthetic (seeded value noise / Gaussian blobs generated on device)",
            "config": dict(desc, parallelism=f"replicas x{world}" if world > 1 else "single GPU",
                           l2="inputs larger than L2" if args.config != "1" else "volume fits L2 (1 MiB)"),
            "frames_per_s": n_frames / secs, "rays_per_s": rays_all / secs,
            "gpu_launches": 2 * args.steps,
            "clocks": clocks,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": traffic,
                         "algorithmic_bytes_per_launch": statistics.mean(alg),
                         "kernel_ms": statistics.mean(kms)},
            "e2e": {"value": e2e_value, "unit": "Msamples/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "frames_per_s": world * e2e_steps / (float(t2[0]) / 1e3)},
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
