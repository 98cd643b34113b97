"""Generate tests/golden/ref_*.npz from the REFERENCE'S OWN code.

    python tests/golden/make_ref_golden.py [--ref /root/reference]

Builds oracle/_ref/libbnref.so (oracle/Makefile, target `ref`): the
reference's RNG and hash, fastLog, Woodcock::sampleRange, sampleAndMap, dda3,
transfer-function map and majorant, principled-volume functions,
linear_to_srgb / make_rgba, and its CPU backend's texture samplers and
binary16 rounding, compiled from its sources where they lie, behind the
stand-in include tree oracle/refshim and the glue in oracle/ref_harness.cpp.
It then evaluates them on seeded inputs and stores inputs and outputs here.

The reference tree is present only where the fixtures are made; the tests
(tests/test_ref_golden.py on the CPU oracle, tests/test_gpu_ref_golden.py on
the CUDA kernels) read the stored files.
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle import reference as R  # noqa: E402
from barney_b200 import synth  # noqa: E402

F32 = np.float32


def scene_arrays(d):
    """The scene inputs a fixture stores, so that tests rebuild the scene
    without the generators."""
    vol = np.ascontiguousarray(d["voxels"])
    cam = d["camera"]
    return {
        "voxels": vol, "dtype": np.array(d["dtype"]), "spacing": np.array(d["spacing"], F32),
        "origin": np.array(d.get("origin", (0.0, 0.0, 0.0)), F32),
        "tf": np.ascontiguousarray(d["tf"], F32).reshape(-1, 4), "domain": np.array(d.get("domain", (0.0, 1.0)), F32),
        "density": np.array(d["density"], F32),
        "cam_position": np.array(cam["position"], F32), "cam_direction": np.array(cam["direction"], F32),
        "cam_up": np.array(cam.get("up", (0.0, 1.0, 0.0)), F32), "cam_fovy": np.array(cam.get("fovy", 60.0), F32),
        "width": np.array(d["width"]), "height": np.array(d["height"]),
    }


def rng_fixture():
    seeds = np.array([(0, 0), (1, 2), (7, 0), (123456, 7890), (4294967295, 5), (1920, 1080), (65, 4),
                      (3000000000, 4000000000)], np.uint64)
    streams = np.stack([R.rng_stream(int(a), int(b), 64) for a, b in seeds])
    floats = np.stack([R.rng_floats(int(a), int(b), 64) for a, b in seeds])
    ray_seeds = np.array([R.ray_seed(int(a), int(b)) for a, b in seeds], np.uint64)
    parents = np.array([0xcafef00dd15ea5e5, 0x1234567890abcdef, 0, 1, 0xffffffffffffffff, int(ray_seeds[3])],
                       np.uint64)
    hashes = np.array([R.hash3(0, 0, 0), 0, 0xdeadbeef, 1 << 40, 290374, R.hash3(3, 1, 4)], np.uint64)
    derived, parent_after = [], []
    for p, h in zip(parents, hashes):
        o, pa = R.rng_derived(int(p), int(h), 16)
        derived.append(o)
        parent_after.append(pa)
    triples = np.array([(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (5, 7, 9), (4294967295, 4294967295, 4294967295)],
                       np.uint32)
    hash3 = np.array([R.hash3(int(a), int(b), int(c)) for a, b, c in triples], np.uint64)
    np.savez_compressed(os.path.join(HERE, "ref_rng.npz"), seeds=seeds, streams=streams, floats=floats,
                        ray_seeds=ray_seeds, parents=parents, hashes=hashes, derived=np.stack(derived),
                        parent_after=np.array(parent_after, np.uint64), triples=triples, hash3=hash3)


def scalar_fixture():
    rng = np.random.default_rng(11)
    # fastLog is called on 1 - r, r in [0, 1): (0, 1] in steps of 2^-24
    r = np.concatenate([np.arange(0, 64), rng.integers(0, 1 << 24, 4000), (1 << 24) - np.arange(1, 64)])
    log_x = (F32(1.0) - (r.astype(F32) * F32(1.0 / 16777216.0))).astype(F32)
    log_x = np.concatenate([log_x, np.array([1e-30, 1e-10, 0.5, 2.0, 10.0, 1e6], F32)])
    # binary16 rounding: random values over the whole half range, ties, subnormals, overflow
    hx = np.concatenate([
        (rng.standard_normal(4000) * np.exp2(rng.uniform(-26, 17, 4000))).astype(F32),
        np.array([0.0, -0.0, 1.0, 65504.0, 65519.99, 65520.0, 1e9, -1e9, 6.1035156e-05, 5.96e-08, 2.98e-08,
                  2.99e-08, 1.0 + 2 ** -11, 1.0 + 3 * 2 ** -11, np.inf, -np.inf], F32)])
    half_bits_all = np.arange(65536, dtype=np.uint16)
    srgb_x = np.concatenate([np.linspace(-0.1, 1.2, 2000, dtype=F32), np.array([0.0031308, 0.0031309, 1.0], F32)])
    rgba = np.concatenate([rng.uniform(-0.1, 1.1, (1000, 4)).astype(F32),
                           np.array([[255 / 256, 1.0, 0.0, 0.5], [0.99999, 0.0039, 0.00390625, 2.0]], F32)])
    np.savez_compressed(os.path.join(HERE, "ref_scalar.npz"), log_x=log_x, fastlog=R.fastlog(log_x), half_x=hx,
                        half_bits=R.f2h(hx), h2f=R.h2f(half_bits_all), srgb_x=srgb_x,
                        srgb=R.linear_to_srgb(srgb_x), rgba=rgba, make_rgba=R.make_rgba(rgba))


def tf_scenes():
    base = synth.scene(np.zeros((2, 2, 2), F32), "f32", 4, 4, synth.tf_linear_ramp(128), 50.0,
                       synth.DEFAULT_CAMERA)
    knots = dict(base, tf=synth.tf_knots(256, 1))
    rng = np.random.default_rng(5)
    odd = dict(base, tf=rng.uniform(0, 1, (7, 4)).astype(F32), domain=(-0.3, 2.1), density=3.5)
    return {"linear128": base, "knots256": knots, "odd7": odd}


def tf_fixture():
    out = {}
    rng = np.random.default_rng(6)
    for name, d in tf_scenes().items():
        sc = oracle.Scene(d)
        lo, hi = d.get("domain", (0.0, 1.0))
        n = np.asarray(d["tf"]).reshape(-1, 4).shape[0]
        knots = np.float32(lo) + (np.arange(n, dtype=F32) / F32(n - 1)) * np.float32(hi - lo)
        v = np.concatenate([rng.uniform(lo - 0.5, hi + 0.5, 2000).astype(F32), knots,
                            np.array([lo, hi, np.nextafter(F32(hi), F32(-1)), -1e30, 1e30], F32)]).astype(F32)
        r = rng.uniform(lo - 0.2, hi + 0.2, (1500, 2)).astype(F32)
        r[:500].sort(axis=1)                     # proper ranges
        r[1000:1100, 1] = r[1000:1100, 0]        # degenerate
        r = np.concatenate([r, np.array([[np.inf, -np.inf], [lo, hi], [hi, lo]], F32)])
        out.update({f"{name}_tf": np.ascontiguousarray(d["tf"], F32).reshape(-1, 4),
                    f"{name}_domain": np.array(d.get("domain", (0.0, 1.0)), F32),
                    f"{name}_density": np.array(d["density"], F32),
                    f"{name}_v": v, f"{name}_map": R.tf_map(sc, v),
                    f"{name}_ranges": r, f"{name}_majorants": R.map_majorants(sc, r)})
    np.savez_compressed(os.path.join(HERE, "ref_tf.npz"), **out)


def field_scenes():
    """Small volumes for the sampler and macrocell fixtures."""
    rng = np.random.default_rng(9)
    out = {}
    ragged = rng.random((4, 7, 5)).astype(F32)  # [z][y][x]: 5 x 7 x 4 scalars
    out["ragged_f32"] = synth.scene(ragged, "f32", 8, 8, synth.tf_linear_ramp(128), 50.0, synth.DEFAULT_CAMERA)
    out["ragged_f32"]["spacing"] = (0.25, 1.0 / 6.0, 1.0 / 3.0)
    out["ragged_f32"]["origin"] = (-0.1, 0.2, 0.05)
    u8 = rng.integers(0, 256, (11, 6, 9)).astype(np.uint8)
    out["ragged_u8"] = synth.scene(u8, "u8", 8, 8, synth.tf_knots(256, 1), 50.0, synth.DEFAULT_CAMERA)
    out["ragged_u8"]["spacing"] = (1.0 / 8.0, 0.2, 0.1)
    blob = synth.blobs(24, 0)
    out["blobs24_f32"] = synth.scene(blob, "f32", 8, 8, synth.tf_linear_ramp(128), 50.0, synth.DEFAULT_CAMERA)
    noise = synth.to_storage(synth.value_noise(40, 0), "u8")
    out["noise40_u8"] = synth.config2(vol=noise, dtype="u8", width=8, height=8)
    big = synth.value_noise(33, 3)[:, :, :29].copy()  # 29 x 33 x 33: macrocells 4 x 4 x 4, last ones partial
    out["noise_ragged_f32"] = synth.config2(vol=big, dtype="f32", width=8, height=8)
    out["noise_ragged_f32"]["spacing"] = (1.0 / 28, 1.0 / 32, 1.0 / 32)
    pv = synth.value_noise(17, 4)
    out["principled17_f32"] = synth.config2(vol=pv, dtype="f32", width=8, height=8)
    out["principled17_f32"]["principled"] = {
        "enabled": True, "density": 2.0, "density_threshold": 0.1, "density_scale": 1.5,
        "value_range": (0.05, 0.9), "scatter_color": (0.9, 0.5, 0.2), "absorption_color": (0.1, 0.2, 0.3),
        "emission_strength": 0.7, "emission_color": (1.0, 0.6, 0.2)}
    return out


def field_fixture():
    out = {}
    rng = np.random.default_rng(10)
    for name, d in field_scenes().items():
        sc = oracle.Scene(d)
        nz, ny, nx = np.asarray(d["voxels"]).shape
        # texel coordinates: the rel+.5 boundaries, edges, outside, random
        grid = np.stack(np.meshgrid(np.arange(-1, nx + 2) * 0.5, np.arange(-1, ny + 2) * 0.5,
                                    np.arange(-1, nz + 2) * 0.5, indexing="ij"), -1).reshape(-1, 3)
        if grid.shape[0] > 4000:  # larger volumes: a subset of the half-texel lattice
            grid = grid[rng.choice(grid.shape[0], 4000, replace=False)]
        tc = np.concatenate([grid, rng.uniform(-0.5, 0.5, (3000, 3)) * np.array([nx, ny, nz]) + np.array([nx, ny, nz]) / 2.0])
        tc = tc.astype(F32)
        org = np.array(d.get("origin", (0, 0, 0)), F32)
        ext = np.array(d["spacing"], F32) * np.array([nx - 1, ny - 1, nz - 1], F32)
        P = (org + rng.uniform(-0.05, 1.05, (3000, 3)).astype(F32) * ext).astype(F32)
        P = np.concatenate([P, org[None, :], (org + ext)[None, :]]).astype(F32)
        scal, rgba = R.sample_points(sc, P)
        ranges = R.build_ranges(sc)
        ent = dict(scene_arrays(d))
        ent.update(tc=tc, tex_linear=R.tex3d(sc, tc, True), tex_nearest=R.tex3d(sc, tc, False), P=P,
                   sample=scal, sample_rgba=rgba, ranges=ranges, majorants=R.map_majorants(sc, ranges))
        if d.get("principled"):
            pvals = np.concatenate([np.linspace(-0.2, 1.2, 500, dtype=F32), scal[:200]])
            m, e = R.principled(sc, pvals)
            ent.update(principled_v=pvals, principled_map=m, principled_emission=e,
                       principled_params=np.array(repr(d["principled"])))
        for k, v in ent.items():
            out[f"{name}__{k}"] = v
    np.savez_compressed(os.path.join(HERE, "ref_field.npz"), names=np.array(list(field_scenes().keys())), **out)


def dda_fixture():
    rays = []
    rng = np.random.default_rng(12)
    grid = (8, 6, 5)
    for o, d, t in [((0.5, 0.5, 0.5), (1, 0, 0), 1e30), ((-2, 3.2, 2.5), (1, 0, 0), 1e30),
                    ((-1, -1, -1), (1, 1, 1), 1e30), ((9, 7, 6), (-1, -1, -1), 1e30),
                    ((4, 3, 2.5), (0, 0, 1), 1e30), ((4, 3, 2.5), (0, 1e-6, -1), 1e30),
                    ((4, 3, 2.5), (1e-6, 1e-6, 1), 1e30), ((-1, 3, 2), (1, 0.3, 0.1), 2.5),
                    ((-1, 3, 2), (1, 0.3, 0.1), 0.5), ((20, 20, 20), (1, 1, 1), 1e30),
                    ((4, 9, 2), (0, 0, 1), 1e30), ((8, 6, 5), (-1, -1, -1), 1e30), ((0, 0, 0), (1, 1, 1), 3.0),
                    ((2, 2, 2), (0.5, -0.25, 0.125), 1e30)]:
        rays.append((o, d, t))
    for _ in range(200):
        o = rng.uniform(-3, 11, 3)
        d = rng.standard_normal(3)
        if rng.random() < 0.2:
            d[rng.integers(0, 3)] = 1e-6
        rays.append((o, d, float(rng.choice([1e30, rng.uniform(0.5, 20)]))))
    org = np.array([r[0] for r in rays], F32)
    dirs = np.array([r[1] for r in rays], F32)
    tmax = np.array([r[2] for r in rays], F32)
    cells = np.full((len(rays), 64, 3), -9, np.int32)
    ts = np.zeros((len(rays), 64, 2), F32)
    counts = np.zeros(len(rays), np.int32)
    for i in range(len(rays)):
        c, t = R.dda_cells(org[i], dirs[i], float(tmax[i]), grid, 64)
        counts[i] = len(c)
        cells[i, :len(c)] = c
        ts[i, :len(c)] = t
    np.savez_compressed(os.path.join(HERE, "ref_dda.npz"), grid=np.array(grid, np.int32), org=org, dir=dirs,
                        tmax=tmax, counts=counts, cells=cells, ts=ts)


def trace_scenes():
    """Frames whose primary rays' first collisions are stored: the
    emission-absorption render of the same frame shows them pixel by pixel."""
    out = {}
    blob = synth.blobs(32, 0)
    out["blobs32_f32"] = (synth.scene(blob, "f32", 64, 48, synth.tf_linear_ramp(128), 50.0, synth.DEFAULT_CAMERA),
                          (0, 1, 7))
    noise = synth.to_storage(synth.value_noise(40, 0), "u8")
    out["noise40_u8"] = (synth.config2(vol=noise, dtype="u8", width=48, height=32), (0, 3))
    # looking straight down -z from above the cube centre: the middle column
    # and row of an odd-sized frame at accumID 0 have exactly-zero components
    cam = {"position": (0.5, 0.5, 2.2), "direction": (0.0, 0.0, -1.0), "up": (0.0, 1.0, 0.0), "fovy": 40.0}
    out["axis_aligned_f32"] = (synth.scene(synth.value_noise(24, 2), "f32", 33, 25, synth.tf_knots(256, 1), 50.0,
                                           cam), (0, 1))
    inside = {"position": (0.45, 0.55, 0.5), "direction": (0.3, -0.2, 1.0), "up": (0.0, 1.0, 0.0), "fovy": 70.0}
    out["camera_inside_f32"] = (synth.scene(synth.blobs(20, 1), "f32", 40, 30, synth.tf_linear_ramp(128), 20.0,
                                            inside), (0, 2))
    ragged = synth.value_noise(21, 7)[:, 2:20, 4:17].copy()
    d = synth.config2(vol=ragged, dtype="f32", width=40, height=28)
    d["spacing"] = (1.0 / 12, 1.0 / 17, 1.0 / 20)
    d["origin"] = (0.02, -0.03, 0.01)
    out["ragged_f32"] = (d, (0, 5))
    return out


def trace_fixture():
    out = {}
    rng = np.random.default_rng(13)
    for name, (d, accum_ids) in trace_scenes().items():
        sc = oracle.Scene(d)
        ent = dict(scene_arrays(d))
        ent["accum_ids"] = np.array(accum_ids, np.int32)
        for a in accum_ids:
            hit, t, rgb, counts = R.trace_frame(sc, a)
            ent.update({f"hit{a}": hit, f"t{a}": t, f"rgb{a}": rgb, f"counts{a}": counts})
        # explicit rays with explicit seed states
        nr = 300
        org = (rng.uniform(-0.5, 1.5, (nr, 3))).astype(F32)
        dirs = rng.standard_normal((nr, 3)).astype(F32)
        dirs[::17, rng.integers(0, 3)] = 0.0
        tmax = np.where(rng.random(nr) < 0.2, rng.uniform(0.1, 1.5, nr), 1e30).astype(F32)
        seeds = rng.integers(0, 2 ** 63, nr, dtype=np.int64).astype(np.uint64)
        rh, rt, rrgb, rc = [], [], [], []
        for i in range(nr):
            h, t, c, cnt = R.trace_ray(sc, org[i], dirs[i], float(tmax[i]), int(seeds[i]))
            rh.append(h)
            rt.append(t)
            rrgb.append(c)
            rc.append(cnt)
        ent.update(ray_org=org, ray_dir=dirs, ray_tmax=tmax, ray_seed=seeds, ray_hit=np.array(rh, np.int32),
                   ray_t=np.array(rt, F32), ray_rgb=np.array(rrgb, F32), ray_counts=np.array(rc, np.int32))
        for k, v in ent.items():
            out[f"{name}__{k}"] = v
    np.savez_compressed(os.path.join(HERE, "ref_trace.npz"), names=np.array(list(trace_scenes().keys())), **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    a = ap.parse_args()
    R.build(a.ref)
    rng_fixture()
    scalar_fixture()
    tf_fixture()
    field_fixture()
    dda_fixture()
    trace_fixture()
    print("wrote", sorted(f for f in os.listdir(HERE) if f.startswith("ref_")))


if __name__ == "__main__":
    main()
