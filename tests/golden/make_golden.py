"""Generate the committed golden fixtures of the structured-volume path.

    python tests/golden/make_golden.py

The reference (Barney) cannot be built or imported here and ships no golden
vectors for this path, so the fixtures are produced by the CPU restatement
in oracle/ (itself pinned by hand-derived known answers in
tests/test_oracle_kat.py).  They freeze its outputs -- macrocell ranges and
majorants, field samples, transfer-function lookups, rendered frames and
work counters -- on small seeded inputs so that the oracle and the CUDA
path are both checked against the same stored numbers.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from barney_b200 import synth  # noqa: E402


def scenes():
    noise = synth.value_noise(21, 7)[:, 2:20, 4:17].copy()  # 21 x 18 x 13, ragged
    out = {}
    for dtype in ("f32", "u8", "f16"):
        vol = synth.to_storage(noise, dtype)
        d = synth.config2(vol=vol, dtype=dtype, width=24, height=16)
        d["spacing"] = (1.0 / 12, 1.0 / 17, 1.0 / 20)
        out[f"noise_{dtype}"] = d
    blob = synth.blobs(17, 0)
    out["blobs_ambient"] = synth.scene(blob, "f32", 24, 16, synth.tf_linear_ramp(128), 50.0,
                                       synth.DEFAULT_CAMERA, ambient=1.0)
    out["blobs_ea"] = synth.scene(blob, "f32", 24, 16, synth.tf_linear_ramp(128), 50.0, synth.DEFAULT_CAMERA,
                                  ambient=0.0, emission_absorption=True, bg_color=(0.1, 0.2, 0.3, 1.0))
    # the multi-scatter build: HG sampling with up to 3 volume bounces; and a
    # principled volume with absorption, emission and blackbody, 2 bounces
    out["noise_multiscatter"] = dict(out["noise_f32"], anisotropy=0.6, max_volume_bounces=3)
    out["noise_principled"] = dict(out["noise_f32"], anisotropy=-0.3, max_volume_bounces=2, principled={
        "enabled": 1, "absorption_color": (0.2, 0.1, 0.05), "emission_strength": 1.5,
        "blackbody_intensity": 0.5, "temperature": 4500.0, "density_threshold": 0.2})
    out["noise_exact_log"] = dict(out["noise_u8"], exact_log=True)
    # isosurfaces with a matte material: alone on the blobs (directional light
    # + ambient), inside the noise volume, and semi-opaque in the multi-scatter build
    out["blobs_iso"] = synth.scene(blob, "f32", 24, 16, synth.tf_linear_ramp(128), 50.0, synth.DEFAULT_CAMERA,
                                   ambient=0.3, dir_lights=synth.CONFIG2_LIGHTS, volume=False,
                                   iso={"value": 0.3, "color": (0.9, 0.5, 0.2)})
    out["noise_iso"] = dict(out["noise_f32"], iso={"value": 0.55, "color": (0.3, 0.6, 0.9)})
    out["noise_iso_multiscatter"] = dict(out["noise_f32"], anisotropy=0.4, max_volume_bounces=2,
                                         iso={"value": 0.5, "color": (0.8, 0.8, 0.3, 0.9), "opacity": 0.7})
    return out


def compute(name, d):
    sc = oracle.Scene(d)
    res = {}
    ranges = oracle.build_ranges(sc)
    res["ranges"] = ranges
    res["majorants"] = oracle.map_majorants(sc, ranges)
    rng = np.random.default_rng(11)
    P = rng.uniform(-0.05, 1.05, size=(256, 3)).astype(np.float32)
    res["points"] = P
    res["point_scalar"], res["point_rgba"] = oracle.sample_points(sc, P)
    for spp in (1, 3):
        acc, _, st = oracle.render(sc, 0, spp, threads=1)
        res[f"accum_spp{spp}"] = acc
        res[f"frame_spp{spp}"] = oracle.resolve(acc, spp, "float4")
        res[f"counts_spp{spp}"] = np.array([st["samples"], st["mc_visits"], st["rays"]], np.uint64)
    return res


def main(names=None):
    """(Re)writes the named fixtures, or all of them."""
    for name, d in scenes().items():
        if names and name not in names:
            continue
        res = compute(name, d)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **res)
        print(name, {k: v.shape for k, v in res.items()})


if __name__ == "__main__":
    main(sys.argv[1:])
