"""Parity at the benchmark workloads' full sizes: the CUDA path against the
CPU oracle, bit-exact, on the volumes and frames the bench renders.

* The 64^3 blob workload's whole 256x256 frame at 16 spp in the reference's
  own semantics (ambient 1, no lights, default single scatter), with the
  work counters.
* A centred 64x64 crop of the 512^3 f32 noise workload's 1920x1080 frame
  (8^3-voxel macrocells, HG single scatter with albedo 0.8, directional
  light plus ambient 0.25), 4 spp.
* 32x32 crops of the 1024^3 noise field stored as f32, f16 and u8, 2 spp.
  The crop's rays enter through the volume's z = 1 face, so its samples read
  voxels at high z indices: for f32, byte offsets beyond 2 GiB (up to
  4 GiB - 4), past what 32-bit signed offsets reach (the sampler indexes in
  64 bits, as rtcore/cpu/Texture.cpp:378-382 does with size_t).

The volumes are generated on the device (barney_b200.synth's torch path,
bit-identical to its numpy path) and copied to the host for the oracle.
"""
import numpy as np
import pytest

import oracle
from barney_b200 import synth
from tests.helpers import assert_bitexact

pytestmark = pytest.mark.gpu


def gpu_frame(d, spp):
    import barney_b200 as bn
    r = bn.VolumeRenderer(d, color_format="float4")
    try:
        r.set_spp(spp)
        r.render()
        return r.read(), r.stats()
    finally:
        r.close()


def oracle_crop(d_host, spp, rect):
    sc = oracle.Scene(d_host)
    acc, _, st = oracle.render(sc, 0, spp, rect=rect, threads=0)
    x0, y0, x1, y1 = rect
    return oracle.resolve(acc, spp)[y0:y1, x0:x1], st


def test_blob_workload_whole_frame():
    d = synth.config1(reference_semantics=True, spp=16)
    img, st = gpu_frame(d, 16)
    sc = oracle.Scene(d)
    acc, _, ost = oracle.render(sc, 0, 16, threads=0)
    assert_bitexact(img, oracle.resolve(acc, 16), "64^3 blobs, 256x256, 16 spp")
    for k in ("samples", "mc_visits", "rays"):
        assert st[k] == ost[k], (k, st[k], ost[k])
    assert st["samples"] > 100000


def test_noise512_centre_crop():
    import torch
    vol = synth.value_noise(512, 0, xp=torch, device="cuda")
    d = synth.config2(vol=vol, spp=4)
    img, _ = gpu_frame(d, 4)
    rect = (928, 508, 992, 572)  # 64 x 64 around the frame's centre
    want, st = oracle_crop(dict(d, voxels=vol.cpu().numpy()), 4, rect)
    del vol, d
    torch.cuda.empty_cache()
    assert st["samples"] > 5000
    x0, y0, x1, y1 = rect
    assert_bitexact(img[y0:y1, x0:x1], want, "512^3 f32 noise, centre crop of 1920x1080, 4 spp")


@pytest.mark.parametrize("dtype", ["f32", "f16", "u8"])
def test_noise1024_crop_at_high_z(dtype):
    import torch
    vol = synth.to_storage(synth.value_noise(1024, 0, xp=torch, device="cuda"), dtype)
    torch.cuda.empty_cache()
    d = synth.config2(vol=vol, dtype=dtype, spp=2)
    img, _ = gpu_frame(d, 2)
    rect = (928, 608, 960, 640)  # rays enter through the z = 1 face
    host = vol.cpu().numpy()
    del vol, d
    torch.cuda.empty_cache()
    d_host = synth.config2(vol=host, dtype=dtype, spp=2)
    want, st = oracle_crop(d_host, 2, rect)
    assert st["samples"] > 1000
    x0, y0, x1, y1 = rect
    assert_bitexact(img[y0:y1, x0:x1], want, f"1024^3 {dtype} noise, crop at z ~ 1, 2 spp")
