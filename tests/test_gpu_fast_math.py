"""The fast-math form (renderer parameter bnx.fastMath) at its accuracy bar.

The fast-math kernels are compiled with FMA contraction and approximate
division and square root, except where a sample's texel coordinate and its
transfer-function coordinate are formed.  They are not bit-exact; they are
held to the bar stated for the path:

* trilinear field samples and TF lookups within 2 ulp of FP32, at the sample
  points of the golden vectors the reference's own code produced
  (tests/golden/ref_field.npz), through bnxVolumeSample;
* with identical per-pixel seeds, each pixel's mean at 4096 spp within 3
  Monte-Carlo standard errors of the oracle's (the standard error of the
  difference estimated per pixel from both sides' 16 batches of 256 waves;
  the share of channels a correct estimator fails by chance is allowed), on
  the 64^3 blob workload and on a crop of the 512^3 noise workload;
* jobs that need the extended kernels (multi-scatter here) run the exact
  kernels and stay bit-exact.
"""
import numpy as np
import pytest

import oracle
from barney_b200 import synth
from tests.helpers import assert_bitexact, oracle_render, render_batches, small_noise_scene
from test_ref_golden import FIELD_NAMES, field_scene, load

pytestmark = pytest.mark.gpu


def ulp_distance(a, b):
    """Units in the last place between float32 arrays of equal sign (0 for
    equal values, including two NaNs)."""
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)

    def ordered(x):
        i = x.view(np.int32).astype(np.int64)
        return np.where(i < 0, -(i & 0x7fffffff), i)

    d = np.abs(ordered(a) - ordered(b))
    both_nan = np.isnan(a) & np.isnan(b)
    return np.where(both_nan, 0, d)


@pytest.mark.parametrize("name", FIELD_NAMES)
def test_fast_samples_within_2_ulp_of_the_reference(name):
    """Trilinear samples within 2 ulp of the reference's sampler at the same
    points; the TF lookup (sampleAndMap's colour and density, principled
    volumes' included) within 2 ulp of the reference's at the scalar the
    fast sampler returned.  (The composite can differ by more: the TF's
    slope magnifies the sample's own 2 ulp.)"""
    import barney_b200 as bn
    import oracle
    z = load("ref_field.npz")
    d = field_scene(z, name)
    r = bn.VolumeRenderer(d)
    try:
        scal, rgba = r.sample(z[name + "__P"], fast_math=True)
    finally:
        r.close()
    ref_s = z[name + "__sample"]
    assert np.array_equal(np.isnan(scal), np.isnan(ref_s))
    if d.get("principled"):  # principled volumes sample (and render) with the exact kernels
        assert_bitexact(scal, ref_s, name)
        assert_bitexact(rgba, z[name + "__sample_rgba"], name)
        return
    ds = ulp_distance(scal, ref_s)
    assert ds.max() <= 2, f"{name}: trilinear {ds.max()} ulp"
    sc = oracle.Scene(d)
    ok = ~np.isnan(scal)
    tf = oracle.tf_map(sc, scal[ok])  # the reference's TF map, bit for bit (test_ref_golden.py)
    if d.get("principled"):  # Volume.h:65-72 on the reference's principledSampleMap
        p, _ = oracle.principled(sc, scal[ok])
        want = np.zeros_like(tf)
        pos = tf[:, 3] > 0
        want[pos, :3] = p[pos, :3] * tf[pos, :3]
        want[pos, 3] = p[pos, 3] * tf[pos, 3]
    else:
        want = tf
    dm = ulp_distance(rgba[ok], want)
    assert dm.max() <= 2, f"{name}: TF lookup {dm.max()} ulp"
    assert np.all(rgba[~ok] == 0)


def pixel_means_within_3_se(d_gpu, d_oracle, rect, batches=16, per_batch=256, what=""):
    """Per-pixel means over batches x per_batch waves: the fast-math kernels
    (on the device, d_gpu) against the oracle (d_oracle: the same scene with
    its volume in host memory), inside rect (x0, y0, x1, y1), with the same
    per-pixel seeds.  Each side's standard error comes from its own batch
    means; a channel passes when its means differ by at most 3 standard
    errors of the difference.  Under that test a correct estimator fails in
    0.27 % of channels by chance, so up to 0.5 % may; none may pass 8."""
    import barney_b200 as bn
    W, H = d_gpu["width"], d_gpu["height"]
    r = bn.VolumeRenderer(dict(d_gpu, fast_math=True), color_format="float4")
    try:
        fb = render_batches(r, W, H, batches, per_batch)
    finally:
        r.close()
    x0, y0, x1, y1 = rect
    fb = fb[:, y0:y1, x0:x1]
    sc = oracle.Scene(d_oracle)
    ob = []
    for b in range(batches):
        acc, _, _ = oracle.render(sc, b * per_batch, per_batch, rect=rect, threads=0)
        ob.append(acc[y0:y1, x0:x1].astype(np.float64) / per_batch)
    ob = np.stack(ob)
    se = np.sqrt(fb.var(axis=0, ddof=1) / batches + ob.var(axis=0, ddof=1) / batches)
    diff = np.abs(fb.mean(axis=0) - ob.mean(axis=0))
    z = diff / np.maximum(se, 1e-7 * np.maximum(1.0, np.abs(ob.mean(axis=0))))
    frac = float((z > 3.0).mean())
    assert frac <= 0.005 and z.max() <= 8.0, \
        f"{what}: {frac:.4%} of channels beyond 3 standard errors, largest {float(z.max()):.2f}"
    return frac, float(z.max())


def test_fast_blob_workload_pixel_means():
    d = synth.config1(reference_semantics=True)
    d["width"], d["height"] = 96, 96
    pixel_means_within_3_se(d, d, (0, 0, 96, 96), what="64^3 blobs, 96x96, 4096 spp")


def test_fast_noise512_crop_pixel_means():
    import torch
    vol = synth.value_noise(512, 0, xp=torch, device="cuda")
    d_gpu = synth.config2(vol=vol)
    d_host = synth.config2(vol=vol.cpu().numpy())
    pixel_means_within_3_se(d_gpu, d_host, (944, 524, 976, 556),
                            what="512^3 noise, 32x32 centre crop of 1920x1080, 4096 spp")
    del vol, d_gpu
    torch.cuda.empty_cache()


def test_fast_math_request_on_extended_scene_runs_exact_kernels():
    d = small_noise_scene(w=32, h=24, max_volume_bounces=2, fast_math=True)
    import barney_b200 as bn
    r = bn.VolumeRenderer(d)
    try:
        r.set_spp(2)
        r.render()
        img = r.read()
    finally:
        r.close()
    want, _, _ = oracle_render(d, 2)
    assert_bitexact(img, want, "multi-scatter scene with bnx.fastMath")


def test_fast_math_frame_differs_only_slightly():
    """The fast kernels follow the same RNG streams: a frame differs from the
    exact one only where a rounding difference flips a Woodcock decision."""
    import barney_b200 as bn
    d = small_noise_scene(n=48, w=64, h=48)
    out = {}
    for fm in (False, True):
        r = bn.VolumeRenderer(dict(d, fast_math=fm))
        try:
            r.set_spp(16)
            r.render()
            out[fm] = r.read().copy()
        finally:
            r.close()
    assert not np.array_equal(out[False], out[True])
    rel = np.abs(out[True] - out[False]).mean() / np.abs(out[False]).mean()
    assert rel < 0.05, rel
