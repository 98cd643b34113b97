"""The CUDA kernels against golden vectors produced by the REFERENCE'S OWN code
(tests/golden/ref_*.npz, made by tests/golden/make_ref_golden.py from the
reference's sources compiled here).

* Macrocell scalar ranges and majorants (StructuredData_computeMCs, mapMCs
  with TransferFunction::DD::majorant and principledMajorant) read back with
  bnxVolumeGetMacrocells.
* The first Woodcock collision of every pixel's primary ray (the reference's
  dda3, Woodcock::sampleRange with fastLog, Random2 / hash, the CPU LINEAR
  tex3D and TransferFunction::DD::map), seen through one emission-absorption
  wave: the wave adds the TF colour at the collision (clamped at
  10 * (1 + accumID)) and alpha 1, or the background for a miss.  The wave's
  accumID is set by restoring a checkpoint of an empty frame buffer, so any
  wave of a frame can be rendered alone.  Work counters (samples, macrocell
  visits) equal the reference's per-pixel sums.

All comparisons are bit-exact.
"""
import numpy as np
import pytest

from test_ref_golden import FIELD_NAMES, TRACE_NAMES, assert_same, field_scene, load, trace_scene
from tests.helpers import empty_checkpoint

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", FIELD_NAMES)
def test_macrocells(name):
    import barney_b200 as bn
    z = load("ref_field.npz")
    d = field_scene(z, name)
    r = bn.VolumeRenderer(d)
    try:
        ranges, maj = r.macrocells()
    finally:
        r.close()
    assert_same(ranges, z[name + "__ranges"], f"{name}: macrocell ranges")
    assert_same(maj, z[name + "__majorants"], f"{name}: majorants")


@pytest.mark.parametrize("name", FIELD_NAMES)
def test_field_samples(name):
    """The render kernels' sampler and sampleAndMap on the device
    (bnxVolumeSample) at the fixture's world points: the reference's CPU
    LINEAR tex3D behind StructuredDataSampler, and its TF map (principled
    sampleAndMap for the principled scene)."""
    import barney_b200 as bn
    z = load("ref_field.npz")
    r = bn.VolumeRenderer(field_scene(z, name))
    try:
        scal, rgba = r.sample(z[name + "__P"])
    finally:
        r.close()
    assert_same(scal, z[name + "__sample"], f"{name}: structured sampler")
    assert_same(rgba, z[name + "__sample_rgba"], f"{name}: sampleAndMap")


def expected_wave(hit, rgb, accum_id, bg=(0.0, 0.0, 0.0, 1.0)):
    """The accumulation buffer after one emission-absorption wave at accum_id
    onto an empty buffer (shadeRays.cu:996-1040 with the collision's colour)."""
    H, W = hit.shape
    clamp = np.float32(10.0 * (1 + accum_id))
    out = np.zeros((H, W, 4), np.float32)
    c = np.minimum(rgb.astype(np.float32), clamp)
    bgc = np.minimum(np.array(bg[:3], np.float32), clamp)
    if accum_id == 0:  # the first wave writes
        out[..., :3] = np.where(hit[..., None] != 0, c, bgc)
        out[..., 3] = np.where(hit != 0, np.float32(1.0), np.float32(bg[3]))
    else:  # later waves add positive channels onto 0
        out[..., :3] = np.where(hit[..., None] != 0, np.where(c > 0, c, 0), np.where(bgc > 0, bgc, 0))
        out[..., 3] = np.where(hit != 0, np.float32(1.0), np.float32(bg[3]) if bg[3] > 0 else np.float32(0))
    return out


@pytest.mark.parametrize("name", TRACE_NAMES)
def test_primary_first_collisions(name):
    import barney_b200 as bn
    z = load("ref_trace.npz")
    p = name + "__"
    d = trace_scene(z, name, emission_absorption=True, ambient=0.0, spp=1)
    W, H = d["width"], d["height"]
    r = bn.VolumeRenderer(d)
    try:
        for a in z[p + "accum_ids"]:
            a = int(a)
            r.accum_reset()
            if a > 0:
                r.restore(empty_checkpoint(W, H, a))
            r.render()
            st = r.stats()
            ck = r.checkpoint()
            accum = np.frombuffer(ck[32:32 + W * H * 16], np.float32).reshape(H, W, 4)
            want = expected_wave(z[f"{p}hit{a}"], z[f"{p}rgb{a}"], a)
            assert_same(accum, want, f"{name}: wave at accumID {a}")
            cnt = z[f"{p}counts{a}"]
            assert st["samples"] == int(cnt[..., 0].sum()), (name, a, st["samples"])
            assert st["mc_visits"] == int(cnt[..., 1].sum()), (name, a, st["mc_visits"])
    finally:
        r.close()
