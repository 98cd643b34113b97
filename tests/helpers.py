"""Shared helpers of the parity tests: render the same scene through the
bn* C ABI (GPU) and through the CPU oracle."""
import numpy as np

import oracle
from barney_b200 import synth


def small_noise_scene(n=40, w=48, h=32, dtype="f32", **kw):
    """Config-2 semantics on a small noise volume (HG phase, dir light,
    ambient 0.25)."""
    vol = synth.to_storage(synth.value_noise(n, 0), dtype)
    d = synth.config2(vol=vol, dtype=dtype, width=w, height=h)
    d.update(kw)
    return d


def small_blob_scene(n=24, w=40, h=40, **kw):
    vol = synth.blobs(n, 0)
    d = synth.scene(vol, "f32", w, h, synth.tf_linear_ramp(128), 50.0, synth.DEFAULT_CAMERA, ambient=1.0)
    d.update(kw)
    return d


def oracle_render(desc, spp, accum_id0=0, accum=None, fmt="float4"):
    sc = oracle.Scene(desc)
    acc, _, st = oracle.render(sc, accum_id0, spp, accum=accum, threads=0)
    img = oracle.resolve(acc, accum_id0 + spp, fmt)
    return img, acc, st


def gpu_render(desc, spp, fmt="float4", renders=1):
    import barney_b200 as bn
    r = bn.VolumeRenderer(desc, color_format=fmt)
    try:
        r.set_spp(spp)
        for _ in range(renders):
            r.render()
        img = r.read()
        st = r.stats()
    finally:
        r.close()
    return img, st


def assert_bitexact(a, b, what=""):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, (a.shape, b.shape)
    if a.dtype == np.float32:
        av, bv = a.view(np.uint32), b.view(np.uint32)
    else:
        av, bv = a, b
    bad = np.argwhere(av != bv)
    assert bad.size == 0, f"{what}: {len(bad)} mismatches, first at {bad[:5].tolist()}: " \
                          f"{a[tuple(bad[0])] if bad.size else ''} vs {b[tuple(bad[0])] if bad.size else ''}"


def empty_checkpoint(width, height, accum_id):
    """A checkpoint of an empty frame buffer at accum_id (bnxFrameBufferRestore
    header: magic, version, width, height, accumID, hasComp, 2 reserved words),
    so that a render continues with the wave accum_id onto an empty buffer."""
    import struct
    return struct.pack("<8I", 0x43584E42, 1, width, height, accum_id, 0, 0, 0) + bytes(width * height * 16)


def render_batches(r, width, height, batches, per_batch):
    """Per-batch mean frames (batches, H, W, 4) of a VolumeRenderer: batch b
    renders waves b*per_batch .. (b+1)*per_batch-1 onto an empty buffer."""
    out = []
    r.set_spp(per_batch)
    for b in range(batches):
        r.accum_reset()
        if b:
            r.restore(empty_checkpoint(width, height, b * per_batch))
        r.render()
        ck = r.checkpoint()
        acc = np.frombuffer(ck[32:32 + width * height * 16], np.float32).reshape(height, width, 4)
        out.append(acc.astype(np.float64) / per_batch)
    return np.stack(out)
