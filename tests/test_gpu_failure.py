"""Failure detection without a GPU fault: a render that exceeds its deadline
is stopped through the kernel's abort word, bnRender reports a timeout, and
the same context renders the next frame correctly."""
import numpy as np
import pytest

from tests.helpers import assert_bitexact, gpu_render, oracle_render, small_noise_scene

pytestmark = pytest.mark.gpu


def test_render_deadline_aborts_and_context_recovers():
    import barney_b200 as bn
    from barney_b200 import synth
    big = synth.config2(n=96, width=1920, height=1080, spp=256)  # a frame of ~50 ms
    r = bn.VolumeRenderer(big, color_format="rgba8")
    try:
        r.set_spp(1)
        r.render()  # the kernels' code is loaded on the first launch of a process
        r.set_spp(256)
        r.set_timeout(1)
        with pytest.raises(bn.BarneyError) as e:
            r.render()
        assert "error 8" in str(e.value)
        assert r.stats()["error_flags"] & 2  # aborted
        r.set_timeout(0)
        r.set_spp(1)
        r.render()  # the context is still usable
        assert r.stats()["error_flags"] == 0
    finally:
        r.close()
    d = small_noise_scene(w=24, h=16)
    img, st = gpu_render(d, 2)
    ref, _, _ = oracle_render(d, 2)
    assert_bitexact(img, ref, "after an aborted frame")


def test_batch_deadline_aborts_and_context_recovers():
    import barney_b200 as bn
    from barney_b200 import synth
    ctx = bn.Context()
    big = [bn.VolumeRenderer(synth.config2(n=96, width=1920, height=1080, spp=128), context=ctx,
                             color_format="rgba8") for _ in range(2)]
    small = bn.VolumeRenderer(small_noise_scene(w=24, h=16), context=ctx, color_format="float4")
    try:
        big[0].set_timeout(1)  # the deadline belongs to the shared context
        with pytest.raises(bn.BarneyError) as e:
            ctx.render_batch(big)
        assert "error 8" in str(e.value)
        assert ctx.stats()["error_flags"] & 2
        big[0].set_timeout(0)
        small.set_spp(2)
        ctx.render_batch([small])
        assert ctx.stats()["error_flags"] == 0
        ref, _, _ = oracle_render(small_noise_scene(w=24, h=16), 2)
        assert_bitexact(small.read(), ref, "batch after an aborted batch")
    finally:
        for r in big + [small]:
            r.close()
        ctx.close()


def test_iteration_cap_ends_runaway_rays_and_sets_the_error_bit():
    # A majorant far above every sample the rays meet: the TF is opaque only
    # at its last entry, which the field reaches at one voxel per macrocell,
    # so every macrocell's majorant is 1e9 times the density rays see and a
    # ray crossing one would take ~1e8 Woodcock steps.  Each ray stops
    # at 2^22 steps, as if it left the grid, with error bit 1; the context
    # then renders normally.
    import barney_b200 as bn
    from barney_b200 import synth
    vol = (0.5 * synth.value_noise(24, 3)).astype(np.float32)
    vol[4::8, 4::8, 4::8] = 1.0  # one spike in every macrocell
    tf = np.zeros((256, 4), np.float32)
    tf[:, :3] = 0.5
    tf[:, 3] = 1e-9
    tf[-1, 3] = 1.0
    d = synth.scene(vol, "f32", 4, 4, tf, 1e9, synth.DEFAULT_CAMERA)
    r = bn.VolumeRenderer(d, color_format="float4")
    try:
        r.set_spp(1)
        r.render()
        st = r.stats()
        assert st["error_flags"] & 1
        assert np.isfinite(r.read()).all()
    finally:
        r.close()
    ok = small_noise_scene(w=16, h=12)
    img, st = gpu_render(ok, 2)
    ref, _, _ = oracle_render(ok, 2)
    assert_bitexact(img, ref, "after capped rays")
    assert st["error_flags"] == 0


def test_injected_allocation_failures_leave_the_context_usable():
    """Host-side fault injection: a device allocation that fails as if the
    device were out of memory (error 6) leaves the object unusable but safe
    (renders and reads of a frame buffer whose resize failed are rejected),
    and the context keeps working."""
    import barney_b200 as bn
    from tests.helpers import assert_bitexact, oracle_render, small_noise_scene
    d = small_noise_scene(w=24, h=16)
    r = bn.VolumeRenderer(d)
    L = r.L
    try:
        L.bnClearLastError()
        L.bnxInjectAllocationFailure(0)  # the next allocation fails
        L.bnFrameBufferResize(r.fb, bn.BN_FLOAT4, 25, 16, 1)
        assert L.bnGetLastError() == 6
        L.bnClearLastError()
        L.bnRender(r.renderer, r.model, r.camera, r.fb)  # not resized: rejected, nothing launched
        assert L.bnGetLastError() == 5
        L.bnClearLastError()
        L.bnxInjectAllocationFailure(1)  # the accumulation buffer succeeds, the colour buffer fails
        L.bnFrameBufferResize(r.fb, bn.BN_FLOAT4, 26, 16, 1)
        assert L.bnGetLastError() == 6
        L.bnClearLastError()
        out = np.zeros((16, 24, 4), np.float32)
        L.bnFrameBufferRead(r.fb, 1, out.ctypes.data, bn.BN_FLOAT4)
        assert L.bnGetLastError() == 5
        L.bnClearLastError()
        L.bnFrameBufferResize(r.fb, bn.BN_FLOAT4, 24, 16, 1)  # no injection left: works
        assert L.bnGetLastError() == 0
        r.set_spp(2)
        r.render()
        ref, _, _ = oracle_render(d, 2)
        assert_bitexact(r.read(), ref, "after failed resizes")
        # a texture that cannot be allocated: NULL and error 6
        L.bnxInjectAllocationFailure(0)
        vox = np.ascontiguousarray(d["voxels"])
        nz, ny, nx = vox.shape
        assert not L.bnTextureData3DCreate(r.ctx, 0, bn.BN_FLOAT32, nx, ny, nz, vox.ctypes.data)
        assert L.bnGetLastError() == 6
        L.bnClearLastError()
        r.accum_reset()
        r.render()
        assert_bitexact(r.read(), ref, "after a failed texture")
    finally:
        L.bnxInjectAllocationFailure(-1)
        r.close()
