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
    big = synth.config2(n=96, width=1920, height=1080, spp=256)  # a frame of ~100 ms
    r = bn.VolumeRenderer(big, color_format="rgba8")
    try:
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
