"""Continuous-batching server: every request's frame is identical whether it
is rendered alone or in the mix with other requests (bit-exact, against the
oracle and against a solo bnRender), requests are admitted by HBM budget, and
a request that can never fit is rejected with an error."""
import time

import numpy as np
import pytest

from barney_b200 import synth
from tests.helpers import assert_bitexact, oracle_render, small_blob_scene, small_noise_scene

pytestmark = pytest.mark.gpu


def _setup(budget, slots, slice_waves, slice_pixel_waves=0):
    import barney_b200 as bn
    ctx = bn.Context()
    scenes = [small_noise_scene(n=40, w=48, h=32), small_blob_scene(n=24, w=40, h=36),
              small_noise_scene(n=33, w=37, h=29, dtype="u8", phase="simple"),
              small_noise_scene(n=24, w=16, h=16, dtype="f16", compensated_accum=True)]
    rs = [bn.VolumeRenderer(d, context=ctx, color_format="float4") for d in scenes]
    server = bn.Server(ctx, hbm_budget_bytes=budget, max_slots=slots, slice_waves=slice_waves,
                       slice_pixel_waves=slice_pixel_waves)
    return bn, ctx, scenes, rs, server


def _expected(scene, cam, w, h, spp):
    d = dict(scene, camera=cam, width=w, height=h)
    if not d.get("compensated_accum"):
        ref, _, _ = oracle_render(d, spp)
        return ref
    import oracle
    sc = oracle.Scene(d)
    acc = np.zeros((h, w, 4), np.float32)
    comp = np.zeros_like(acc)
    oracle.render(sc, 0, spp, accum=acc, comp=comp)
    return oracle.resolve(acc, spp, comp=comp)


@pytest.mark.parametrize("budget,slots,slice_waves,slice_pixel_waves",
                         [(1 << 30, 8, 2, 0), (60000, 4, 1, 0), (1 << 30, 64, 16, 0), (1 << 30, 64, 4, 3000)])
def test_mixed_requests_equal_solo_renders(budget, slots, slice_waves, slice_pixel_waves):
    """(the last setting caps a launch at 3000 pixel-waves: most requests wait
    out some launches, and their frames are still exact)"""
    bn, ctx, scenes, rs, server = _setup(budget, slots, slice_waves, slice_pixel_waves)
    try:
        rng = np.random.default_rng(5)
        reqs = []
        for i in range(20):
            k = i % len(scenes)
            spp = int(rng.integers(1, 7))
            w, h = 24 + 8 * (i % 4), 16 + 4 * (i % 3)
            cam = synth.orbit_camera(rng)
            reqs.append((server.submit(rs[k], cam, w, h, spp, "float4"), k, cam, w, h, spp))
            time.sleep(float(rng.exponential(0.001)))
        for rid, k, cam, w, h, spp in reqs:
            out = np.zeros((h, w, 4), np.float32)
            assert server.wait(rid, out, timeout_ms=60000)
            assert_bitexact(out, _expected(scenes[k], cam, w, h, spp), f"request {rid}")
        st = server.stats()
        assert st["completed"] == 20 and st["rejected"] == 0
        assert st["p50Ms"] > 0 and st["p99Ms"] >= st["p50Ms"]
        assert st["peakBytes"] <= budget
    finally:
        server.close()
        for r in rs:
            r.close()
        ctx.close()


def test_request_beyond_budget_is_rejected_and_solo_render_matches():
    bn, ctx, scenes, rs, server = _setup(50000, 4, 4)
    try:
        cam = synth.DEFAULT_CAMERA
        big = server.submit(rs[0], cam, 200, 200, 2, "float4")  # 200*200*20 B > 50 kB budget
        small = server.submit(rs[0], cam, 24, 16, 3, "float4")
        with pytest.raises(bn.BarneyError):
            server.wait(big, np.zeros((200, 200, 4), np.float32), timeout_ms=60000)
        out = np.zeros((16, 24, 4), np.float32)
        assert server.wait(small, out, timeout_ms=60000)
        solo = bn.VolumeRenderer(dict(scenes[0], camera=cam, width=24, height=16), color_format="float4")
        solo.set_spp(3)
        solo.render()
        assert_bitexact(out, solo.read(), "server vs bnRender")
        solo.close()
        assert server.stats()["rejected"] == 1
    finally:
        server.close()
        for r in rs:
            r.close()
        ctx.close()


def test_reserved_buffers_serve_identical_frames():
    bn, ctx, scenes, rs, server = _setup(1 << 30, 8, 2)
    try:
        with pytest.raises(bn.BarneyError):
            server.reserve(2 << 30)  # beyond the budget
        server.reserve(300 << 20)  # two 256 MiB chunks
        rng = np.random.default_rng(11)
        reqs = []
        for i in range(8):
            k = i % len(scenes)
            cam = synth.orbit_camera(rng)
            w, h, spp = 20 + 4 * i, 18, 1 + i % 3
            reqs.append((server.submit(rs[k], cam, w, h, spp, "float4"), k, cam, w, h, spp))
        for rid, k, cam, w, h, spp in reqs:
            out = np.zeros((h, w, 4), np.float32)
            assert server.wait(rid, out, timeout_ms=60000)
            assert_bitexact(out, _expected(scenes[k], cam, w, h, spp), f"request {rid}")
        assert server.stats()["completed"] == 8
    finally:
        server.close()
        for r in rs:
            r.close()
        ctx.close()


def test_extended_requests_in_the_server_equal_the_oracle():
    # multi-scatter, principled, exact-log and isosurface requests run the
    # extended batch kernels beside plain ones; each frame still equals the oracle's
    import barney_b200 as bn
    ctx = bn.Context()
    scenes = [small_noise_scene(n=24, w=24, h=16, anisotropy=0.6, max_volume_bounces=3),
              small_noise_scene(n=24, w=20, h=18, principled={"enabled": 1, "emission_strength": 1.0}),
              small_noise_scene(n=24, w=16, h=16, dtype="u8", exact_log=True),
              small_blob_scene(n=20, w=24, h=20),
              small_noise_scene(n=24, w=20, h=16, iso={"value": 0.5}),
              small_blob_scene(n=20, w=16, h=20, volume=False, iso={"value": 0.3, "opacity": 0.7})]
    rs = [bn.VolumeRenderer(d, context=ctx, color_format="float4") for d in scenes]
    server = bn.Server(ctx, hbm_budget_bytes=1 << 30, max_slots=8, slice_waves=2)
    try:
        rng = np.random.default_rng(17)
        reqs = []
        for i in range(18):
            k = i % len(scenes)
            cam = synth.orbit_camera(rng)
            w, h, spp = scenes[k]["width"], scenes[k]["height"], 1 + i % 4
            reqs.append((server.submit(rs[k], cam, w, h, spp, "float4"), k, cam, w, h, spp))
        for rid, k, cam, w, h, spp in reqs:
            out = np.zeros((h, w, 4), np.float32)
            assert server.wait(rid, out, timeout_ms=60000)
            assert_bitexact(out, _expected(scenes[k], cam, w, h, spp), f"request {rid}")
    finally:
        server.close()
        for r in rs:
            r.close()
        ctx.close()


def test_malformed_dropped_and_failed_requests_leave_the_server_serving():
    """Serving-queue stress on the host side: malformed requests are refused at
    submit, requests never waited for are dropped with the server, and a request
    whose buffers cannot be allocated (injected failure) fails alone; every
    other request still returns the oracle's frame."""
    bn, ctx, scenes, rs, server = _setup(1 << 30, 8, 2)
    L = ctx.L
    try:
        cam = synth.DEFAULT_CAMERA
        for bad in ((0, 16, 1, "float4"), (16, 16, 0, "float4"), (70000, 70000, 1, "float4")):
            with pytest.raises(bn.BarneyError):
                server.submit(rs[0], cam, *bad)
        L.bnClearLastError()
        # the next device allocation (this request's buffers) fails as out of memory
        L.bnxInjectAllocationFailure(0)
        failing = server.submit(rs[1], cam, 40, 36, 2, "float4")
        with pytest.raises(bn.BarneyError):
            server.wait(failing, np.zeros((36, 40, 4), np.float32), timeout_ms=60000)
        L.bnxInjectAllocationFailure(-1)
        rng = np.random.default_rng(5)
        reqs = []
        for i in range(12):
            k = i % len(scenes)
            c = synth.orbit_camera(rng)
            w, h, spp = scenes[k]["width"], scenes[k]["height"], 1 + i % 3
            reqs.append((server.submit(rs[k], c, w, h, spp, "float4"), k, c, w, h, spp))
        for rid, k, c, w, h, spp in reqs[::2]:  # every other request is never waited for
            out = np.zeros((h, w, 4), np.float32)
            assert server.wait(rid, out, timeout_ms=60000)
            assert_bitexact(out, _expected(scenes[k], c, w, h, spp), f"request {rid}")
    finally:
        L.bnxInjectAllocationFailure(-1)
        server.close()  # drops the requests nobody waited for
        for r in rs:
            r.close()
        ctx.close()
