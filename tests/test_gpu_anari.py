"""The ANARI front-end over the native API: the renderer's commit
(bnxAnariRendererCommit, barney/anari/Renderer.cpp:22-51) and a frame that
starts its accumulation over after any commit (bnxAnariRenderFrame,
barney/anari/Frame.cpp:172-178), checked bit-exact against the CPU oracle."""
import pytest

from tests.helpers import assert_bitexact, oracle_render, small_blob_scene, small_noise_scene

pytestmark = pytest.mark.gpu


def _renderer(d):
    import barney_b200 as bn
    return bn.VolumeRenderer(d)


def test_committed_parameters_render_like_the_oracle():
    d = small_noise_scene(w=40, h=28)
    r = _renderer(d)
    try:
        r.anari_commit_renderer(pixelSamples=3, ambientRadiance=0.5, background=(0.2, 0.3, 0.4, 1.0),
                                cutPlane=(1.0, 0.0, 0.0, -0.55))
        r.render()
        img = r.read()
    finally:
        r.close()
    ref, _, _ = oracle_render(dict(d, ambient=0.5, bg_color=(0.2, 0.3, 0.4, 1.0), cut_plane=(1.0, 0.0, 0.0, -0.55)), 3)
    assert_bitexact(img, ref, "ANARI renderer commit")


def test_parameters_left_unset_take_the_anari_defaults():
    # one path per pixel, ambient 1, black background, cut plane (0,0,0,0):
    # a zero normal clips nothing
    d = small_blob_scene(w=36, h=30, ambient=0.3, bg_color=(0.5, 0.5, 0.5, 1.0))
    r = _renderer(d)
    try:
        r.set_spp(7)
        r.anari_commit_renderer()
        r.render()
        img = r.read()
    finally:
        r.close()
    ref, _, _ = oracle_render(dict(d, ambient=1.0, bg_color=(0.0, 0.0, 0.0, 1.0), cut_plane=(0.0, 0.0, 0.0, 0.0)), 1)
    assert_bitexact(img, ref, "ANARI renderer defaults")


def test_frames_accumulate_until_something_is_committed():
    from barney_b200 import synth
    d = small_blob_scene(w=32, h=24)
    moved = dict(d, camera=synth.look_at((1.8, 1.2, 2.3)))
    r = _renderer(d)
    try:
        r.anari_commit_renderer(pixelSamples=2)
        r.anari_render_frame()
        r.anari_render_frame()  # nothing committed in between: 4 paths per pixel
        first = r.read().copy()
        r.set_camera(moved["camera"])  # a commit: the next frame starts over
        r.anari_render_frame()
        restarted = r.read().copy()
        r.anari_render_frame()
        continued = r.read().copy()
    finally:
        r.close()
    assert_bitexact(first, oracle_render(d, 4)[0], "two frames accumulated")
    assert_bitexact(restarted, oracle_render(moved, 2)[0], "first frame after the commit")
    assert_bitexact(continued, oracle_render(moved, 4)[0], "second frame after the commit")
