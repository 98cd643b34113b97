"""The bounds-checked build (libbarney_b200_bc.so, -DBNB_BOUNDS_CHECK): every
indexed access of the render and macrocell kernels is checked against its
array; on small and ragged volumes of every storage type, with isosurfaces,
multi-scatter paths, batches and accumulation, it counts no out-of-range
access and renders exactly the oracle's frames.  It runs in a child process,
since a process loads one build of the library."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import numpy as np
import barney_b200 as bn
from barney_b200 import synth
from tests.helpers import assert_bitexact, oracle_render, small_blob_scene, small_noise_scene

scenes = [
    small_noise_scene(n=8, w=19, h=13),
    small_noise_scene(n=13, w=23, h=17, dtype="u8", phase="simple"),
    small_noise_scene(n=21, w=16, h=16, dtype="f16", max_volume_bounces=3, anisotropy=0.5),
    small_noise_scene(n=32, w=24, h=20, dtype="u16", iso={"value": 0.5, "opacity": 0.8}),
    small_noise_scene(n=17, w=21, h=15, dtype="bf16", cut_plane=(0.0, 1.0, 0.0, -0.4)),
    small_blob_scene(n=9, w=17, h=11, volume=False, iso={"value": 0.2}),
    small_blob_scene(n=24, w=31, h=7, compensated_accum=False, principled={"enabled": 1}, phase="hg",
                     max_volume_bounces=2),
]
ragged = synth.value_noise(21, 3)[:, 2:15, 4:13].copy()
scenes.append(dict(synth.config2(vol=ragged, width=15, height=11), spacing=(1 / 8, 1 / 12, 1 / 20)))
ctx = bn.Context()
assert ctx.L.bnxBoundsViolations(ctx.ctx) == 0, "bounds-checked build expected"
for i, d in enumerate(scenes):
    r = bn.VolumeRenderer(d, color_format="float4", context=ctx)
    r.set_spp(3)
    r.render()
    r.render()  # a second launch accumulates (reads the accumulation buffer)
    ref, _, _ = oracle_render(d, 6)
    assert_bitexact(r.read(), ref, f"scene {i}")
    r.close()
rs = [bn.VolumeRenderer(d, color_format="float4", context=ctx) for d in scenes[:4]]
for r in rs:
    r.set_spp(2)
ctx.render_batch(rs)
for r, d in zip(rs, scenes[:4]):
    ref, _, _ = oracle_render(d, 2)
    assert_bitexact(r.read(), ref, "batch")
    r.close()
n = ctx.L.bnxBoundsViolations(ctx.ctx)
ctx.close()
assert n == 0, f"{n} out-of-range accesses"
print("bounds-checked build: 0 out-of-range accesses")
"""


def test_bounds_checked_build_counts_no_out_of_range_access():
    from barney_b200 import build as _build
    lib = _build.build(bounds_check=True)
    env = dict(os.environ, BARNEY_B200_LIBRARY=lib, PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
    r = subprocess.run([sys.executable, "-c", CHILD], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "0 out-of-range accesses" in r.stdout
