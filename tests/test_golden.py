"""Committed fixtures (tests/golden/*.npz, made by make_golden.py) are
reproduced bit-exactly by the CPU oracle and by the CUDA path."""
import os

import numpy as np
import pytest

import oracle
from tests.helpers import assert_bitexact

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = ["noise_f32", "noise_u8", "noise_f16", "blobs_ambient", "blobs_ea", "noise_multiscatter",
         "noise_principled", "noise_exact_log", "blobs_iso", "noise_iso", "noise_iso_multiscatter"]


def _scene(name):
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg.scenes()[name]


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_fixture(name):
    g = np.load(os.path.join(HERE, name + ".npz"))
    d = _scene(name)
    sc = oracle.Scene(d)
    r = oracle.build_ranges(sc)
    assert_bitexact(r, g["ranges"], "ranges")
    assert_bitexact(oracle.map_majorants(sc, r), g["majorants"], "majorants")
    s, rgba = oracle.sample_points(sc, g["points"])
    assert_bitexact(s, g["point_scalar"], "samples")
    assert_bitexact(rgba, g["point_rgba"], "tf")
    for spp in (1, 3):
        acc, _, st = oracle.render(sc, 0, spp, threads=2)
        assert_bitexact(acc, g[f"accum_spp{spp}"], f"accum spp={spp}")
        assert [st["samples"], st["mc_visits"], st["rays"]] == g[f"counts_spp{spp}"].tolist()


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_gpu_reproduces_fixture(name):
    import barney_b200 as bn
    g = np.load(os.path.join(HERE, name + ".npz"))
    d = _scene(name)
    r = bn.VolumeRenderer(d, color_format="float4")
    try:
        if d.get("volume", True):  # an isosurface alone has no volume to query
            ranges, maj = r.macrocells()
            assert_bitexact(ranges, g["ranges"], "ranges")
            assert_bitexact(maj, g["majorants"], "majorants")
        for spp in (1, 3):
            r.accum_reset()
            r.set_spp(spp)
            r.render()
            assert_bitexact(r.read(), g[f"frame_spp{spp}"], f"frame spp={spp}")
            st = r.stats()
            assert [st["samples"], st["mc_visits"], st["rays"]] == g[f"counts_spp{spp}"].tolist()
    finally:
        r.close()
