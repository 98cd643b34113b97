"""The CPU oracle against golden vectors produced by the REFERENCE'S OWN code.

tests/golden/ref_*.npz come from the reference's sources compiled here
(oracle/Makefile target `ref`, generator tests/golden/make_ref_golden.py):
barney-common.h (RNG, hash), Volume.h (fastLog, Woodcock::sampleRange,
sampleAndMap), DDA.h (dda3), TransferFunction.h (map, majorant),
PrincipledVolume.h, math.h (linear_to_srgb, make_rgba) and the CPU
backend's Texture.cpp (NEAREST / LINEAR tex3D) and Float16.cpp.  Every
comparison is bit-exact.
"""
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def bits(a):
    a = np.ascontiguousarray(a, np.float32)
    return a.view(np.uint32)


def assert_same(a, b, what):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    if a.dtype == np.float32 or b.dtype == np.float32:
        a, b = bits(a), bits(b)
    bad = np.flatnonzero(a.reshape(-1) != b.reshape(-1))
    assert bad.size == 0, f"{what}: {bad.size} of {a.size} differ, first at {bad[:5].tolist()}"


def scene_from(z, prefix, **over):
    """Scene description from a fixture's stored inputs."""
    g = lambda k: z[prefix + k]  # noqa: E731
    d = {"voxels": g("voxels"), "dtype": str(g("dtype")), "spacing": tuple(float(v) for v in g("spacing")),
         "origin": tuple(float(v) for v in g("origin")), "tf": g("tf"),
         "domain": tuple(float(v) for v in g("domain")), "density": float(g("density")),
         "camera": {"position": tuple(float(v) for v in g("cam_position")),
                    "direction": tuple(float(v) for v in g("cam_direction")),
                    "up": tuple(float(v) for v in g("cam_up")), "fovy": float(g("cam_fovy"))},
         "width": int(g("width")), "height": int(g("height"))}
    d.update(over)
    return d


def test_rng_hash():
    z = load("ref_rng.npz")
    for i, (a, b) in enumerate(z["seeds"]):
        assert_same(oracle.rng_stream(int(a), int(b), 64), z["streams"][i], f"Random2({a},{b}) stream")
        assert_same(oracle.rng_floats(int(a), int(b), 64), z["floats"][i], f"Random2({a},{b}) floats")
    for i, (p, h) in enumerate(zip(z["parents"], z["hashes"])):
        out, parent = oracle.rng_derived(int(p), int(h), 16)
        assert_same(out, z["derived"][i], f"Random2(seed {p:#x}, {h:#x})")
        assert parent == int(z["parent_after"][i])
    for (a, b, c), h in zip(z["triples"], z["hash3"]):
        assert oracle.hash3(int(a), int(b), int(c)) == int(h)


def test_fastlog_half_resolve():
    z = load("ref_scalar.npz")
    got = np.array([oracle.fastlog(float(x)) for x in z["log_x"]], np.float32)
    assert_same(got, z["fastlog"], "fastLog")
    # binary16 rounding of path throughputs: the reference's CPU backend
    # rounds an exact tie up in magnitude (Float16.cpp:73-76,125-131), its
    # CUDA backend (cuda_fp16's float-to-half) to nearest even, which the
    # oracle and the kernels follow.  Away from ties the two agree.
    x = z["half_x"]
    got = np.array([oracle.f2h(float(v)) for v in x], np.uint16)
    xb = x.view(np.uint32)
    exp = ((xb >> 23) & 0xff).astype(np.int64) - 112
    normal_tie = (exp > 0) & (exp < 31) & ((xb & 0x1fff) == 0x1000)
    assert normal_tie.sum() >= 2
    assert_same(got[~normal_tie], z["half_bits"][~normal_tie], "float32ToFloat16 away from ties")
    ref_t, got_t = z["half_bits"][normal_tie].astype(np.int64), got[normal_tie].astype(np.int64)
    assert np.all(np.isin(ref_t - got_t, (0, 1)))
    assert np.all(got_t % 2 == 0), "ties round to an even significand"
    assert np.all(ref_t == (xb[normal_tie] >> 16 & 0x8000) | ((exp[normal_tie] << 10) +
                  ((xb[normal_tie] & 0x7fffff) >> 13) + 1)), "the reference's CPU backend rounds ties up"
    got = np.array([oracle.lib().orc_h2f(int(h)) for h in range(65536)], np.float32)
    nan = np.isnan(z["h2f"])  # NaN codes: NaN on both sides, payloads not compared
    assert np.array_equal(np.isnan(got), nan) and nan.sum() == 2046
    assert_same(got[~nan], z["h2f"][~nan], "float16ToFloat32")
    # make_rgba through the resolve (accumID 1: a scale of exactly 1)
    rgba = z["rgba"].reshape(-1, 1, 4)
    assert_same(oracle.resolve(rgba, 1, "rgba8").reshape(-1), z["make_rgba"], "make_rgba")
    # linear_to_srgb: the sRGB resolve's bytes equal make_8bit of the reference's values
    x = z["srgb_x"]
    acc = np.stack([x, x, x, np.ones_like(x)], -1).reshape(-1, 1, 4).astype(np.float32)
    s = z["srgb"]
    want = np.stack([s, s, s, np.ones_like(s)], -1).astype(np.float32)
    b8 = np.clip((want * np.float32(256.0)).astype(np.int64), 0, 255).astype(np.uint32)
    want_px = b8[:, 0] | (b8[:, 1] << 8) | (b8[:, 2] << 16) | (b8[:, 3] << 24)
    assert_same(oracle.resolve(acc, 1, "rgba8_srgb").reshape(-1), want_px, "linear_to_srgb + make_rgba")


@pytest.mark.parametrize("name", ["linear128", "knots256", "odd7"])
def test_transfer_function(name):
    z = load("ref_tf.npz")
    d = {"voxels": np.zeros((2, 2, 2), np.float32), "dtype": "f32", "spacing": (1.0, 1.0, 1.0),
         "tf": z[f"{name}_tf"], "domain": tuple(float(v) for v in z[f"{name}_domain"]),
         "density": float(z[f"{name}_density"]),
         "camera": {"position": (2, 2, 2), "direction": (-1, -1, -1)}, "width": 4, "height": 4}
    sc = oracle.Scene(d)
    assert_same(oracle.tf_map(sc, z[f"{name}_v"]), z[f"{name}_map"], f"{name}: TF map")
    assert_same(oracle.map_majorants(sc, z[f"{name}_ranges"]), z[f"{name}_majorants"], f"{name}: TF majorant")


FIELD_NAMES = ["ragged_f32", "ragged_u8", "blobs24_f32", "noise40_u8", "noise_ragged_f32", "principled17_f32"]


def field_scene(z, name):
    over = {}
    if f"{name}__principled_params" in z.files:
        import ast
        over["principled"] = ast.literal_eval(str(z[f"{name}__principled_params"]))
    return scene_from(z, name + "__", **over)


@pytest.mark.parametrize("name", FIELD_NAMES)
def test_field_sampling_and_macrocells(name):
    z = load("ref_field.npz")
    d = field_scene(z, name)
    sc = oracle.Scene(d)
    p = name + "__"
    assert_same(oracle.tex3d(sc, z[p + "tc"]), z[p + "tex_linear"], f"{name}: LINEAR tex3D")
    # NEAREST at integer texel coordinates inside the grid is the voxel itself
    # (the macrocell build reads voxels directly)
    tc = z[p + "tc"]
    vol = z[p + "voxels"]
    nz, ny, nx = vol.shape
    integ = np.all(tc == np.floor(tc), axis=1) & np.all(tc >= 0, axis=1) & (tc[:, 0] < nx) & (tc[:, 1] < ny) & \
        (tc[:, 2] < nz)
    assert integ.sum() > 0
    ii = tc[integ].astype(np.int64)
    direct = vol[ii[:, 2], ii[:, 1], ii[:, 0]]
    direct = direct.astype(np.float32) * np.float32(1.0) / np.float32(255.0) if vol.dtype == np.uint8 else direct
    assert_same(direct.astype(np.float32), z[p + "tex_nearest"][integ], f"{name}: NEAREST tex3D at voxels")
    scal, rgba = oracle.sample_points(sc, z[p + "P"])
    assert_same(scal, z[p + "sample"], f"{name}: structured sampler")
    assert_same(rgba, z[p + "sample_rgba"], f"{name}: sampleAndMap")
    ranges = oracle.build_ranges(sc)
    assert_same(ranges, z[p + "ranges"], f"{name}: macrocell ranges")
    assert_same(oracle.map_majorants(sc, ranges), z[p + "majorants"], f"{name}: majorants")
    if p + "principled_v" in z.files:
        m, e = oracle.principled(sc, z[p + "principled_v"])
        assert_same(m, z[p + "principled_map"], f"{name}: principledSampleMap")
        assert_same(e, z[p + "principled_emission"], f"{name}: principledEmission")


def test_dda():
    z = load("ref_dda.npz")
    for i in range(z["org"].shape[0]):
        c, t = oracle.dda_cells(z["org"][i], z["dir"][i], float(z["tmax"][i]), z["grid"], 64)
        n = int(z["counts"][i])
        assert len(c) == n, (i, len(c), n)
        assert_same(c, z["cells"][i, :n], f"ray {i}: cells")
        assert_same(t, z["ts"][i, :n], f"ray {i}: cell t ranges")


TRACE_NAMES = ["blobs32_f32", "noise40_u8", "axis_aligned_f32", "camera_inside_f32", "ragged_f32"]


def trace_scene(z, name, **over):
    return scene_from(z, name + "__", **over)


@pytest.mark.parametrize("name", TRACE_NAMES)
def test_primary_first_collisions(name):
    """Every pixel's primary ray: hit, distance and TF colour at the first
    Woodcock collision, as the reference's own traversal finds them; and the
    work counted (samples, macrocell visits) through the oracle's render."""
    z = load("ref_trace.npz")
    p = name + "__"
    d = trace_scene(z, name)
    sc = oracle.Scene(d)
    W, H = d["width"], d["height"]
    for a in z[p + "accum_ids"]:
        a = int(a)
        hit, t, rgb = z[f"{p}hit{a}"], z[f"{p}t{a}"], z[f"{p}rgb{a}"]
        for iy in range(H):
            for ix in range(W):
                h, tt, c = oracle.trace_primary(sc, ix, iy, a)
                assert h == bool(hit[iy, ix]), (name, a, ix, iy)
                if h:
                    assert_same(np.float32(tt), t[iy, ix], f"{name} accumID {a} pixel ({ix},{iy}) t")
                    assert_same(c, rgb[iy, ix], f"{name} accumID {a} pixel ({ix},{iy}) rgb")
        # emission-absorption renders trace primary rays only: their work
        # counters are the per-pixel sums of the reference's
        ea = oracle.Scene(dict(d, emission_absorption=True, ambient=0.0))
        _, _, st = oracle.render(ea, a, 1)
        cnt = z[f"{p}counts{a}"]
        assert st["samples"] == int(cnt[..., 0].sum()), (name, a)
        assert st["mc_visits"] == int(cnt[..., 1].sum()), (name, a)
    # explicit rays with explicit RNG states
    for i in range(z[p + "ray_org"].shape[0]):
        h, tt, c, cnt = oracle.trace_ray(sc, z[p + "ray_org"][i], z[p + "ray_dir"][i], float(z[p + "ray_tmax"][i]),
                                         int(z[p + "ray_seed"][i]))
        assert h == bool(z[p + "ray_hit"][i]), (name, i)
        assert_same(cnt, z[p + "ray_counts"][i], f"{name} ray {i} counts")
        if h:
            assert_same(np.float32(tt), z[p + "ray_t"][i], f"{name} ray {i} t")
            assert_same(c, z[p + "ray_rgb"][i], f"{name} ray {i} rgb")
