"""Known-answer tests pinning the CPU oracle (oracle/bn_oracle.cpp).

The reference ships no golden vectors for the structured-volume path, so
each expected value here is derived independently: the RNG and hash are
restated a second time in Python integers from barney-common.h:21-108;
fastLog, trilinear sampling and the transfer function are re-evaluated
with numpy float32 scalars in the reference's operation order; DDA cell
sequences are worked out by hand from DDA.h:61-201.
"""
import math

import numpy as np
import pytest

import oracle

M64 = (1 << 64) - 1
M32 = (1 << 32) - 1
f32 = np.float32


def py_next(state):
    x = state
    count = x >> 61
    state = (x * 6364136223846793005) & M64
    x ^= x >> 22
    return state, (x >> (22 + count)) & M32


def py_seed(a, b):
    st = 0xcafef00dd15ea5e5
    st ^= (2 * a + 1) & M32
    st, _ = py_next(st)
    st ^= (2 * b) & M32
    st, _ = py_next(st)
    return st


def test_rng_stream_matches_python_restatement():
    for a, b in [(0, 0), (1, 2), (1919, 1079), (0xFFFFFFFF, 7), (123456, 654321)]:
        st = py_seed(a, b)
        expect = []
        for _ in range(32):
            st, v = py_next(st)
            expect.append(v)
        assert list(oracle.rng_stream(a, b, 32)) == expect


def test_rng_float_is_24bit_uniform():
    st = py_seed(5, 9)
    vals = oracle.rng_floats(5, 9, 64)
    for v in vals:
        st, u = py_next(st)
        assert v == f32((u & 0xFFFFFF)) * f32(1.0 / 16777216.0)
    assert vals.min() >= 0.0 and vals.max() < 1.0


def test_rng_derived_stream():
    # Random2(RNGSeed &seed, b): child = parent; parent.next(); child.next(b ? b : 290374)
    parent = py_seed(3, 4)
    for h in [0, 1, 0x3f800000, oracle.hash3(0, 0, 0)]:
        child = parent ^ (((h if h else 290374) << 1) & M64)
        child, _ = py_next(child)
        exp = []
        for _ in range(8):
            child, v = py_next(child)
            exp.append(v)
        got, parent_after = oracle.rng_derived(parent, h, 8)
        assert list(got) == exp
        assert parent_after == (parent * 6364136223846793005) & M64


def test_hash_fnv():
    basis, prime = 0xcbf29ce484222325, 0x100000001b3
    def h1(v): return basis ^ ((prime * v) & M64)
    def h2(h, v): return ((h * prime) & M64) ^ v
    for a, b, c in [(0, 0, 0), (1, 2, 3), (7, 0, 9)]:
        assert oracle.hash3(a, b, c) == h2(h2(h1(a), b), c)


def test_fastlog_series():
    for x in [1.0, 0.5, 0.25, 1e-3, 0.999, 2.0 ** -24, 0.75]:
        f = f32(x)
        g = (f - f32(1)) / (f + f32(1))
        g2 = g * g
        s = g
        g = g * g2
        s = s + f32(1.0 / 3.0) * g
        g = g * g2
        s = s + f32(1.0 / 5.0) * g
        assert oracle.fastlog(float(f)) == s + s
    # the series is biased: at 2^-24 it returns ~ -3.07 instead of -16.6
    assert -3.1 < oracle.fastlog(2.0 ** -24) < -3.0


@pytest.mark.filterwarnings("ignore::RuntimeWarning")
def test_float_to_half_round_nearest_even():
    rng = np.random.default_rng(0)
    vals = np.concatenate([
        rng.standard_normal(2000).astype(np.float32) * 10,
        np.array([0.0, -0.0, 65504.0, 65519.99, 65520.0, 1e-8, 6e-8, 5.96e-8, 2.98e-8, 1e5,
                  1.0 + 2.0 ** -11, 1.0 + 3 * 2.0 ** -11, np.inf, -np.inf], np.float32),
        (rng.random(2000) * 1e-4).astype(np.float32)])
    for v in vals:
        assert oracle.f2h(float(v)) == int(np.array(v, np.float32).astype(np.float16).view(np.uint16))


def test_dda_axis_aligned():
    cells, ts = oracle.dda_cells((-1.0, 0.5, 0.5), (1.0, 0.0, 0.0), 1e30, (4, 4, 4))
    assert cells.tolist() == [[0, 0, 0], [1, 0, 0], [2, 0, 0], [3, 0, 0]]
    assert ts.tolist() == [[1, 2], [2, 3], [3, 4], [4, 5]]


def test_dda_diagonal_steps_all_axes_at_once():
    cells, ts = oracle.dda_cells((-1.0, -1.0, -1.0), (1.0, 1.0, 1.0), 1e30, (2, 2, 2))
    assert cells.tolist() == [[0, 0, 0], [1, 1, 1]]
    assert ts.tolist() == [[1, 2], [2, 3]]


def test_dda_tmax_quirk_keeps_walking():
    # DDA.h:175 clamps cell_t1 to ray_t0 + tMax and never stops at tMax
    cells, ts = oracle.dda_cells((-1.0, 0.5, 0.5), (1.0, 0.0, 0.0), 1.5, (4, 4, 4))
    assert cells.tolist() == [[0, 0, 0], [1, 0, 0], [2, 0, 0], [3, 0, 0]]
    assert ts.tolist() == [[1, 2], [2, 2.5], [3, 2.5], [4, 2.5]]


def test_dda_negative_direction_and_miss():
    cells, _ = oracle.dda_cells((3.5, 0.5, 0.5), (-1.0, 0.0, 0.0), 1e30, (4, 4, 4))
    assert cells.tolist() == [[3, 0, 0], [2, 0, 0], [1, 0, 0], [0, 0, 0]]
    cells, _ = oracle.dda_cells((0.5, 5.0, 0.5), (1.0, 0.0, 0.0), 1e30, (4, 4, 4))
    assert len(cells) == 0


def _tiny_scene(vol, dtype="f32", tf=None, **kw):
    if tf is None:
        tf = np.array([[0, 0, 1, 0], [1, 0, 0, 1]], np.float32)
    d = {"voxels": vol, "dtype": dtype, "spacing": (1.0, 1.0, 1.0), "tf": tf, "density": 2.0,
         "camera": {"position": (0, 0, -5), "direction": (0, 0, 1)}, "width": 4, "height": 4}
    d.update(kw)
    return oracle.Scene(d)


def _trilinear_ref(v, fx, fy, fz, i):
    x0, x1, y0, y1, z0, z1 = i
    lerp = lambda f, a, b: (f32(1) - f) * a + f * b
    c00 = lerp(fx, v[z0, y0, x0], v[z0, y0, x1])
    c01 = lerp(fx, v[z0, y1, x0], v[z0, y1, x1])
    c10 = lerp(fx, v[z1, y0, x0], v[z1, y0, x1])
    c11 = lerp(fx, v[z1, y1, x0], v[z1, y1, x1])
    return lerp(fz, lerp(fy, c00, c01), lerp(fy, c10, c11))


def test_trilinear_interior_edges_and_outside():
    rng = np.random.default_rng(1)
    vol = rng.random((3, 4, 5)).astype(np.float32)
    sc = _tiny_scene(vol)
    P = np.array([[0.25, 0.5, 0.75], [0.0, 0.0, 0.0], [3.5, 2.25, 1.5], [4.0, 0.0, 0.0],
                  [-1e-7, 0.0, 0.0], [1.0, 1.0, 1.0], [np.nextafter(np.float32(4), 0), 0.5, 0.5]], np.float32)
    scal, _ = oracle.sample_points(sc, P)
    assert scal[0] == _trilinear_ref(vol, f32(0.25), f32(0.5), f32(0.75), (0, 1, 0, 1, 0, 1))
    assert scal[1] == vol[0, 0, 0]
    assert scal[2] == _trilinear_ref(vol, f32(0.5), f32(0.25), f32(0.5), (3, 4, 2, 3, 1, 2))
    assert math.isnan(scal[3]) and math.isnan(scal[4])       # rel >= numCells, rel < 0
    assert scal[5] == vol[1, 1, 1]
    # rel = 4 - ulp: rel + .5 rounds to 4.5, so tc - .5 >= N - 1 clamps to x = 4
    assert scal[6] == _trilinear_ref(vol, f32(0), f32(0), f32(0), (4, 4, 0, 1, 0, 1)) or \
        scal[6] == (f32(1) - f32(0.5)) * ((f32(1) - f32(0.5)) * vol[0, 0, 4] + f32(0.5) * vol[0, 1, 4]) + \
        f32(0.5) * ((f32(1) - f32(0.5)) * vol[1, 0, 4] + f32(0.5) * vol[1, 1, 4])


def test_uchar_texels_divide_by_255():
    vol = np.arange(8, dtype=np.uint8).reshape(2, 2, 2) * 30
    sc = _tiny_scene(vol, dtype="u8")
    scal, _ = oracle.sample_points(sc, np.array([[0, 0, 0], [0.999, 0, 0]], np.float32))
    assert scal[0] == f32(0) and scal[1] > 0
    sc2 = _tiny_scene(np.full((2, 2, 2), 200, np.uint8), dtype="u8")
    s2, _ = oracle.sample_points(sc2, np.array([[0.0, 0.0, 0.0], [0.3, 0.3, 0.3]], np.float32))
    c = f32(200) / f32(255)
    assert s2[0] == c
    assert s2[1] == _trilinear_ref(np.full((2, 2, 2), c, np.float32), f32(0.3), f32(0.3), f32(0.3), (0, 1, 0, 1, 0, 1))


def test_transfer_function_map():
    tf = np.array([[0, 0, 1, 0], [0.5, 0, 0.5, 0.25], [1, 0, 0, 1]], np.float32)
    sc = _tiny_scene(np.zeros((2, 2, 2), np.float32), tf=tf, domain=(0.0, 2.0))
    v = np.array([-1.0, 0.0, 0.5, 1.0, 1.5, 2.0, 3.0], np.float32)
    rgba = oracle.tf_map(sc, v)
    for s, out in zip(v, rgba):
        f = (s - f32(0)) / f32(2)
        f = min(f32(1), max(f32(0), f)) * f32(2)
        idx = min(1, max(0, int(f)))
        f = f - f32(idx)
        exp = (f32(1) - f) * tf[idx] + f * tf[idx + 1]
        exp[3] = exp[3] * f32(2.0)
        assert np.array_equal(out, exp)


def test_majorant_of_ranges():
    tf = np.array([[0, 0, 0, 0.0], [0, 0, 0, 0.8], [0, 0, 0, 0.2], [0, 0, 0, 0.4]], np.float32)
    sc = _tiny_scene(np.zeros((2, 2, 2), np.float32), tf=tf)
    ranges = np.array([[0.0, 1.0], [0.9, 1.0], [0.1, 0.2], [0.5, 0.4], [0.0, 0.0]], np.float32)
    m = oracle.map_majorants(sc, ranges)
    assert m[0] == f32(0.8) * f32(2)                       # interior knot 1 inside [0,1]
    assert m[4] == f32(0)
    assert m[3] == 0.0                                     # empty range
    f = (f32(0.9) - 0) / f32(1) * f32(3)
    lo = (f32(1) - (f - f32(2))) * f32(0.2) + (f - f32(2)) * f32(0.4)
    assert m[1] == max(f32(0), lo, f32(0.4)) * f32(2)
    fl = f32(0.1) * f32(3)
    fh = f32(0.2) * f32(3)
    e_lo = (f32(1) - fl) * f32(0) + fl * f32(0.8)
    e_hi = (f32(1) - fh) * f32(0) + fh * f32(0.8)
    assert m[2] == max(f32(0), e_lo, e_hi) * f32(2)


def test_macrocell_ranges_bruteforce():
    rng = np.random.default_rng(2)
    vol = rng.random((19, 10, 23)).astype(np.float32)  # ragged: 18 x 9 x 22 cells
    sc = _tiny_scene(vol)
    r = oracle.build_ranges(sc)
    assert r.shape == (3, 2, 3, 2)
    for z in range(3):
        for y in range(2):
            for x in range(3):
                blk = vol[8 * z:8 * z + 9, 8 * y:8 * y + 9, 8 * x:8 * x + 9]
                assert r[z, y, x, 0] == blk.min() and r[z, y, x, 1] == blk.max()


def test_compensated_accumulation_tracks_double_sum():
    """Precision form: Neumaier-compensated accumulation across waves stays at
    the double-precision sum of the same per-wave fragments, where the plain
    float sum drifts."""
    from barney_b200 import synth
    vol = synth.blobs(12, 0)
    base = synth.scene(vol, "f32", 6, 4, synth.tf_linear_ramp(32), 20.0, synth.DEFAULT_CAMERA, ambient=1.0)
    plain = oracle.Scene(dict(base))
    comp_sc = oracle.Scene(dict(base, compensated_accum=True))
    spp = 600
    acc_p, _, _ = oracle.render(plain, 0, spp, threads=1)
    acc_c = np.zeros_like(acc_p)
    cbuf = np.zeros_like(acc_p)
    oracle.render(comp_sc, 0, spp, accum=acc_c, comp=cbuf, threads=1)
    exact = np.zeros(acc_p.shape, np.float64)
    for k in range(spp):  # each wave alone onto a zero buffer = that wave's fragments
        one, _, _ = oracle.render(plain, k, 1, accum=np.zeros_like(acc_p), threads=1)
        exact += one
    err_plain = np.abs(acc_p - exact).sum()
    err_comp = np.abs(acc_c.astype(np.float64) + cbuf - exact).sum()
    assert err_comp <= err_plain
    assert err_comp < 1e-3 * max(err_plain, 1e-30) or err_comp < 1e-5


def test_unorm16_reciprocal_form_is_exact():
    """The kernels normalise unorm16 voxels as q + (x - 65535 q) / 65535 with
    q = x * (1/65535), unfused; that equals x / 65535 for every 16-bit x."""
    x = np.arange(65536, dtype=np.float32)
    r = f32(1) / f32(65535)
    q = x * r
    assert np.array_equal(q + (x - q * f32(65535)) * r, x / f32(65535))


def test_u16_texels_divide_by_65535():
    vol = (np.arange(8, dtype=np.uint16).reshape(2, 2, 2) * 9000).astype(np.uint16)
    sc = _tiny_scene(vol, dtype="u16")
    scal, _ = oracle.sample_points(sc, np.array([[0, 0, 0]], np.float32))
    assert scal[0] == f32(0)
    sc2 = _tiny_scene(np.full((2, 2, 2), 40000, np.uint16), dtype="u16")
    s2, _ = oracle.sample_points(sc2, np.array([[0.0, 0.0, 0.0]], np.float32))
    assert s2[0] == f32(40000) / f32(65535)


def test_portable_sincos_matches_float64_within_two_ulp():
    # one binary32 sin/cos shared by the oracle and the kernels (the HG
    # sampler's azimuth runs over [0, 2pi])
    x = np.linspace(0, 2 * np.pi, 100001, dtype=np.float32)
    sn, cs = oracle.sincos(x)
    x64 = x.astype(np.float64)
    assert np.abs(sn - np.sin(x64)).max() < 2.4e-7
    assert np.abs(cs - np.cos(x64)).max() < 2.4e-7
    big = np.abs(np.sin(x64)) > 0.25
    assert (np.abs(sn[big] - np.sin(x64[big])) <= 2 * np.spacing(np.abs(sn[big]))).all()
    # quadrant boundaries reduce to exact values
    s0, c0 = oracle.sincos(np.array([0.0], np.float32))
    assert s0[0] == 0.0 and c0[0] == 1.0


@pytest.mark.parametrize("g", [0.0, 0.6, -0.5, 0.9])
def test_hg_direction_sampler_has_mean_cosine_g(g):
    # Phase.h:76-101: the mean cosine of Henyey-Greenstein is g
    d = oracle.hg_sample([0.0, 0.0, 1.0], g, 0x1234567, 100000)
    assert np.abs(np.linalg.norm(d, axis=1) - 1).max() < 3e-7
    assert abs(d[:, 2].mean() - g) < 0.01
    # the sampler is symmetric about the incoming direction
    assert abs(d[:, 0].mean()) < 0.01 and abs(d[:, 1].mean()) < 0.01


def test_multi_scatter_adds_energy_and_rays():
    from tests.helpers import small_noise_scene
    d = small_noise_scene(w=24, h=16, phase="hg", anisotropy=0.6)
    means, rays = [], []
    for mvb in (0, 1, 4):
        sc = oracle.Scene(dict(d, max_volume_bounces=mvb))
        acc = np.zeros((16, 24, 4), np.float32)
        _, _, st = oracle.render(sc, 0, 32, accum=acc)
        means.append(float(oracle.resolve(acc, 32)[..., :3].mean()))
        rays.append(st["rays"])
    assert means[0] < means[1] < means[2]
    assert rays[0] < rays[1] < rays[2]
    with pytest.raises(ValueError):
        oracle.render_expected_fp64(oracle.Scene(dict(d, max_volume_bounces=1)))
    # the default build (SimplePhase) ignores maxVolumeBounces, as the reference's does
    simple = small_noise_scene(w=24, h=16, phase="simple")
    imgs = []
    for mvb in (0, 3):
        acc = np.zeros((16, 24, 4), np.float32)
        oracle.render(oracle.Scene(dict(simple, max_volume_bounces=mvb)), 0, 4, accum=acc)
        imgs.append(acc)
    assert np.array_equal(imgs[0], imgs[1])


def test_path_depth_cap_binds_before_the_bounce_budget():
    # MAX_PATH_DEPTH = 10 (shadeRays.cu:31): a hit of generation 10 does not
    # scatter, so budgets of 10 and 14 bounces give the same sums, 9 does not
    from tests.helpers import small_noise_scene
    accs = {}
    for mvb in (9, 10, 14):
        d = small_noise_scene(phase="hg", anisotropy=0.3, max_volume_bounces=mvb)
        acc = np.zeros((d["height"], d["width"], 4), np.float32)
        oracle.render(oracle.Scene(d), 0, 8, accum=acc)
        accs[mvb] = acc
    assert np.array_equal(accs[10], accs[14])
    assert not np.array_equal(accs[9], accs[10])


def test_portable_log_within_two_ulp_on_free_flight_inputs():
    # bnx.exactLog draws dt = -log(1 - r) / majorant, r a multiple of 2^-24 in [0, 1)
    r = np.arange(0, 2 ** 24, 37, dtype=np.float64) * 2.0 ** -24
    x = (1.0 - r).astype(np.float32)
    v = oracle.logp(x).astype(np.float64)
    t = np.log(x.astype(np.float64))
    ulp = np.spacing(np.abs(t).astype(np.float32)).astype(np.float64)
    nz = t != 0
    assert (np.abs(v - t)[nz] <= 2 * ulp[nz]).all()
    assert oracle.logp(np.array([1.0], np.float32))[0] == 0.0
    p2 = np.float32(2.0) ** -np.arange(1, 24, dtype=np.float32)
    assert np.allclose(oracle.logp(p2), np.log(p2.astype(np.float64)), rtol=2 ** -23, atol=0)


def test_portable_exp_within_two_ulp():
    x = np.linspace(-20, 20, 200001, dtype=np.float32)
    v = oracle.expp(x).astype(np.float64)
    t = np.exp(x.astype(np.float64))
    assert (np.abs(v - t) <= 2 * np.spacing(t.astype(np.float32))).all()
    assert oracle.expp(np.array([0.0], np.float32))[0] == 1.0


@pytest.mark.parametrize("kelvin", [500.0, 1500.0, 1900.0, 3000.0, 6500.0, 6700.0, 8000.0, 20000.0, 50000.0])
def test_blackbody_colour_matches_the_reference_formula(kelvin):
    # PrincipledVolume.h:64-82, evaluated here in float64
    k = min(max(kelvin, 1000.0), 40000.0)
    t = k / 100.0
    cl = lambda v: min(max(v, 0.0), 1.0)
    if t <= 66.0:
        r, g = 1.0, cl(0.390081578 * np.log(t) - 0.631841444)
    else:
        r = cl(1.292936186 * (t - 60.0) ** -0.1332047592)
        g = cl(1.129890860 * (t - 60.0) ** -0.0755148492)
    b = 1.0 if t >= 66.0 else (0.0 if t <= 19.0 else cl(0.543206789 * np.log(t - 10.0) - 1.196254089))
    assert np.allclose(oracle.blackbody(kelvin), [r, g, b], rtol=0, atol=2e-6)


def test_principled_volume_emission_adds_light():
    from tests.helpers import small_noise_scene
    d = small_noise_scene(w=24, h=16, phase="hg", anisotropy=0.4)
    means = []
    for pv in ({"enabled": 1}, {"enabled": 1, "emission_strength": 2.0},
               {"enabled": 1, "emission_strength": 2.0, "blackbody_intensity": 1.0, "temperature": 5000.0}):
        acc = np.zeros((16, 24, 4), np.float32)
        oracle.render(oracle.Scene(dict(d, principled=pv)), 0, 16, accum=acc)
        means.append(float(oracle.resolve(acc, 16)[..., :3].mean()))
    assert means[0] < means[1] < means[2]
    # the default build (SimplePhase) has no emission
    s = small_noise_scene(w=24, h=16, phase="simple")
    a = np.zeros((16, 24, 4), np.float32)
    b = np.zeros_like(a)
    oracle.render(oracle.Scene(dict(s, principled={"enabled": 1})), 0, 4, accum=a)
    oracle.render(oracle.Scene(dict(s, principled={"enabled": 1, "emission_strength": 5.0})), 0, 4, accum=b)
    assert np.array_equal(a, b)


# ---------------------------------------------------------------------------
# isosurfaces (MCIsoSurfaceAccel::isProg) with a matte (Lambertian) material
# ---------------------------------------------------------------------------
def ramp_scene(iso=0.37, nx=17, ny=9, nz=9, **kw):
    """Field f(x, y, z) = x on [0,1]^3: an x-ramp whose isosurface is the plane
    x = iso with normal +x.  Values i/16 are exact in binary32."""
    from barney_b200 import synth
    x = (np.arange(nx, dtype=np.float32) / f32(nx - 1))
    vol = np.broadcast_to(x[None, None, :], (nz, ny, nx)).astype(np.float32).copy()
    d = synth.scene(vol, "f32", 16, 16, synth.tf_linear_ramp(2), 1.0,
                    {"position": (2.0, 0.5, 0.5), "direction": (-1.0, 0.0, 0.0), "up": (0.0, 1.0, 0.0), "fovy": 10.0},
                    volume=False, iso={"value": iso, "color": (0.9, 0.6, 0.3)})
    d.update(kw)
    return d


def test_iso_ramp_plane_hit_distance_and_normal():
    sc = oracle.Scene(ramp_scene(0.37))
    # from the -x side and from the +x side: the plane x = 0.37; linear
    # interpolation of a linear field finds it to rounding
    hit, t, n = oracle.iso_trace(sc, (-0.5, 0.5, 0.5), (1.0, 0.0, 0.0))
    assert hit and abs(t - 0.87) < 2e-6
    assert n.tolist() == [1.0, 0.0, 0.0]  # gradient +x, normalized, binary16
    hit, t, n = oracle.iso_trace(sc, (1.5, 0.5, 0.5), (-1.0, 0.0, 0.0))
    assert hit and abs(t - 1.13) < 2e-6
    assert n.tolist() == [1.0, 0.0, 0.0]  # the stored normal does not face the ray
    # an oblique ray: t where 0.2 + t * 0.6 = 0.37 (direction normalized)
    d = np.array([0.6, 0.48, 0.64], np.float32)
    hit, t, _ = oracle.iso_trace(sc, (0.2, 0.1, 0.1), d)
    assert hit and abs(t - (0.17 / 0.6)) < 2e-6
    # short of the plane, or an iso value outside the field's range: no hit
    assert not oracle.iso_trace(sc, (-0.5, 0.5, 0.5), (1.0, 0.0, 0.0), tmax=0.8)[0]
    assert not oracle.iso_trace(oracle.Scene(ramp_scene(1.5)), (-0.5, 0.5, 0.5), (1.0, 0.0, 0.0))[0]


def test_frame_is_orthonormal_and_maps_z_to_the_normal():
    rng = np.random.default_rng(5)
    for _ in range(64):
        N = rng.normal(size=3).astype(np.float32)
        N = (N / np.linalg.norm(N)).astype(np.float32)
        assert np.array_equal(oracle.frame_xfm(N, (0.0, 0.0, 1.0)), N)
        ex, ey = oracle.frame_xfm(N, (1.0, 0.0, 0.0)), oracle.frame_xfm(N, (0.0, 1.0, 0.0))
        for a, b in ((ex, ey), (ex, N), (ey, N)):
            assert abs(float(np.dot(a, b))) < 1e-6
        assert abs(float(np.linalg.norm(ex)) - 1) < 1e-6 and abs(float(np.linalg.norm(ey)) - 1) < 1e-6
        # right-handed: dy = N x dx
        assert np.allclose(np.cross(N, ex), ey, atol=1e-6)


def test_iso_plane_facing_a_directional_light_radiance():
    """Every sample of the plane x = 0.37 seen along -x, lit head-on by one
    directional light with no ambient: the shadow ray's fragment is
    halfRound(tp) with tp = (.85 c / pi) / pi * cos * (1/pi * |cos|) -- the
    Lambertian's albedo carries 1/pi, its eval another, the surface cosine a
    third (shadeRays.cu:686-691) -- and the diffuse bounce escapes into a black
    environment."""
    d = ramp_scene(0.37, ambient=0.0, dir_lights=[{"direction": (-1.0, 0.0, 0.0), "radiance": 1.0}])
    spp = 8
    acc, _, st = oracle.render(oracle.Scene(d), 0, spp)
    one_over_pi = f32(1.0) / f32(math.pi)
    expect = []
    for c in (0.9, 0.6, 0.3):
        albedo = f32(0.85) * f32(c) * one_over_pi
        fval = albedo * one_over_pi * f32(1.0)
        tp = f32(1.0) * f32(1.0) * fval * f32(1.0) * (one_over_pi * f32(1.0))
        expect.append(float(np.float16(tp)))
    img = acc / spp
    assert np.array_equal(img[..., :3], np.broadcast_to(np.array(expect, np.float32), img[..., :3].shape))
    assert np.all(img[..., 3] == 1.0)
    # per sample: the primary ray, its shadow ray and the diffuse bounce
    assert st["rays"] == 3 * 16 * 16 * spp and st["samples"] == 0


def test_iso_opacity_zero_passes_every_ray_and_one_blocks():
    d = ramp_scene(0.37, bg_color=(0.25, 0.5, 0.75, 1.0))
    acc, _, st = oracle.render(oracle.Scene(dict(d, iso={"value": 0.37, "opacity": 0.0})), 0, 2)
    assert np.array_equal(acc / 2, np.broadcast_to(np.array([0.25, 0.5, 0.75, 1.0], np.float32), acc.shape))
    assert st["rays"] == 16 * 16 * 2
    acc1, _, _ = oracle.render(oracle.Scene(d), 0, 2)
    assert not np.array_equal(acc1, acc)


def test_iso_scan_step_table_is_the_correctly_rounded_quotient():
    # The isosurface scan's step fractions (MCAccelerator.h: (float)i / 10.f)
    # come from a table in the kernels; every entry must be that quotient,
    # rounded once to binary32, as the oracle evaluates it.
    import os
    import re
    src = open(os.path.join(os.path.dirname(__file__), "..", "barney_b200", "csrc", "bn_kernels.cu")).read()
    m = re.search(r"kIsoTenths\[11\]\s*=\s*\{([^}]*)\}", src)
    assert m, "step table not found"
    table = [np.float32(float(x.strip().rstrip("f"))) for x in m.group(1).split(",")]
    assert len(table) == 11
    for i, t in enumerate(table):
        assert t.view(np.uint32) == (np.float32(i) / np.float32(10)).view(np.uint32), i
