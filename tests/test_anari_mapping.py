"""ANARI parameter mapping (barney/anari/Volume.cpp:82-234) restated in
bnxAnariTransferFunction1D / bnxAnariDensityScale: checked on the CPU
against a step-by-step numpy float32 restatement of the reference loop."""
import numpy as np
import pytest

import barney_b200 as bn

f32 = np.float32


def reference_table(colors, opacities, uc=(1, 1, 1, 1), uo=1.0):
    uc = np.array(uc, np.float32)
    u_op = f32(uo) * uc[3]
    nc = 1 if colors is None else len(colors)
    no = 1 if opacities is None else len(opacities)
    n = max(nc, no)
    out = np.zeros((n, 4), np.float32)
    for i in range(n):
        cp = (f32(i) / f32(n - 1)) * f32(nc - 1) if n > 1 else f32(0)
        cf = cp - np.floor(cp)
        c0 = np.array([uc[0], uc[1], uc[2], u_op], np.float32)
        c1 = c0.copy()
        if colors is not None:
            a, b = int(np.floor(cp)), int(np.ceil(cp))
            if colors.shape[1] == 3:
                c0 = np.array([*colors[a], u_op], np.float32)
                c1 = np.array([*colors[b], u_op], np.float32)
            else:
                c0, c1 = colors[a].copy(), colors[b].copy()
        col = (f32(1) - cf) * c0 + cf * c1
        if opacities is not None:
            ap = (f32(i) / f32(n - 1)) * f32(no - 1) if n > 1 else f32(0)
            af = ap - np.floor(ap)
            a0, a1 = opacities[int(np.floor(ap))], opacities[int(np.ceil(ap))]
            col[3] = col[3] * ((f32(1) - af) * a0 + af * a1)
        out[i] = col
    return out


@pytest.mark.parametrize("nc,ch,no", [(5, 3, 17), (17, 4, 5), (8, 4, 8), (1, 3, 9), (0, 3, 7), (6, 4, 0), (0, 3, 0)])
def test_transfer_function_resampling(nc, ch, no):
    rng = np.random.default_rng(nc * 100 + no)
    colors = rng.random((nc, ch)).astype(np.float32) if nc else None
    ops = rng.random(no).astype(np.float32) if no else None
    got = bn.anari_transfer_function_1d(colors, ops, uniform_color=(0.3, 0.6, 0.9, 0.5), uniform_opacity=0.8)
    exp = reference_table(colors, ops, (0.3, 0.6, 0.9, 0.5), 0.8)
    assert np.array_equal(got.view(np.uint32), exp.view(np.uint32))


def test_density_scale():
    L = bn.lib()
    assert L.bnxAnariDensityScale(0.5) == 2.0
    assert L.bnxAnariDensityScale(0.0) == 1.0
    assert L.bnxAnariDensityScale(-3.0) == 1.0


# Renderer::commitParameters (barney/anari/Renderer.cpp:22-37): the value of
# each parameter the application did not set
ANARI_RENDERER_DEFAULTS = {"pixelSamples": 1, "ambientRadiance": 1.0, "background": (0.0, 0.0, 0.0, 1.0),
                           "cutPlane": (0.0, 0.0, 0.0, 0.0), "maxVolumeBounces": 0, "crosshairs": 0}


def test_renderer_defaults():
    got = bn.anari_renderer_params()
    assert got.pop("set") == 0x3F
    assert got == ANARI_RENDERER_DEFAULTS


@pytest.mark.parametrize("mask", range(64))
def test_renderer_parameters_set_and_default(mask):
    rng = np.random.default_rng(mask)
    values = {"pixelSamples": int(rng.integers(1, 64)), "ambientRadiance": float(f32(rng.random())),
              "background": tuple(float(x) for x in rng.random(4).astype(np.float32)),
              "cutPlane": tuple(float(x) for x in (rng.random(4) - 0.5).astype(np.float32)),
              "maxVolumeBounces": int(rng.integers(0, 9)), "crosshairs": 1}
    names = list(ANARI_RENDERER_DEFAULTS)
    given = {k: values[k] for i, k in enumerate(names) if mask >> i & 1}
    got = bn.anari_renderer_params(**given)
    assert got.pop("set") == 0x3F
    want = dict(ANARI_RENDERER_DEFAULTS, **given)
    assert got == want


def test_renderer_unknown_parameter_is_refused():
    with pytest.raises(ValueError):
        bn.anari_renderer(denoise=True)
