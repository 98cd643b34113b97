"""The FP64 ray-marched expectation (oracle/bn_fp64.cpp) is what the
estimator converges to: the FP32 restatement with exact -log free-flight
sampling, averaged over many waves, agrees with it within Monte-Carlo error
(3 standard errors plus the quadrature's discretisation) in every lighting
mode; with the reference's fastLog series the estimator is visibly biased."""
import numpy as np
import pytest

import oracle
from barney_b200 import synth

W, H, SPP = 6, 5, 3000


def _scene(**kw):
    vol = synth.value_noise(20, 3)
    d = synth.scene(vol, "f32", W, H, synth.tf_knots(64, 1), 8.0, synth.look_at((1.6, 1.2, 1.7), fovy=30.0),
                    exact_log=True)
    d.update(kw)
    return d


def _per_wave_mean_and_se(d):
    sc = oracle.Scene(d)
    waves = np.zeros((SPP, H, W, 4), np.float64)
    for k in range(SPP):
        one, _, _ = oracle.render(sc, k + 1, 1, accum=np.zeros((H, W, 4), np.float32), threads=0)
        waves[k] = one
    return waves.mean(0), waves.std(0, ddof=1) / np.sqrt(SPP)


@pytest.mark.parametrize("mode", ["emission_absorption", "ambient_simple", "dirlight_hg", "both_hg_aniso"])
def test_fp64_expectation_matches_exact_log_estimator(mode):
    kw = {
        "emission_absorption": dict(emission_absorption=True, ambient=0.0, bg_color=(0.2, 0.3, 0.4, 1.0)),
        "ambient_simple": dict(ambient=1.0),
        "dirlight_hg": dict(ambient=0.0, phase="hg", anisotropy=0.0, scattering_albedo=0.8,
                            dir_lights=synth.CONFIG2_LIGHTS),
        "both_hg_aniso": dict(ambient=0.25, phase="hg", anisotropy=0.4, scattering_albedo=0.8,
                              dir_lights=synth.CONFIG2_LIGHTS),
    }[mode]
    d = _scene(**kw)
    mean, se = _per_wave_mean_and_se(d)
    exp = oracle.render_expected_fp64(oracle.Scene(d), step=0.25 / 19, subpix=4, env_dirs=256)
    diff = np.abs(mean[..., :3] - exp[..., :3])
    tol = 3 * se[..., :3] + 0.02 * np.abs(exp[..., :3]) + 2e-3
    assert np.all(diff <= tol), (diff.max(), (diff - tol).max())
