"""CPU checks of the densities the guided path tracer's one-sample MIS uses.

The guided tracer (research_b200/csrc/guided.cu) draws a bounce either from a
vMF mixture or from the reference's brdf_sample (BRDF.slang:116-172) and
weights it by f cos (actual/ref) / (alpha p_guide + (1 - alpha) actual), where
`ref` is the density the reference divides by and `actual` the density
brdf_sample really draws from (rr_vmf.cuh, brdf_sample_pdfs). The formula for
`actual` is restated here in numpy and checked against a histogram of the
oracle's brdf_sample, which follows the reference line by line.
"""
import math

import numpy as np
import pytest


def fresnel(cos_t, F0):
    x = np.clip(1.0 - cos_t, 0.0, 1.0)
    return F0 + (1.0 - F0) * x ** 5


def brdf_pdfs(wo, wi, base, metallic, roughness):
    """(ref, actual) densities at unit directions wi (rows), normal +z."""
    r = min(max(roughness, 0.04), 1.0)
    F0 = 0.04 * (1 - metallic) + np.asarray(base) * metallic
    p_spec = float(np.clip(fresnel(max(wo[2], 0.0), F0).mean(), 0.1, 0.9))
    a = r * r
    h = wo[None, :] + wi
    h /= np.linalg.norm(h, axis=1, keepdims=True)
    nh = np.maximum(h[:, 2], 1e-6)
    vh = np.maximum(h @ wo, 1e-6)
    D = a * a / np.maximum(math.pi * (nh * nh * (a * a - 1) + 1) ** 2, 1e-7)
    diff = np.maximum(wi[:, 2], 0.0) / math.pi
    ref = np.maximum(p_spec * D * nh / np.maximum(4 * vh, 1e-6) + (1 - p_spec) * diff, 1e-6)
    vz = max(wo[2], 0.0)
    lam = math.sqrt(a * a * (wo[0] ** 2 + wo[1] ** 2) + vz * vz)
    actual = p_spec * D / (2 * (vz + lam)) + (1 - p_spec) * diff
    return ref, actual


def _histogram_check(O, theta_o, base, metallic, roughness, n_samples=120_000, seed=0):
    rng = np.random.default_rng(seed)
    wo = np.array([math.sin(theta_o), 0.0, math.cos(theta_o)], np.float32)
    n = np.array([0, 0, 1], np.float32)
    base = np.asarray(base, np.float32)
    u = rng.random((n_samples, 2)).astype(np.float32)
    dirs = []
    for u0, u1 in u:
        wi, _, f = O.brdf_sample(wo, n, base, metallic, roughness, float(u0), float(u1))
        if np.any(f != 0) and wi[2] > 0:       # rejected VNDF samples carry nothing
            dirs.append(wi)
    dirs = np.array(dirs, np.float64)
    # equal-solid-angle bins in (cos theta, phi)
    nc, nphi = 16, 24
    ci = np.minimum((dirs[:, 2] * nc).astype(int), nc - 1)
    pi_ = np.minimum(((np.arctan2(dirs[:, 1], dirs[:, 0]) + math.pi) / (2 * math.pi) * nphi).astype(int), nphi - 1)
    counts = np.zeros((nc, nphi))
    np.add.at(counts, (ci, pi_), 1)
    d_omega = (1.0 / nc) * (2 * math.pi / nphi)
    emp = counts / (n_samples * d_omega)
    # bin averages of the two densities (8 x 8 sub-points per bin)
    sub = (np.arange(8) + 0.5) / 8
    pred_ref = np.zeros((nc, nphi)); pred_act = np.zeros((nc, nphi))
    for i in range(nc):
        for j in range(nphi):
            c = (i + sub[:, None]) / nc * np.ones((1, 8))
            ph = ((j + sub[None, :]) / nphi * 2 * math.pi - math.pi) * np.ones((8, 1))
            s = np.sqrt(np.maximum(0, 1 - c * c))
            wi = np.stack([s * np.cos(ph), s * np.sin(ph), c], -1).reshape(-1, 3)
            ref, act = brdf_pdfs(wo.astype(np.float64), wi, base, metallic, roughness)
            pred_ref[i, j], pred_act[i, j] = ref.mean(), act.mean()
    return emp, counts, pred_ref, pred_act


def _poisson_z(counts, density, n_samples=120_000, min_expected=100.0):
    """(observed - expected) / sqrt(expected) over bins expecting enough counts."""
    d_omega = (1.0 / counts.shape[0]) * (2 * math.pi / counts.shape[1])
    expected = density * n_samples * d_omega
    keep = expected >= min_expected
    return (counts[keep] - expected[keep]) / np.sqrt(expected[keep])


@pytest.mark.parametrize("theta_deg,base,metallic,roughness", [
    (75.0, (0.9, 0.9, 0.9), 1.0, 0.6),
    (40.0, (0.8, 0.3, 0.2), 0.0, 0.5),
    (60.0, (0.5, 0.5, 0.5), 1.0, 0.9),
])
def test_actual_density_matches_brdf_sample_histogram(O, theta_deg, base, metallic, roughness):
    emp, counts, pred_ref, pred_act = _histogram_check(O, math.radians(theta_deg), base, metallic, roughness)
    z = _poisson_z(counts, pred_act)
    assert len(z) >= 40
    # counting statistics only: mean z^2 ~ 1 (chi-square per bin), no outlier
    assert np.mean(z * z) < 1.6 and np.abs(z).max() < 5.0, (np.mean(z * z), np.abs(z).max())
    # total mass: the sampled directions integrate to the predicted mass
    assert (emp.sum() - pred_act.sum()) / pred_act.sum() == pytest.approx(0.0, abs=0.02)


def test_reference_formula_is_not_the_sampling_density(O):
    """At a grazing view the reference's D*NdotH/(4 VdotH) differs from the
    VNDF density it samples, which is why the guided estimator carries the
    ratio actual/ref (a plain MIS over `ref` would converge elsewhere)."""
    emp, counts, pred_ref, pred_act = _histogram_check(O, math.radians(75.0), (0.9, 0.9, 0.9), 1.0, 0.6)
    z_act, z_ref = _poisson_z(counts, pred_act), _poisson_z(counts, pred_ref)
    assert np.mean(z_act * z_act) < 1.6
    assert np.mean(z_ref * z_ref) > 20.0, np.mean(z_ref * z_ref)
