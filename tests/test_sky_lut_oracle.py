"""Sky-view LUT lookup (sample_sky_lut, scene.slang:469-518) and the own
atan2 / asin it uses, on the oracle (CPU).

* atan2 and asin against the C library in float64: a few float ulps for
  atan2 everywhere and for asin away from the poles (the lookup clamps the
  altitude 0.01 rad short of them).
* The float lookup against an independent float64 restatement written here
  with numpy's arcsin/arctan2: the same (u, v) mapping and wrapped bilinear
  fetch, within float rounding.
* A constant LUT gives its value times the sun's outer-space illuminance in
  every direction, and a direction along `up` (no azimuth) stays finite.
"""

import math

import numpy as np
import pytest


def _lighting(lut, sun=(0.3, 0.5, 0.81), up=(0.0, 1.0, 0.0), intensity=2.5):
    import nan_b200

    return nan_b200.Lighting(sun_direction=sun, sun_intensity=intensity, sun_color=(1.0, 0.9, 0.8),
                             sky_view_lut=lut, sky_view_up=up)


def _dirs(n, seed):
    d = np.random.default_rng(seed).normal(size=(n, 3))
    return (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)


def test_own_atan2_and_asin_match_the_c_library(oracle_mod):
    rng = np.random.default_rng(1)
    y = rng.uniform(-3, 3, 20000).astype(np.float32)
    x = rng.uniform(-3, 3, 20000).astype(np.float32)
    y[:8] = [0, 0, 1, -1, 0, 1e-30, -2, 5]
    x[:8] = [1, -1, 0, 0, 0, 1, 0, -1e-30]
    a, _ = oracle_mod.atan2_asin(y, x)
    ref = np.arctan2(y.astype(np.float64), x.astype(np.float64))
    assert np.max(np.abs(a - ref)) <= 5e-7
    assert a[4] == 0.0  # atan2(0, 0)
    s_in = rng.uniform(-1, 1, 20000).astype(np.float32)
    _, s = oracle_mod.atan2_asin(s_in, np.ones_like(s_in))
    err = np.abs(s - np.arcsin(s_in.astype(np.float64)))
    inner = np.abs(s_in) <= np.cos(0.01)
    assert np.max(err[inner]) <= 2e-6 and np.max(err) <= 5e-4


def _reference_lookup(lut, d, sun, up, horizon, outer):
    """The Slang lookup in float64 with numpy's inverse trig functions."""
    h, w = lut.shape[:2]
    up = np.asarray(up, np.float64)
    sun = np.asarray(sun, np.float64)
    d = d.astype(np.float64)
    mu = d @ up
    alt = np.clip(np.arcsin(np.clip(mu, -1, 1)), -0.5 * math.pi + 1e-2, 0.5 * math.pi - 1e-2)
    right = np.cross(sun, up)
    fwd = np.cross(up, right)
    proj = d - np.outer(mu, up)
    proj /= np.linalg.norm(proj, axis=1, keepdims=True)
    az = np.arctan2(proj @ right, proj @ fwd)
    adj = (alt + horizon) / (0.5 * math.pi)
    v = np.where(adj < 0, 0.5 * (1 - np.sqrt(np.clip(-adj, 0, 1))), 0.5 * (1 + np.sqrt(np.clip(adj, 0, 1))))
    u = az / (2 * math.pi) + 0.5
    fx, fy = u * w - 0.5, v * h - 0.5
    x0, y0 = np.floor(fx).astype(int), np.floor(fy).astype(int)
    tx, ty = (fx - x0)[:, None], (fy - y0)[:, None]
    t = lut[..., :3].astype(np.float64)

    def at(x, y):
        return t[y % h, x % w]

    top = at(x0, y0) + tx * (at(x0 + 1, y0) - at(x0, y0))
    bot = at(x0, y0 + 1) + tx * (at(x0 + 1, y0 + 1) - at(x0, y0 + 1))
    return (top + ty * (bot - top)) * outer


def test_lookup_matches_an_independent_float64_restatement(oracle_mod):
    from nan_b200.scene import sky_view_horizon_angle

    h, w = 200, 200
    yy, xx = np.meshgrid(np.linspace(0, 1, h), np.linspace(0, 1, w), indexing="ij")
    lut = np.zeros((h, w, 4), np.float32)
    lut[..., 0] = 0.2 + 0.5 * yy * yy
    lut[..., 1] = 0.3 + 0.2 * np.sin(2 * np.pi * xx)
    lut[..., 2] = 0.5 + 0.3 * yy * np.cos(2 * np.pi * xx)
    L = _lighting(lut)
    d = _dirs(5000, 2)
    got = oracle_mod.sky_radiance(L, d)
    outer = np.array(L.sun_color, np.float64) * L.sun_intensity
    ref = _reference_lookup(lut, d, L.sun_direction, L.sky_view_up, sky_view_horizon_angle(), outer)
    rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-3)
    assert np.quantile(rel, 0.999) <= 1e-4 and np.max(rel) <= 2e-3
    f64 = oracle_mod.sky_radiance(L, d, precision=oracle_mod.F64)
    assert np.max(np.abs(f64 - ref) / np.maximum(np.abs(ref), 1e-3)) <= 1e-5


def test_constant_lut_and_straight_up(oracle_mod):
    lut = np.zeros((8, 16, 4), np.float32)
    lut[..., :3] = (0.25, 0.5, 1.0)
    L = _lighting(lut, intensity=2.0)
    d = np.concatenate([_dirs(1000, 3), np.array([[0, 1, 0], [0, -1, 0]], np.float32)])
    got = oracle_mod.sky_radiance(L, d)
    expect = np.array([0.25, 0.5, 1.0], np.float32) * np.array(L.sun_color, np.float32) * np.float32(2.0)
    assert np.all(np.isfinite(got))
    np.testing.assert_allclose(got, np.broadcast_to(expect, got.shape), rtol=2e-7)


def test_no_lut_is_the_constant_sky(oracle_mod):
    import nan_b200

    L = nan_b200.Lighting(sky_radiance=(0.1, 0.2, 0.3))
    got = oracle_mod.sky_radiance(L, _dirs(10, 4))
    np.testing.assert_array_equal(got, np.broadcast_to(np.array([0.1, 0.2, 0.3], np.float32), got.shape))
