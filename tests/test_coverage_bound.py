"""The FP32 raster's single coverage test (CPU, no GPU needed).

The raster covers a pixel when r^2 <= thr, thr = min(s^2, the largest float
below (log2 alpha + 8) / (4.5 log2 e)), formed once per splat and tile. In
exact arithmetic w = alpha e^(-4.5 r^2) > 1/256 holds exactly when r^2 is
below that bound, so one comparison stands for the reference fragment rule's
alpha discard (splat_surface_direct.wgsl:356-369). These tests restate the
bound in float32 the way the kernel and the oracle form it and check it
against the weight evaluated in float64: the two tests disagree only on a
sliver at the bound, the same class of pixels on which the hardware and the
oracle's exponentials may already differ."""

import numpy as np

K = np.float32(6.49212768)  # 4.5 log2(e), the constant both the kernel and the oracle use


def coverage_bound(log2a, s2):
    log2a = np.asarray(log2a, np.float32)
    s2 = np.asarray(s2, np.float32)
    wlim = (log2a + np.float32(8.0)) / K  # float32 add and IEEE division, as on the device
    below = np.nextafter(wlim, np.float32(0.0))
    return np.where(wlim > 0, np.minimum(s2, below), np.float32(-1.0)).astype(np.float32)


def weight64(log2a, r2):
    return np.exp2(np.asarray(log2a, np.float64)) * np.exp(-4.5 * np.asarray(r2, np.float64))


def test_bound_matches_the_alpha_threshold_away_from_the_boundary():
    rng = np.random.default_rng(7)
    n = 2_000_000
    alpha = rng.uniform(1.0 / 255.0, 1.0, n).astype(np.float32)
    log2a = np.log2(alpha).astype(np.float32)
    r2 = rng.uniform(0.0, 1.2, n).astype(np.float32)
    s2 = np.full(n, np.float32(1.0))
    covered = r2 <= coverage_bound(log2a, s2)
    exact = (weight64(log2a, r2) > 1.0 / 256.0) & (r2 <= s2)
    differ = covered != exact
    # only at the bound: within a few float32 ulps of the exact r^2 where w = 1/256
    r2_star = (np.float64(log2a) + 8.0) / (4.5 / np.log(2.0))
    gap = np.abs(r2[differ].astype(np.float64) - r2_star[differ])
    assert np.all(gap <= 4 * np.spacing(np.float32(1.0)) * np.maximum(r2_star[differ], 1e-3))
    assert differ.mean() < 1e-5


def test_no_coverage_when_alpha_is_below_the_threshold():
    log2a = np.log2(np.array([1e-4, 1.0 / 300.0, 1.0 / 256.5], np.float32)).astype(np.float32)
    thr = coverage_bound(log2a, np.ones(3, np.float32))
    assert np.all(thr < 0)  # r^2 >= 0 never passes


def test_bound_is_capped_by_the_quad_clip():
    log2a = np.zeros(4, np.float32)  # alpha = 1: the weight bound lies at r^2 = 1.232
    s2 = np.array([0.25, 0.5, 1.0, 2.0], np.float32)
    thr = coverage_bound(log2a, s2)
    assert np.array_equal(thr[:3], s2[:3])
    assert thr[3] < np.float32(1.2323) and thr[3] > np.float32(1.2322)


def test_weight_at_the_bound_is_the_threshold():
    rng = np.random.default_rng(3)
    log2a = np.log2(rng.uniform(0.01, 1.0, 10_000)).astype(np.float32)
    thr = coverage_bound(log2a, np.full(log2a.shape, np.float32(4.0)))
    w = weight64(log2a, thr)
    # the last covered r^2 carries the smallest weight the raster blends: 1/256 up to rounding
    assert np.all(np.abs(w * 256.0 - 1.0) < 1e-5)
