"""Tile-sorted accumulation (samples emitted as records, counting-sorted by
band and 64x64-pixel tile, summed in shared memory): the exact histogram
must be the same bits as the direct exact splat's, which adds the same
integers."""

import copy

import numpy as np
import pytest

from ffb200 import synthetic

pytestmark = pytest.mark.gpu


def both(renderer, cfg, W, H, **job):
    a = renderer.histogram_u64(cfg, W, H, accumulate="direct", **job)
    b = renderer.histogram_u64(cfg, W, H, accumulate="tiled", **job)
    return a, b


def same(a, b):
    (ca, ra, oa), (cb, rb, ob) = a, b
    assert oa.total_iterations == ob.total_iterations
    assert oa.inframe_samples == ob.inframe_samples
    assert np.array_equal(ca, cb)
    assert np.array_equal(ra, rb)
    assert int(ca.sum()) == oa.inframe_samples


def test_linear_flame(renderer):
    same(*both(renderer, synthetic.sierpinski(), 300, 200, iterations=2048 * 500, walkers=2048))


def test_full_flame_supersampled(renderer):
    same(*both(renderer, synthetic.full_flame(6), 350, 250, supersample=2, iterations=4096 * 400, walkers=4096))


@pytest.mark.parametrize("schedule", ["plain", "sorted"])
def test_symmetry_copies(renderer, schedule):
    cfg = copy.deepcopy(synthetic.plain_flame(2))
    cfg["flame"]["post_symmetry"] = {"ty": "point", "order": 5, "center_x": 0.0, "center_y": 0.0, "distance": 1.25,
                                     "rotation_deg": 6.0}
    same(*both(renderer, cfg, 257, 193, iterations=2000 * 300, walkers=2000, schedule=schedule))


def test_pcg_stream(renderer):
    same(*both(renderer, synthetic.plain_flame(3), 200, 120, iterations=1024 * 2000, walkers=1024, rng="pcg",
               iterations_per_thread=256))


def test_hot_tile_split_over_slices(renderer):
    """Every sample in one pixel: its tile holds more records than a slice, so
    several blocks sum it and add it with atomics."""
    cfg = {"flame": {"transforms": [{"a": 0, "b": 0, "c": 0, "d": 0, "e": 0.3, "f": -0.2, "weight": 1, "color": 0.5,
                                     "color_speed": 0.5, "variations": {"linear": 1.0}}]}, "deterministic_rng": True}
    a, b = both(renderer, cfg, 128, 128, iterations=4096 * 300, walkers=4096)
    same(a, b)
    assert int((a[0] > 0).sum()) == 1 and int(a[0].max()) == 4096 * 300


def test_several_launches(renderer):
    """More iterations than one launch's record budget: the passes add up."""
    same(*both(renderer, synthetic.plain_flame(4), 640, 360, iterations=65536 * 9000, walkers=65536))


# ---- the u32-count / FP32-colour histogram through the same passes --------

def both32(renderer, cfg, W, H, **job):
    a = renderer.histogram(cfg, W, H, accumulate="direct", **job)
    b = renderer.histogram(cfg, W, H, accumulate="tiled", **job)
    return a, b


def same32(a, b):
    """Counts bit for bit; colour sums within the FP32 summation bound.
    Either path adds a pixel's n colours (each in [0, 1]) in some order, a
    recursive sum whose error is at most (n + 1) u S (u = 2^-24, S the sum),
    so the two differ by at most 2 (n + 1) u S."""
    (ca, ra, oa), (cb, rb, ob) = a, b
    assert oa.total_iterations == ob.total_iterations
    assert oa.inframe_samples == ob.inframe_samples
    assert np.array_equal(ca, cb)
    assert int(ca.sum()) == oa.inframe_samples
    n = ca.astype(np.float64)[..., None]
    s = np.maximum(np.abs(ra), np.abs(rb)).astype(np.float64)
    assert np.all(np.abs(ra.astype(np.float64) - rb) <= 2.0 * (n + 1.0) * 2.0 ** -24 * s)
    assert np.array_equal(ra == 0, rb == 0)


def test_f32_linear_flame(renderer):
    same32(*both32(renderer, synthetic.sierpinski(), 300, 200, iterations=2048 * 500, walkers=2048))


def test_f32_full_flame_supersampled(renderer):
    same32(*both32(renderer, synthetic.full_flame(6), 350, 250, supersample=2, iterations=4096 * 400, walkers=4096))


def test_f32_symmetry_copies_sorted(renderer):
    cfg = copy.deepcopy(synthetic.plain_flame(2))
    cfg["flame"]["post_symmetry"] = {"ty": "point", "order": 5, "center_x": 0.0, "center_y": 0.0, "distance": 1.25,
                                     "rotation_deg": 6.0}
    same32(*both32(renderer, cfg, 257, 193, iterations=2000 * 300, walkers=2000, schedule="sorted"))


def test_f32_hot_tile_split_over_slices(renderer):
    """Every sample in one pixel (colour index fixed at 0.5 after the
    burn-in, so one palette colour): the tiled sum, split over several
    slices added with atomics, within the summation bound of n times it."""
    cfg = {"flame": {"transforms": [{"a": 0, "b": 0, "c": 0, "d": 0, "e": 0.3, "f": -0.2, "weight": 1, "color": 0.5,
                                     "color_speed": 0.5, "variations": {"linear": 1.0}}]}, "deterministic_rng": True}
    a, b = both32(renderer, cfg, 128, 128, iterations=4096 * 300, walkers=4096)
    same32(a, b)
    assert int((a[0] > 0).sum()) == 1 and int(a[0].max()) == 4096 * 300


def test_f32_several_launches(renderer):
    same32(*both32(renderer, synthetic.plain_flame(4), 640, 360, iterations=65536 * 9000, walkers=65536))


def test_tiled_is_refused_with_the_spatial_filter(renderer):
    from ffb200 import _native
    cfg = copy.deepcopy(synthetic.plain_flame(1))
    cfg["filter_radius"] = 0.5
    with pytest.raises(_native.EngineError, match="spatial filter"):
        renderer.histogram_f32(cfg, 64, 64, iterations=10_000, accumulate="tiled")
