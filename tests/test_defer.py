"""Deferred plotting (ffb_job.plot = 2): the chaos kernel stores each kept
sample (its point after the transform, colour index, opacity draw, and the
draws its final chain takes) and a plot kernel on a second stream applies
the final chain, the palette, the symmetry copies and the splat, beside the
next launch.  It is the same render: the same samples reach the same
pixels, so the count plane is identical to the inline plot's, and in exact
mode (order-independent fixed-point sums) the colour sums are too.

CPU: the deferred module builds and captures the final chain's draws.
GPU: identical histograms, inline against deferred, across schedules,
finals with draws, post-symmetry, xaos and exact accumulation.
"""

import copy

import numpy as np
import pytest

from ffb200 import synthetic
from ffb200 import _native


def full_with_final_draws(seed=6):
    cfg = synthetic.full_flame(seed, de_radius=0)
    cfg["flame"]["final_transform"]["variations"]["julia"] = 0.3       # the final takes a draw
    return cfg


def test_deferred_module_captures_the_final_draws():
    n, src = _native.specialize_job(full_with_final_draws(), plot="deferred")
    assert n > 0 and "#define FFB_DEFER 1" in src and "#define FFB_NFD 1" in src
    assert "ffb_capture_final_draws" in src and "ffb_plot(" in src
    # Only the counter-based stream defers (a PCG launch must cover whole dispatches).
    _, src = _native.specialize_job(full_with_final_draws(), plot="deferred", rng="pcg")
    assert "#define FFB_DEFER 1" not in src


def test_auto_defers_the_sorted_schedule_over_many_walkers():
    cfg = full_with_final_draws()
    _, src = _native.specialize_job(cfg, walkers=65536)
    assert "#define FFB_DEFER 1" in src
    for job in (dict(walkers=4096), dict(walkers=65536, schedule="plain"), dict(walkers=65536, count_bits=64,
                accumulate="tiled", width=7680, height=4320), dict(walkers=65536, plot="inline")):
        _, src = _native.specialize_job(cfg, **job)
        assert "#define FFB_DEFER 1" not in src, job


def test_fused_kernel_is_in_the_deferred_module():
    """plot 3 (fused): the deferred module of the counter-based stream also
    compiles ffb_chaos_fused; the PCG stream and orbit refresh have none."""
    _, src = _native.specialize_job(full_with_final_draws(), plot="fused")
    assert "#define FFB_DEFER 1" in src and "ffb_chaos_fused(" in src and "#define FFB_REFRESH" not in src
    _, src = _native.specialize_job(full_with_final_draws(), plot="fused", rng="pcg")
    assert "#define FFB_DEFER 1" not in src


def run(renderer, cfg, w, h, **job):
    return renderer.histogram(cfg, w, h, **job)


@pytest.mark.gpu
@pytest.mark.parametrize("schedule", ["plain", "sorted"])
def test_deferred_equals_inline(renderer, schedule):
    cfg = full_with_final_draws()
    job = dict(iterations=20_000_000, walkers=16384, supersample=2, schedule=schedule)
    a, ra, oa = run(renderer, cfg, 320, 180, plot="inline", **job)
    b, rb, ob = run(renderer, cfg, 320, 180, plot="deferred", **job)
    assert oa.inframe_samples == ob.inframe_samples == int(a.sum()) > 0
    assert np.array_equal(a, b)
    np.testing.assert_allclose(ra, rb, rtol=1e-4, atol=1e-3)
    assert ob.kernel_launches > oa.kernel_launches                   # the plot kernels ran


@pytest.mark.gpu
@pytest.mark.parametrize("sym", [{"ty": "point", "order": 5, "center_x": 0.1, "center_y": 0.0, "distance": 1.25,
                                  "rotation_deg": 0.0},
                                 {"ty": "xaxis", "order": 2, "center_x": 0.0, "center_y": 0.2, "distance": 0.8,
                                  "rotation_deg": 20.0}])
def test_deferred_with_post_symmetry(renderer, sym):
    cfg = full_with_final_draws(7)
    cfg["flame"]["post_symmetry"] = sym
    job = dict(iterations=8_000_000, walkers=8192)
    a, _, oa = run(renderer, cfg, 200, 150, plot="inline", **job)
    b, _, ob = run(renderer, cfg, 200, 150, plot="deferred", **job)
    assert np.array_equal(a, b) and oa.inframe_samples == ob.inframe_samples


@pytest.mark.gpu
def test_deferred_with_xaos_and_exact_sums(renderer):
    cfg = synthetic.full_flame(9, de_radius=0)
    n = len(cfg["flame"]["transforms"])
    cfg["flame"]["xaos"] = [[(0.3 if i == j else 1.0) for j in range(n)] for i in range(n)]
    job = dict(iterations=10_000_000, walkers=8192, count_bits=64, accumulate="direct")
    a, ra, oa = renderer.histogram_u64(cfg, 256, 256, plot="inline", **job)
    b, rb, ob = renderer.histogram_u64(cfg, 256, 256, plot="deferred", **job)
    assert np.array_equal(a, b) and np.array_equal(ra, rb)            # fixed-point sums: order-independent


@pytest.mark.gpu
def test_deferred_render_is_the_same_image(renderer):
    cfg = synthetic.full_flame(6)                                      # with density estimation
    job = dict(iterations=30_000_000, walkers=16384, supersample=2)
    a, _ = renderer.render(cfg, 320, 180, plot="inline", **job)
    b, _ = renderer.render(cfg, 320, 180, plot="deferred", **job)
    assert np.abs(a.astype(int) - b.astype(int)).max() <= 1           # FP32 colour sums in another order


@pytest.mark.gpu
@pytest.mark.parametrize("walkers,iters", [(16384, 20_000_000), (10000, 9_000_000), (2048, 2048 * 5000), (4096, 4096 * 1),
                                           (4096, 4096 * 2), (33 * 32, 33 * 32 * 9)])
def test_fused_equals_inline(renderer, walkers, iters):
    """The fused kernel walks the same orbits and plots the same samples:
    identical count planes.  Cases: a block of inactive producer threads
    (10,000 walkers), launches of several ring cycles and of 4096+
    iterations (two launches), one and two iterations past the burn-in,
    and a ragged iteration count."""
    cfg = full_with_final_draws()
    job = dict(iterations=iters, walkers=walkers, supersample=2, burn_in=20)
    a, ra, oa = run(renderer, cfg, 320, 180, plot="inline", **job)
    b, rb, ob = run(renderer, cfg, 320, 180, plot="fused", **job)
    assert oa.inframe_samples == ob.inframe_samples == int(a.sum()) > 0
    assert np.array_equal(a, b)
    np.testing.assert_allclose(ra, rb, rtol=1e-4, atol=1e-3)


@pytest.mark.gpu
def test_fused_with_post_symmetry_xaos_and_exact_sums(renderer):
    cfg = full_with_final_draws(7)
    cfg["flame"]["post_symmetry"] = {"ty": "point", "order": 5, "center_x": 0.1, "center_y": 0.0, "distance": 1.25,
                                     "rotation_deg": 0.0}
    job = dict(iterations=8_000_000, walkers=8192)
    a, _, oa = run(renderer, cfg, 200, 150, plot="inline", **job)
    b, _, ob = run(renderer, cfg, 200, 150, plot="fused", **job)
    assert np.array_equal(a, b) and oa.inframe_samples == ob.inframe_samples
    cfg = synthetic.full_flame(9, de_radius=0)
    n = len(cfg["flame"]["transforms"])
    cfg["flame"]["xaos"] = [[(0.3 if i == j else 1.0) for j in range(n)] for i in range(n)]
    job = dict(iterations=10_000_000, walkers=8192, count_bits=64, accumulate="direct")
    a, ra, oa = renderer.histogram_u64(cfg, 256, 256, plot="inline", **job)
    b, rb, ob = renderer.histogram_u64(cfg, 256, 256, plot="fused", **job)
    assert np.array_equal(a, b) and np.array_equal(ra, rb)            # fixed-point sums: order-independent


@pytest.mark.gpu
def test_fused_render_is_the_same_image(renderer):
    cfg = synthetic.full_flame(6)                                      # with density estimation
    job = dict(iterations=30_000_000, walkers=16384, supersample=2)
    a, _ = renderer.render(cfg, 320, 180, plot="deferred", **job)
    b, _ = renderer.render(cfg, 320, 180, plot="fused", **job)
    assert np.abs(a.astype(int) - b.astype(int)).max() <= 1           # FP32 colour sums in another order


@pytest.mark.gpu
def test_plot_bench_plots_the_same_frame(renderer):
    """ffb_plot_bench (each plot launch alone after its chaos launch) makes
    the render's splats: the same plotted samples and in-frame count as the
    deferred histogram, a positive plot time; refused for fused plotting,
    which has no plot kernel of its own."""
    cfg = full_with_final_draws()
    job = dict(iterations=16384 * 600, walkers=16384, plot="deferred")
    cnt, _, o = renderer.histogram(cfg, 320, 200, **job)
    ms, samples, inframe = renderer.plot_bench(cfg, 320, 200, **job)
    assert ms > 0.0
    assert samples == o.total_iterations
    assert inframe == o.inframe_samples == int(cnt.sum())
    with pytest.raises(_native.EngineError, match="deferred plotting"):
        renderer.plot_bench(cfg, 320, 200, iterations=16384 * 600, walkers=16384, plot="fused")
