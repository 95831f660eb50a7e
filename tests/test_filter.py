"""The spatial filter (Apophysis `filter`: shaders/histogram_blur.wgsl:17-119,
src/renderer/compute_kernel.rs:1663-1725): a separable bilateral Gaussian
on each batch's histogram, spatial sigma `filter_radius` pixels (taps
within min(ceil(3 sigma), 8), edges clamped), density sigma from the
batch's mean density x 100^(2 filter_blur_edges - 1), the centre density
of both passes the unfiltered batch's; each filtered batch is added into
the render's histogram.

CPU: the oracle's filter against properties the definition implies.
GPU: the kernel against the oracle (FP32 both; 1e-5 relative), and a
whole filtered render of a linear-only flame (identical orbits, so
identical batch histograms) against the oracle's batch-by-batch render.
"""

import json

import numpy as np
import pytest

from ffb200 import Engine, EngineError, synthetic
from ffb200 import _native


def random_batch(seed, h=48, w=64, fill=0.3):
    rng = np.random.default_rng(seed)
    cnt = (rng.random((h, w)) < fill) * rng.integers(1, 40, (h, w))
    rgb = rng.random((h, w, 3)).astype(np.float32) * cnt[..., None]
    return cnt.astype(np.uint32), rgb.astype(np.float32)


def rgbc(cnt, rgb):
    return np.concatenate([rgb, cnt[..., None].astype(np.float32)], axis=2)


# --------------------------------------------------------------------- CPU --

def test_uniform_histogram_is_unchanged(oracle):
    cnt = np.full((20, 30), 7, np.uint32)
    rgb = np.full((20, 30, 3), 3.5, np.float32)
    out = oracle.hist_filter(rgbc(cnt, rgb), 1.5, 0.05)
    np.testing.assert_allclose(out[..., 3], 7.0, rtol=1e-6)
    np.testing.assert_allclose(out[..., :3], 3.5, rtol=1e-6)


def test_loose_density_sigma_is_a_plain_gaussian(oracle):
    """With sigma_d far above every density difference the bilateral weight
    is 1: a separable, normalised Gaussian with clamped edges."""
    cnt, rgb = random_batch(1)
    sigma = 1.2
    out = oracle.hist_filter(rgbc(cnt, rgb), sigma, 1e9)
    kh = min(int(np.ceil(3 * sigma)), 8)
    k = np.exp(-np.arange(-kh, kh + 1) ** 2 / (2 * sigma * sigma))
    k /= k.sum()
    def conv(a, axis):
        n = a.shape[axis]
        out = np.zeros_like(a, dtype=np.float64)
        for j, wj in zip(range(-kh, kh + 1), k):
            idx = np.clip(np.arange(n) + j, 0, n - 1)
            out += wj * np.take(a, idx, axis=axis)
        return out
    ref = conv(conv(cnt.astype(np.float64), 1), 0)
    np.testing.assert_allclose(out[..., 3], ref, rtol=2e-5, atol=1e-4)


def test_tight_density_sigma_keeps_an_isolated_pixel(oracle):
    """Edge preservation: a lone bright pixel among empty ones keeps its
    count and lends none to its neighbours."""
    cnt = np.zeros((15, 15), np.uint32)
    cnt[7, 7] = 100
    rgb = np.zeros((15, 15, 3), np.float32)
    rgb[7, 7] = (50, 20, 10)
    out = oracle.hist_filter(rgbc(cnt, rgb), 2.0, 0.05)
    assert abs(out[7, 7, 3] - 100) < 1e-3
    assert np.abs(np.delete(out[..., 3].ravel(), 7 * 15 + 7)).max() < 1e-6


def test_filtered_configs_parse_and_specialize():
    cfg = synthetic.plain_flame(1)
    cfg["filter_radius"] = 0.5
    cfg["filter_blur_edges"] = 0.3
    n, _ = _native.specialize(json.dumps(cfg))
    assert n > 0
    xml = ('<flames><flame name="F" size="64 48" center="0 0" scale="40" filter="0.5">'
           '<xform weight="1" color="0" spherical="1" coefs="0.9 0 0 0.9 0 0"/>'
           '<xform weight="1" color="1" linear="1" coefs="0.5 0 0 0.5 0.5 0"/></flame></flames>')
    imported = _native.flame_import(xml)[0]
    assert imported["filter_radius"] == 0.5
    assert _native.specialize(json.dumps(imported))[0] > 0


# --------------------------------------------------------------------- GPU --

@pytest.mark.gpu
@pytest.mark.parametrize("sigma,sigma_d", [(0.5, 0.05), (1.3, 1.0), (3.0, 100.0), (8.0, 5.0)])
def test_filter_kernel_matches_oracle(renderer, oracle, sigma, sigma_d):
    cnt, rgb = random_batch(int(sigma * 10 + sigma_d))
    got = renderer.hist_filter(cnt, rgb, sigma, sigma_d)
    ref = oracle.hist_filter(rgbc(cnt, rgb), sigma, sigma_d)
    np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-5 * max(1.0, float(ref.max())))


@pytest.mark.gpu
@pytest.mark.parametrize("blur_edges", [0.0, 0.5, 1.0])
def test_filtered_render_matches_oracle(renderer, oracle, blur_edges):
    """A linear-only flame: the GPU walks the oracle's orbits, batch by batch
    (ipt 256 iterations), so each batch histogram is the same and so is its
    filter."""
    cfg = synthetic.sierpinski()
    cfg["filter_radius"] = 0.9
    cfg["filter_blur_edges"] = blur_edges
    W, H, walkers, per, ipt = 96, 64, 2048, 4 * 256 - 20, 256
    cnt, rgb, out = renderer.histogram_f32(cfg, W, H, iterations=walkers * per, walkers=walkers,
                                           iterations_per_thread=ipt, rng="philox")
    fl = oracle.Flame(cfg, W, H)
    plotted, inframe, ref = fl.render_filtered(walkers, per + 20, 0.9, blur_edges, ipt=ipt, threads=8)
    assert out.total_iterations == plotted and out.inframe_samples == inframe
    scale = max(1.0, float(ref[..., 3].max()))
    np.testing.assert_allclose(cnt, ref[..., 3], rtol=1e-4, atol=1e-5 * scale)
    np.testing.assert_allclose(rgb, ref[..., :3], rtol=1e-3, atol=1e-4 * scale)
    # Total mass stays within a few percent of the unfiltered count (normalised kernel).
    assert abs(cnt.sum() - inframe) < 0.05 * inframe


@pytest.mark.gpu
def test_imported_apophysis_flame_with_filter_renders():
    xml = ('<flames><flame name="F" size="96 64" center="0 0" scale="60" filter="0.5" brightness="3">'
           '<xform weight="1" color="0" spherical="1" coefs="0.9 0 0 0.9 0 0"/>'
           '<xform weight="1" color="1" linear="1" julian="0.4" julian_power="3" coefs="0.5 0 0 0.5 0.5 0"/>'
           '</flame></flames>')
    e = Engine()
    cfg = e.flame_import(xml)[0]
    img = e.render(cfg, 96, 64, iterations=2_000_000, iterations_per_thread=256)
    px = np.frombuffer(img.rgba, np.uint8).reshape(64, 96, 4)
    assert px[..., :3].max() > 0


@pytest.mark.gpu
def test_filter_is_refused_where_it_is_not_built(renderer):
    cfg = synthetic.plain_flame(1)
    cfg["filter_radius"] = 0.5
    with pytest.raises(EngineError, match="fractional"):
        renderer.histogram(cfg, 32, 32, iterations=10000)
    with pytest.raises(EngineError, match="filter"):
        renderer.histogram_u64(cfg, 32, 32, iterations=10000)
