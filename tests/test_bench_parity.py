"""Parity of the benchmarked path with the oracle: the 1920x1080 ss2
workload's flame (8 transforms + a final, 3-5 of the twelve variations
each, density estimation radius 9) through the path the benchmark times --
the transform-sorted chaos kernel with deferred plotting (the counter-based
stream over 65,536 walkers, so the automatic plan defers) -- at a reduced
size and budget that keep the benchmark's samples a pixel.

The flame's variations take transcendental arithmetic, so the GPU's orbits
(CUDA's libm) and the oracle's (glibc's) part after a few dozen steps and
the comparison is at Monte-Carlo noise: GPU against an oracle render within
1.25x of two oracle renders against each other, on the normalised
log-density (L1 and 99th percentile), on 16x16-block z-scores, and on the
tone-mapped RGBA8 image after density estimation (oracle/parity.py).
Reference semantics: shaders/core/main_template.wgsl:20-1428; the density
comparison follows src/renderer/density_gates.rs:24-119 in spirit (a
log-density gate at a stated sample count).
"""

import json

import pytest

import bench
from ffb200 import _native

SIZE = (480, 270)          # output pixels; 960x540 internal at ss 2
WALKERS = 65536


def bench_job():
    wl = bench.workload("full_1080p_ss2")
    spp = wl["iterations"] / float(wl["width"] * wl["supersample"] * wl["height"] * wl["supersample"])
    samples = int(spp * SIZE[0] * SIZE[1] * wl["supersample"] ** 2)
    return wl, samples


def test_benchmark_flame_is_planned_deferred_and_sorted():
    """The reduced case takes the benchmark's plan: deferred plotting on the
    sorted schedule (the counter-based stream, >= 16,384 walkers)."""
    wl, _ = bench_job()
    _, src = _native.specialize_job(wl["cfg"], walkers=WALKERS, width=SIZE[0], height=SIZE[1], supersample=2)
    assert "#define FFB_DEFER 1" in src


@pytest.mark.gpu
def test_benchmark_flame_within_monte_carlo_noise(renderer):
    from oracle import parity
    wl, samples = bench_job()
    m = parity.render_parity(renderer, wl["cfg"], SIZE[0], SIZE[1], 2, samples, WALKERS)
    # The plot kernels ran: a chaos and a plot launch a 256-iteration chunk.
    chunks = -(-(samples // WALKERS + 1 + 20) // 256)
    assert m["kernel_launches"] >= 2 * chunks, m
    assert abs(m["samples_per_px"] - wl["iterations"] / (3840 * 2160)) < 1.0
    assert m["inframe"] > 0.2 * m["samples"]
    assert parity.within_noise(m), json.dumps(m)
