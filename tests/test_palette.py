"""The palette lookup pipeline (src/scene/palette.rs:485-800): squeeze --
linear repeats (`palette_squeeze`) or geometric octaves of ratio
`palette_squeeze_falloff` (`palette_squeeze_mode`) --, exponential
redistribution (`palette_log_strength`), rotation, reverse.  Each remapping
stage builds entry i of its table from the previous table's entry
min(floor(src_t * size), size - 1), src_t the stage's map of t = i / size.

CPU: the oracle's table against each stage's map computed here in f32
(numpy), one stage at a time and all four in order; the parser's names.
GPU: a render's exact colour sums against the oracle's for a flame whose
palette goes through every stage.
"""

import json

import numpy as np
import pytest

from ffb200 import EngineError
from ffb200 import _native

F = np.float32
RAMP = {"stops": [{"position": 0.0, "color": [0.0, 0.1, 1.0]}, {"position": 0.4, "color": [1.0, 0.2, 0.0]},
                  {"position": 1.0, "color": [0.2, 1.0, 0.6]}]}


def table(oracle, **kw):
    cfg = {"palette": RAMP, "palette_size": 256}
    cfg.update(kw)
    return oracle.palette_table(cfg).reshape(-1, 3)


def src_of(size, fn):
    """The stage's source index of each entry (saturating cast, capped)."""
    out = []
    for i in range(size):
        t = F(i) / F(size)
        st = F(fn(t))
        fi = F(st * F(size))
        out.append(min(0 if not fi > 0 else int(fi), size - 1))
    return np.array(out)


def linear(factor):
    return lambda t: (lambda x: x - np.trunc(x))(F(t * F(factor)))


def geometric(r):
    def g(t):
        r32 = F(r)
        if r32 >= F(0.999):
            return t
        if r32 <= F(0.001):
            return min(max(t / max(r32, F(1e-6)), F(0)), F(1))
        if t <= 0:
            return F(0)
        start, rn = F(0), F(1)
        for _ in range(64):
            width = F(rn * (F(1) - r32))
            end = F(start + width)
            if t < end:
                return F(0) if width <= 0 else min(max(F((t - start) / width), F(0)), F(1))
            start, rn = end, F(rn * r32)
            if rn < F(1e-10):
                return F(1)
        return F(1)
    return g


def redistribute(s):
    s = F(s)
    def g(t):
        if s > 0:
            return min(max(F(np.expm1(F(s * t)) / np.expm1(s)), F(0)), F(1))
        return min(max(F(F(1) - F(np.expm1(F(-s * F(F(1) - t))) / np.expm1(-s))), F(0)), F(1))
    return g


# --------------------------------------------------------------------- CPU --

@pytest.mark.parametrize("factor", [2.0, 3.5, 0.5])
def test_linear_squeeze(oracle, factor):
    base, sq = table(oracle), table(oracle, palette_squeeze=factor)
    np.testing.assert_array_equal(sq, base[src_of(256, linear(factor))])


@pytest.mark.parametrize("r", [0.5, 0.3, 0.8])
def test_geometric_squeeze(oracle, r):
    """Octave n covers t in [1 - r^n, 1 - r^(n+1)) and spans the whole palette."""
    base = table(oracle)
    sq = table(oracle, palette_squeeze_mode="geometric", palette_squeeze_falloff=r, palette_squeeze=7.0)
    np.testing.assert_array_equal(sq, base[src_of(256, geometric(r))])
    if r == 0.5:                                  # first half, next quarter, next eighth
        assert (sq[0] == base[0]).all() and (sq[128] == base[0]).all() and (sq[192] == base[0]).all()


@pytest.mark.parametrize("s", [2.0, -1.5])
def test_log_redistribution(oracle, s):
    base, lg = table(oracle), table(oracle, palette_log_strength=s)
    np.testing.assert_array_equal(lg, base[src_of(256, redistribute(s))])


def test_stage_order(oracle):
    """squeeze, then redistribution, then rotation, then reverse."""
    base = table(oracle)
    got = table(oracle, palette_squeeze=3.0, palette_log_strength=1.0, palette_rotation=0.2, palette_reverse=True)
    a = base[src_of(256, linear(3.0))]
    b = a[src_of(256, redistribute(1.0))]
    amt = round(0.2 * 256)
    c = b[[(i + amt) % 256 for i in range(256)]]
    np.testing.assert_array_equal(got, c[::-1])


def test_squeeze_mode_names():
    cfg = {"flame": {"transforms": [{"a": 1, "b": 0, "c": 0, "d": 1, "e": 0, "f": 0, "weight": 1, "color": 0,
                                     "variations": {"linear": 1.0}}]}, "palette_squeeze_mode": "Geometric"}
    assert _native.specialize(json.dumps(cfg))[0] > 0
    cfg["palette_squeeze_mode"] = "spiral"
    with pytest.raises(EngineError, match="palette squeeze mode"):
        _native.specialize(json.dumps(cfg))


def test_speed_colour_known_answer(oracle):
    """Speed colour mode (main_template.wgsl:483-506, utilities.wgsl:148-156):
    two constant transforms that xaos makes alternate, so every step moves
    |2P| = 1; with speed_factor 1 each sample carries the palette's entry
    at clamp(ln(10 + 1) / 3, 0, 1)."""
    t = [{"a": 0, "b": 0, "c": 0, "d": 0, "e": 0.3 * s, "f": 0.4 * s, "weight": 1.0, "color": 0.0,
          "variations": {"linear": 1.0}} for s in (1.0, -1.0)]
    cfg = {"flame": {"transforms": t, "xaos": [[0, 1], [1, 0]]}, "deterministic_rng": True, "palette": RAMP,
           "color_mode": "speed", "speed_factor": 1.0}
    fl = oracle.Flame(cfg, 64, 48)
    _, inframe, cnt, rgb = fl.render(256, 100, threads=4)
    lit = np.argwhere(cnt > 0)
    assert len(lit) == 2
    speed = F(np.sqrt(F(F(0.6) * F(0.6)) + F(F(0.8) * F(0.8))))
    entry = table(oracle)[int(np.floor(F(np.log(F(speed * F(10)) + F(1)) / F(3)) * F(256)))]
    for y, x in lit:
        np.testing.assert_allclose(rgb[y, x] / cnt[y, x], entry, rtol=1e-6)


def test_speed_mode_names():
    cfg = {"flame": {"transforms": [{"a": 1, "b": 0, "c": 0, "d": 1, "e": 0, "f": 0, "weight": 1, "color": 0,
                                     "variations": {"linear": 1.0}}]}, "color_mode": "Speed"}
    _, src = _native.specialize(json.dumps(cfg))
    assert "#define FFB_SPEED 1" in src
    cfg["color_mode"] = "PathMap"
    with pytest.raises(EngineError, match="colour mode"):
        _native.specialize(json.dumps(cfg))


# --------------------------------------------------------------------- GPU --

@pytest.mark.gpu
@pytest.mark.parametrize("rng_mode", ["philox", "pcg"])
def test_speed_colour_render(renderer, oracle, rng_mode):
    """A linear flame in speed colour mode: the same counts as the oracle,
    bit for bit, and the same colour sums but where a log's last bit moved
    a step's speed across a palette entry (rare; the colour then differs by
    one entry, mixed in by speed_factor)."""
    t = [{"a": 0.5, "b": 0, "c": 0, "d": 0.5, "e": e, "f": f, "weight": w, "color": 0.0,
          "variations": {"linear": 1.0}} for e, f, w in ((0.0, 0.5, 1.0), (-0.5, -0.5, 0.7), (0.5, -0.5, 1.3))]
    cfg = {"flame": {"transforms": t}, "deterministic_rng": True, "palette": RAMP, "color_mode": "speed",
           "speed_factor": 0.3}
    W, H, walkers, per = 96, 64, 2048, 300
    cnt, rgb, out = renderer.histogram_u64(cfg, W, H, iterations=walkers * per, walkers=walkers, count_bits=64,
                                           rng=rng_mode, iterations_per_thread=256)
    fl = oracle.Flame(cfg, W, H)
    _, inframe, rc, rrgb = fl.render(walkers, per + 20, rng=rng_mode, ipt=256, threads=8)
    assert np.array_equal(cnt.astype(np.int64), rc.astype(np.int64)) and inframe == out.inframe_samples
    lit = cnt > 0
    close = np.isclose(rgb[lit], rrgb[lit], rtol=1e-4, atol=1e-4).all(axis=1)
    assert close.mean() > 0.99, close.mean()


@pytest.mark.gpu
def test_render_colours_go_through_the_pipeline(renderer, oracle):
    """A linear flame (bit-identical orbits) with exact colour sums: each
    pixel's sum is its samples' palette entries, the palette through every
    stage."""
    t = [{"a": 0.5, "b": 0, "c": 0, "d": 0.5, "e": e, "f": f, "weight": 1.0, "color": c, "color_speed": 0.2,
          "variations": {"linear": 1.0}} for e, f, c in ((0.0, 0.5, 0.0), (-0.5, -0.5, 0.45), (0.5, -0.5, 0.9))]
    cfg = {"flame": {"transforms": t}, "deterministic_rng": True, "palette": RAMP,
           "palette_squeeze_mode": "geometric", "palette_squeeze_falloff": 0.4, "palette_log_strength": -0.8,
           "palette_rotation": 0.1, "palette_reverse": True}
    W, H, walkers, per = 96, 64, 2048, 400
    cnt, rgb, out = renderer.histogram_u64(cfg, W, H, iterations=walkers * per, walkers=walkers, count_bits=64)
    fl = oracle.Flame(cfg, W, H)
    _, inframe, rc, rrgb = fl.render(walkers, per + 20, threads=8)
    assert np.array_equal(cnt.astype(np.int64), rc.astype(np.int64)) and inframe == out.inframe_samples
    # The exact sums round each sample's colour to a multiple of 2^-24 (the
    # same way for the same palette entry): a pixel's sum is within its
    # count x 2^-25 of the oracle's, plus the f32 of the result.
    bound = cnt.astype(np.float64)[..., None] * 2.0 ** -25 + 2e-7 * np.abs(rrgb) + 1e-9
    assert (np.abs(rgb.astype(np.float64) - rrgb) <= bound).all()
