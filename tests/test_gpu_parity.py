"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Tolerances:
* per-step iterate, per variation: <= 4 ulp FP32 (cancellations: 4 ulp of
  the terms' magnitude);
* histograms: bit-exact counts for a linear-only flame (no transcendental
  arithmetic, identical orbits); otherwise normalised log-density within
  the Monte-Carlo noise measured between two oracle renders;
* tone map and density estimation: 1e-5 relative of the FP64 oracle.
"""

import json
import math

import numpy as np
import pytest

from ffb200 import synthetic

pytestmark = pytest.mark.gpu

TWELVE = synthetic.TWELVE
PROBE_PTS = None


def ulp_dist(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    a = np.where(a < 0, -(a & 0x7FFFFFFF), a)
    b = np.where(b < 0, -(b & 0x7FFFFFFF), b)
    return np.abs(a - b)


EXACT = {"linear", "spherical", "horseshoe", "bubble", "curl"}   # no transcendental arithmetic
ULPS = 4
EPS = 2.0 ** -23


def within(gpu, ref, scale):
    """<= 4 ulp of the result, or <= 4 ulp of the magnitude of the terms the
    result was summed from (`scale`, from the oracle): a cancellation's
    error is a few ulp of its terms.  NaN and infinities must agree."""
    gpu = np.asarray(gpu, np.float32)
    ref = np.asarray(ref, np.float32)
    finite = np.isfinite(gpu) & np.isfinite(ref)
    same_special = (np.isnan(gpu) & np.isnan(ref)) | (~np.isnan(gpu) & ~np.isnan(ref) & ~finite & (gpu == ref))
    ok_ulp = ulp_dist(np.where(finite, gpu, 0), np.where(finite, ref, 0)) <= ULPS
    diff = np.abs(np.where(finite, gpu, 0).astype(np.float64) - np.where(finite, ref, 0))
    ok_scale = diff <= ULPS * EPS * np.asarray(scale, np.float64)
    return np.where(finite, ok_ulp | ok_scale, same_special)


def bit_equal(gpu, ref):
    g = np.asarray(gpu, np.float32)
    r = np.asarray(ref, np.float32)
    return (g.view(np.uint32) == r.view(np.uint32)) | (np.isnan(g) & np.isnan(r))


def one_xform(name, a=(1, 0, 0, 1, 0, 0), params=None):
    t = {"a": a[0], "b": a[1], "c": a[2], "d": a[3], "e": a[4], "f": a[5], "weight": 1.0, "color": 0.5,
         "variations": {name: 1.0}}
    if params:
        t["variation_params"] = params
    return {"flame": {"transforms": [t]}, "deterministic_rng": True}


@pytest.fixture(scope="module")
def pts(oracle):
    _, _, _ = oracle.probe("linear")
    # The 27 probe inputs (src/probe/inputs.rs:49-77), as the oracle holds them.
    vals = []
    for x, y in [(0.0, 0.0), (0.0, -0.0), (-0.0, 0.0), (-0.0, -0.0), (1, 0), (-1, 0), (0, 1), (0, -1), (1, 1), (-1, 1),
                 (-1, -1), (1, -1), (0.5, 0.3), (0.12345679, -0.9876543), (2.5, -1.5), (math.pi, math.e), (1, 0),
                 (0.70710677, 0.70710677), (1e-20, -1e-20), (1.1754944e-38, 1.1754944e-38), (1e-40, -1e-40),
                 (1e20, -1e20), (9e31, -9e31), (1e33, -1e33), (1e30, 1e-30), (1.0, -0.0), (-0.0, 1.0)]:
        vals += [x, y]
    return np.array(vals, np.float32).reshape(-1, 2)


@pytest.mark.parametrize("name", TWELVE)
def test_probe_matches_oracle(renderer, oracle, pts, name):
    """The variation probe at the 27 inputs: CUDA (precise math) vs the oracle,
    both at probe slot 0 (RNG rng_init(point, 0x9E3779B9)).  Variations with
    no transcendental arithmetic are bit-identical; the others within 4 ulp
    (of the terms, where the result cancels)."""
    out = renderer.probe(one_xform(name), pts, 1)[0]
    _, _, ref = oracle.probe(name, xform_slot=0, fold_first=False)
    ref = ref.reshape(27, 2)
    if name in EXACT:
        ok = bit_equal(out, ref)
    else:
        flushed = np.where(np.abs(pts) < 1.17549435e-38, np.copysign(0.0, pts), pts).astype(np.float32)
        draws = np.array([oracle.probe_draw(i) for i in range(27)], np.float32)
        sx, sy = oracle.variation_scale(name, flushed[:, 0], flushed[:, 1], draws if name == "julia" else None)
        ok = within(out, ref, np.stack([sx, sy], axis=1))
    bad = [(i, pts[i].tolist(), out[i].tolist(), ref[i].tolist()) for i in range(27) if not ok[i].all()]
    assert not bad, f"{name}: {bad}"


def test_probe_sfu_math_reproduces_reference_classes(renderer, oracle, pts):
    """With the hardware's approximate sin/cos (math = sfu) the CUDA probe
    reproduces the reference GPU's class glyphs at every input, including
    those where IEEE sin differs (tests/golden/variation_probe_2d.txt)."""
    import os
    GOLDEN = {}
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "variation_probe_2d.txt")) as f:
        for line in f:
            if not line.startswith("#") and line.strip():
                n, c, d, slot = line.split()
                GOLDEN[n] = (c, int(d, 16), int(slot))
    mism = {}
    for name in TWELVE:
        slot = GOLDEN[name][2]
        # Place the variation at its probe-batch transform so julia's draw matches.
        cfg = {"flame": {"transforms": [one_xform(name)["flame"]["transforms"][0]] * (slot + 1)}}
        out = renderer.probe(cfg, pts, slot + 1, math="sfu")[slot].reshape(-1)
        classes, _ = oracle.probe_digest(out)
        gold = GOLDEN[name][0]
        if name == "linear":
            # signed zeros: the reference compiler folded 0 + x into x for the batch's first variation
            gold = gold.replace("o", "0")
            classes = classes.replace("o", "0")
        diff = [i for i in range(54) if classes[i] != gold[i]]
        if diff:
            mism[name] = (classes, gold, diff)
    assert len(mism) <= 2, mism


def test_apply_points_matches_oracle(renderer, oracle):
    """Single step of every transform of a flame using all twelve variations
    (affine, weighted variation sum, post-affine; finals too) at 4096 random
    points with random draws: within 4 ulp (of the terms, where they cancel);
    a transform of non-transcendental variations only is bit-identical."""
    rng = np.random.default_rng(5)
    t1 = {"a": 0.7, "b": -0.3, "c": 0.4, "d": 0.9, "e": 0.1, "f": -0.2, "weight": 1.0, "color": 0.1,
          "variations": {n: float(rng.uniform(0.1, 1.0)) for n in TWELVE[:6]},
          "variation_params": {"curl.c1": 0.7, "curl.c2": 0.2}}
    t2 = {"a": -0.5, "b": 0.6, "c": 0.3, "d": 0.2, "e": -0.4, "f": 0.3, "weight": 2.0, "color": 0.9,
          "post_affine_enabled": True, "post_a": 0.9, "post_b": 0.1, "post_c": -0.2, "post_d": 1.1, "post_e": 0.05,
          "post_f": 0.0, "variations": {n: float(rng.uniform(0.1, 1.0)) for n in TWELVE[6:]},
          "variation_params": {"curl.c1": 0.4, "curl.c2": -0.3}}
    t3 = {"a": 0.3, "b": 0.2, "c": -0.6, "d": 0.4, "e": 0.2, "f": 0.1, "weight": 1.0, "color": 0.5,
          "variations": {n: float(rng.uniform(0.1, 1.0)) for n in sorted(EXACT)},
          "variation_params": {"curl.c1": 0.3, "curl.c2": 0.1}}
    fin = {"a": 1.0, "b": 0.1, "c": -0.1, "d": 1.0, "e": 0.0, "f": 0.0, "weight": 1.0, "color": 0.0,
           "variations": {"julia": 0.5, "swirl": 0.3, "disc": 0.2}}
    cfg = {"flame": {"transforms": [t1, t2, t3], "final_transform": fin}}
    fl = oracle.Flame(cfg, 64, 64)
    n = 4096
    xs = rng.uniform(-2.5, 2.5, n).astype(np.float32)
    ys = rng.uniform(-2.5, 2.5, n).astype(np.float32)
    words = (rng.integers(0, 1 << 24, (n, 64)) / float(1 << 24)).astype(np.float32)
    for xi in range(4):
        for aff in (True, False):
            gx, gy = renderer.apply_points(cfg, xi, xs, ys, words, with_affine=aff)
            rx, ry, sx, sy = fl.apply_xform(xi, xs, ys, words, with_affine=aff, scales=True)
            if xi == 2:
                ok = bit_equal(gx, rx) & bit_equal(gy, ry)
            else:
                ok = within(gx, rx, sx) & within(gy, ry, sy)
            bad = np.where(~ok)[0]
            assert len(bad) == 0, (xi, aff, [(xs[i], ys[i], gx[i], rx[i], gy[i], ry[i], sx[i], sy[i]) for i in bad[:5]])


@pytest.mark.parametrize("rng_mode", ["pcg", "philox"])
def test_histogram_bit_exact_for_a_linear_flame(renderer, oracle, rng_mode):
    """No transcendentals: the GPU walks the oracle's orbits exactly, so the
    count plane is identical, pixel for pixel, and sums to the in-frame count."""
    cfg = synthetic.sierpinski()
    W, H = 96, 64
    job = dict(iterations=2048 * 700, walkers=2048, rng=rng_mode, iterations_per_thread=256)
    cnt, rgb, out = renderer.histogram(cfg, W, H, **job)
    fl = oracle.Flame(cfg, W, H)
    plotted, inframe, rc, rr = fl.render(2048, 700 + 20, rng=rng_mode, ipt=256, threads=8)
    assert out.total_iterations == plotted == 2048 * 700
    assert int(cnt.sum()) == out.inframe_samples == inframe
    assert np.array_equal(cnt, rc)
    # Colour sums: FP32 atomics in any order vs an f64 sum of the same
    # values: within n * 2^-24 of the sum's magnitude.
    tol = cnt[..., None].astype(np.float64) * 2.0 ** -24 * np.maximum(rr, 1.0) + 1e-6
    assert np.all(np.abs(rgb - rr) <= tol)


def test_sorted_schedule_walks_the_same_orbits(renderer):
    """The transform-sorted schedule moves walkers between threads but keeps
    each walker's stream: the count plane is identical to one walker a
    thread, for a flame with every variation, a final and 2x supersampling."""
    from ffb200 import synthetic as S
    cfg = S.full_flame(6, de_radius=0)
    job = dict(iterations=3_000_000, walkers=6000, supersample=2)
    a, ra, oa = renderer.histogram(cfg, 160, 90, schedule="plain", **job)
    b, rb, ob = renderer.histogram(cfg, 160, 90, schedule="sorted", **job)
    assert np.array_equal(a, b)
    assert oa.inframe_samples == ob.inframe_samples == int(a.sum())
    np.testing.assert_allclose(ra, rb, rtol=1e-4, atol=1e-3)
    for rng in ("pcg", "philox"):
        a, _, _ = renderer.histogram(cfg, 160, 90, schedule="plain", rng=rng, iterations_per_thread=64, **job)
        b, _, _ = renderer.histogram(cfg, 160, 90, schedule="sorted", rng=rng, iterations_per_thread=64, **job)
        assert np.array_equal(a, b), rng


def log_density_l1(a, b):
    la, lb = np.log1p(a.astype(np.float64)), np.log1p(b.astype(np.float64))
    lit = (a > 0) | (b > 0)
    d = np.abs(la - lb)[lit]
    return d.mean(), np.percentile(d, 99)


@pytest.mark.parametrize("seed", [1, 2])
def test_histogram_density_within_monte_carlo_noise(renderer, oracle, seed):
    """A plain 3-transform flame (linear/sinusoidal/spherical): the GPU's
    normalised log-density differs from the oracle's by no more than two
    independent oracle renders differ (L1 and 99th percentile)."""
    cfg = synthetic.plain_flame(seed)
    W = H = 128
    walkers, per = 8192, 400
    cnt, _, out = renderer.histogram(cfg, W, H, iterations=walkers * per, walkers=walkers, seed=1001)
    fl = oracle.Flame(cfg, W, H)
    _, _, o1, _ = fl.render(walkers, per + 20, seed=1001, threads=8)
    _, _, o2, _ = fl.render(walkers, per + 20, seed=2002, threads=8)
    if o1.sum() < 1000:
        pytest.skip("flame lights too little of the frame")
    l1_go, p99_go = log_density_l1(cnt, o1)
    l1_oo, p99_oo = log_density_l1(o2, o1)
    assert l1_go <= 1.25 * l1_oo + 0.01, (l1_go, l1_oo)
    assert p99_go <= 1.25 * p99_oo + 0.05, (p99_go, p99_oo)
    # 16x16-block densities: |z| > 5 blocks no more than between the oracle's replicates.
    def blocks(c):
        return c.reshape(H // 16, 16, W // 16, 16).sum(axis=(1, 3)).astype(np.float64)
    bg, b1, b2 = blocks(cnt), blocks(o1), blocks(o2)
    se = np.sqrt(np.maximum(b1 + b2, 1.0))
    assert (np.abs(bg - b1) / se > 5).sum() <= max(2, (np.abs(b2 - b1) / se > 5).sum() + 2)


def tonemap_params(oracle, cfg, w, h, sd, transparent=0):
    return oracle.tonemap_params_for(cfg, w, h, sd, transparent)


TONEMAP_VARIANTS = [
    {},
    {"vibrancy": 0.5, "gamma": 2.2, "gamma_threshold": 0.01},
    {"saturation": 1.5, "hue_shift": 40.0, "highlight_mode": "max_norm"},
    {"highlight_mode": "reinhard", "exposure": 3.0, "levels_enabled": False},
    {"highlight_mode": "filmic", "background_color": [0.2, 0.1, 0.05]},
    {"tonemap_mode": "linear", "gamma": 2.0},
    {"tonemap_mode": "density", "exposure": 0.5},
    {"highlight_mode": "agx", "exposure": 2.0},
    {"highlight_mode": "agx_punchy", "saturation": 1.2},
]


@pytest.fixture(scope="module")
def c1_hist(renderer):
    cfg = synthetic.plain_flame(3)
    cnt, rgb, out = renderer.histogram(cfg, 128, 128, iterations=2_000_000, seed=77)
    return cfg, cnt, rgb, out


@pytest.mark.parametrize("variant", range(len(TONEMAP_VARIANTS)))
@pytest.mark.parametrize("transparent", [0, 1, 2])
def test_tonemap_matches_f64_oracle(renderer, oracle, c1_hist, variant, transparent):
    base, cnt, rgb, out = c1_hist
    cfg = dict(base, **TONEMAP_VARIANTS[variant])
    h, w = cnt.shape
    sd = out.total_iterations / (w * h)
    u8, f = renderer.tonemap(cfg, cnt.astype(np.float32), rgb, sd, ss=1, transparent=transparent, want_float=True)
    P = tonemap_params(oracle, cfg, w, h, sd, transparent)
    rf, ru = oracle.tonemap(P, cnt.astype(np.float64), rgb.astype(np.float64))
    f = f.reshape(-1, 4).astype(np.float64)
    err = np.abs(f - rf) / np.maximum(np.abs(rf), 1e-3)
    assert err.max() <= 1e-5, (variant, transparent, float(err.max()), np.unravel_index(err.argmax(), err.shape))
    # 8-bit output: equal except where the value sits on a rounding tie.
    d = np.abs(u8.reshape(-1, 4).astype(int) - ru.astype(int))
    frac = np.abs(rf * 255 - np.floor(rf * 255))
    assert d.max() <= 1
    assert np.all((d == 0) | (np.abs(frac - 0.5) < 1e-4))


def test_supersample_downsample_matches_oracle(renderer, oracle, c1_hist):
    """ss 2: the fused tone map + firefly box vs the oracle's tone map, 8-bit
    quantisation and supersample.rs:132-167."""
    cfg, cnt, rgb, out = c1_hist
    h, w = cnt.shape
    sd = out.total_iterations / (w * h)
    u8 = renderer.tonemap(cfg, cnt.astype(np.float32), rgb, sd, ss=2)
    P = tonemap_params(oracle, cfg, w, h, sd)
    _, ru = oracle.tonemap(P, cnt.astype(np.float64), rgb.astype(np.float64))
    ref = oracle.downsample_firefly(ru.reshape(h, w, 4), w // 2, h // 2)
    d = np.abs(u8.astype(int) - ref.astype(int))
    assert d.max() <= 1 and (d > 0).mean() < 0.002


@pytest.mark.parametrize("radius", [3.0, 9.0, 18.0])
def test_density_estimation_matches_f64_oracle(renderer, oracle, radius):
    cfg = synthetic.plain_flame(3)
    cnt, rgb, _ = renderer.histogram(cfg, 96, 80, iterations=150_000, seed=5)
    gc, grgb = renderer.density_estimate(cnt, rgb, radius, 0.0, 0.4)
    oc, orgb = oracle.density_estimate(cnt, rgb, 96, 80, radius, 0.0, 0.4)
    # Conservation: DE moves density, it does not make or lose it (away from the edges).
    assert abs(gc.sum() - cnt.sum()) / cnt.sum() < 0.05
    scale = max(oc.max(), 1.0)
    assert np.max(np.abs(gc - oc) / np.maximum(np.abs(oc), 1e-3 * scale)) <= 1e-5
    assert np.max(np.abs(grgb - orgb) / np.maximum(np.abs(orgb), 1e-3 * max(orgb.max(), 1.0))) <= 1e-5


def test_point_render_known_answer(renderer):
    """compute_kernel.rs:6502-6511 through the CUDA path: at 64x64 a point at
    x = -1.96875 lights column 0 of the middle row alone; -2.03125 lights nothing."""
    for x, lit in ((-1.96875, 1), (-2.03125, 0)):
        cfg = {"flame": {"transforms": [{"a": 0, "b": 0, "c": 0, "d": 0, "e": x, "f": 0, "weight": 1, "color": 0.5,
                                         "color_speed": 0.5, "variations": {"linear": 1.0}}]}, "deterministic_rng": True}
        cnt, _, out = renderer.histogram(cfg, 64, 64, iterations=200_000)
        assert int((cnt > 0).sum()) == lit
        if lit:
            assert cnt[32, 0] == out.inframe_samples == out.total_iterations
        img, o = renderer.render(cfg, 64, 64, iterations=200_000)
        assert int((img[..., :3].max(axis=2) > 0).sum()) == lit


def test_render_counts_what_it_plotted(renderer):
    """render.rs:598-708: the render stops on plotted samples and reports them."""
    cfg = synthetic.plain_flame(2)
    _, o = renderer.render(cfg, 32, 32, iterations=4_000_000, iterations_per_thread=16, burn_in=30)
    assert o.total_iterations >= 4_000_000


def test_errors_are_reported_not_raised_on_the_device(renderer, native):
    t = synthetic.plain_flame(1)["flame"]["transforms"][0]
    with pytest.raises(native.EngineError) as e:
        renderer.render({"flame": {"transforms": [t] * 129}}, 16, 16, iterations=1000)
    assert e.value.status == native.ERR_TOO_LARGE and "129" in str(e.value)
    with pytest.raises(native.EngineError) as e:
        renderer.render(synthetic.plain_flame(1), 0, 16)
    assert e.value.status == native.ERR_INVALID
    with pytest.raises(native.EngineError) as e:
        renderer.render('{"flame": ', 16, 16)
    assert e.value.status == native.ERR_CONFIG
    # The renderer still works after refusing.
    img, _ = renderer.render(synthetic.plain_flame(1), 16, 16, iterations=10_000)
    assert img.shape == (16, 16, 4)


def test_engine_renders_like_pyfae():
    """python/tests/test_render.py:34-41, 52-57 against the drop-in Engine."""
    import ffb200
    eng = ffb200.Engine()
    cfg = synthetic.plain_flame(3)
    image = eng.render(cfg, 160, 120, iterations=5_000_000)
    assert (image.width, image.height) == (160, 120)
    assert len(image.rgba) == 160 * 120 * 4
    assert image.info["iterations"] >= 5_000_000
    assert image.info["iterations_per_thread"] == 1024
    lit = int((image.array()[..., :3].max(axis=2) > 0).sum())
    assert lit > 1000
    again = ffb200.Engine().render(cfg, 160, 120, iterations=5_000_000)
    a, b = image.array().astype(int), again.array().astype(int)
    # Counts are exact; FP32 colour sums may round in another order.
    assert np.abs(a - b).max() <= 1 and (a != b).mean() < 0.01


def test_exact_u64_counts_carry_past_2_32(renderer):
    """compute_kernel.rs:6996-7072 (exact u64 count, carry into the high
    word) through the render: every sample of a point flame lands in one
    pixel, 65,536 x 65,537 = 2^32 + 65,536 of them.  With count_bits 64 the
    count is exact and the mean colour stays the palette entry's."""
    cfg = {"flame": {"transforms": [{"a": 0, "b": 0, "c": 0, "d": 0, "e": 0.25, "f": -0.25, "weight": 1, "color": 0.7,
                                     "color_speed": 0.0, "variations": {"linear": 1.0}}]}, "deterministic_rng": True}
    n = 65536 * 65537
    cnt, rgb, out = renderer.histogram_u64(cfg, 16, 16, iterations=n, walkers=65536)
    assert out.total_iterations == n
    lit = np.argwhere(cnt > 0)
    assert len(lit) == 1
    y, x = lit[0]
    assert int(cnt[y, x]) == n == out.inframe_samples
    assert n > 2 ** 32
    # Every plotted sample carries one palette entry (the colour index has
    # converged to 0.7 after the burn-in): the exact sums give its colour.
    import sys, os
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from oracle import oracle as O
    entry = O.palette_table(cfg).reshape(-1, 3)[int(np.floor(np.float32(0.7) * 256))]
    mean = rgb[y, x].astype(np.float64) / n
    np.testing.assert_allclose(mean, entry, rtol=2e-6)


@pytest.mark.parametrize("schedule", ["sorted", "plain"])
def test_batch_matches_single_renders(renderer, schedule):
    """A batch of flames of different transform counts and sizes, one
    launch, graph-replayed: each flame's picture is the single render of the
    same walkers and budget (the streams are keyed by walker and seed), with
    either kernel schedule."""
    from ffb200 import Batch
    items = synthetic.batch_flames(n=12, seed=5, spp=(20, 60), sizes=(64, 96, 128))
    b = Batch(renderer, items, tune=False, threads=128, iterations_per_thread=256, schedule=schedule)
    info = b.info()
    assert info["groups"] == 1 and info["threads"] == 128
    ms = b.run()
    assert ms > 0
    b.run()                                   # replays give the same pictures
    for k, (cfg, w, h, samples, seed) in enumerate(items):
        img, plotted = b.output(k)
        walkers, per = Batch.walkers_for(samples, 128, 256)
        assert plotted == walkers * per >= samples
        ref, o = renderer.render(cfg, w, h, iterations=walkers * per, walkers=walkers, seed=seed, schedule=schedule,
                                 threads=128)
        assert o.total_iterations == plotted
        d = np.abs(img.astype(int) - ref.astype(int))
        assert d.max() <= 1 and (d > 0).mean() < 0.01, (k, d.max(), (d > 0).mean())
    b.close()


def test_batch_autotune_picks_a_candidate(renderer):
    from ffb200 import Batch
    items = synthetic.batch_flames(n=6, seed=9, spp=(20, 40), sizes=(64, 128))
    b = Batch(renderer, items, tune=True)
    info = b.info()
    assert info["threads"] in (128, 256, 512) and info["iterations_per_walker"] in (256, 1024, 4096)
    b.run()
    img, _ = b.output(0)
    assert (img[..., :3].max(axis=2) > 0).sum() > 0
    b.close()
