"""Subflames and stateful variations (shaders/core/subflame.wgsl:1-412;
src/variations/defs/subflame.rs; klein_group_misc.rs; the walker state of
transforms.rs:226-300 and main_template.wgsl:117-170).

`subflame_wf` steps an inner flame's chaos game one visible iteration a
call and returns its placed output q (its weight divided out);
`pre_subflame_wf` replaces the point with q.  The walk, its colour and the
last q are walker state, as is klein_group's previous generator; state
starts at zero, persists across launches, and klein_group's state-init
draw is taken at every dispatch start of the reference's stream.

CPU: parsing and structure, and the oracle's subflame on chains with known
answers (a constant subflame, the reference's own finals example -- a walk
p -> 0.5 p + (1, 0) with a final + (10, 0) settles at q = (12, 0) --, a
hidden transform, the colour register, an empty subflame).
GPU: bit-identical count planes against the oracle for subflames of
exactly rounded arithmetic (linear, spherical, klein_group; finals, hidden
and translucent transforms, placement), both RNG modes, both schedules,
across launches, deferred plotting; transcendental inner variations
(blob, julian) within Monte-Carlo noise of the oracle.
"""

import ctypes
import json
import math

import numpy as np
import pytest

from ffb200 import EngineError
from ffb200 import _native

from test_gpu_parity import log_density_l1


def xf(a=1.0, b=0.0, c=0.0, d=1.0, e=0.0, f=0.0, w=1.0, col=0.5, v=None, **kw):
    t = {"a": a, "b": b, "c": c, "d": d, "e": e, "f": f, "weight": w, "color": col,
         "variations": v if v is not None else {"linear": 1.0}}
    t.update(kw)
    return t


def parent(sub_id=0.0, name="subflame_wf", w=1.0, **params):
    """A parent transform (identity affine) whose only variation steps subflame `sub_id`."""
    p = {f"{name}.subflame_id": sub_id}
    p.update({f"{name}.{k}": v for k, v in params.items()})
    return xf(v={name: w}, variation_params=p)


def flame(transforms, subflames, **extra):
    cfg = {"flame": {"transforms": transforms, "subflames": subflames}, "deterministic_rng": True}
    cfg.update(extra)
    return cfg


def sierpinski():
    return {"transforms": [xf(a=0.5, d=0.5, e=e, f=f, col=c)
                           for e, f, c in ((0.0, 0.5, 0.0), (-0.5, -0.5, 0.5), (0.5, -0.5, 1.0))]}


def plastic():
    """A thin subflame transform beside a heavy spherical one (the shape of
    the reference's plastic-sierpinski visual config), the subflame's colour
    taken over (color_mode 0, direct colour 1)."""
    t0 = parent(color_mode=0.0)
    t0["weight"] = 0.05
    t0["direct_color"] = 1.0
    t0["variations"] = {"flatten": 1.0, "subflame_wf": 1.0, "blur": 0.0}
    t1 = xf(a=0.6, b=0.2, c=-0.2, d=0.6, e=0.1, f=0.0, w=5.0, col=0.9,
            v={"flatten": 1.0, "linear": 0.075, "spherical": 1.2})
    return flame([t0, t1], [sierpinski()])


def klein():
    """Grandma's recipe at trace 2, 2 (an Apollonian gasket) as a subflame."""
    k = xf(v={"klein_group": 1.0}, variation_params={"klein_group.a_re": 2.0, "klein_group.a_im": 0.0,
                                                      "klein_group.b_re": 2.0, "klein_group.b_im": 0.0,
                                                      "klein_group.recipe": 0.0, "klein_group.avoid_reversal": 1.0})
    return flame([parent(scale=0.5)], [{"transforms": [k]}], zoom=0.5)


def placed():
    """Finals, a hidden and a translucent transform, a post-affine, and the
    placement by scale, angle and offsets; two parent transforms on two
    subflames, one of them the pre-phase variation."""
    s0 = {"transforms": [xf(a=0.5, d=0.5, e=0.5, f=0.0, col=0.1),
                         xf(a=0.4, b=0.1, c=-0.1, d=0.4, e=-0.3, f=0.4, col=0.8, opacity=0.0),
                         xf(a=0.3, d=0.6, e=0.1, f=-0.5, col=0.6, opacity=0.5, post_affine_enabled=True,
                            post_a=0.9, post_b=0.2, post_c=-0.2, post_d=0.9, post_e=0.05, post_f=0.0)],
          "final_transforms": [xf(a=0.8, b=0.1, c=-0.1, d=0.8, e=0.1, f=0.2, col=0.3, color_speed=0.5)]}
    s1 = sierpinski()
    t0 = parent(scale=1.5, angle=30.0, offset_x=0.2, offset_y=-0.1)
    t1 = xf(a=0.5, d=0.5, e=0.2, f=0.1, w=0.7, col=0.4, v={"pre_subflame_wf": 1.0, "linear": 1.0},
            variation_params={"pre_subflame_wf.subflame_id": 1.0, "pre_subflame_wf.scale": 0.8})
    return flame([t0, t1], [s0, s1], zoom=0.8)


def one_pixel(oracle, cfg, w=64, h=48, rng="philox"):
    fl = oracle.Flame(cfg, w, h)
    plotted, inframe, cnt, rgb = fl.render(500, 150, rng=rng, threads=4)
    lit = np.argwhere(cnt > 0)
    return fl, inframe, cnt, rgb, lit


# --------------------------------------------------------------------- CPU --

def test_subflames_specialize_with_state_and_colour():
    n, src = _native.specialize(json.dumps(plastic()))
    assert n > 0
    assert "ffb_sub_0(" in src and "#define FFB_DC 1" in src and "#define FFB_NSTATE 6" in src
    n, src = _native.specialize(json.dumps(klein()))
    assert "#define FFB_NSTATE 7" in src and "#define FFB_NINIT 1" in src   # subflame 6 + klein_group 1
    n, src = _native.specialize(json.dumps(placed()))
    assert "ffb_sub_1(" in src and "#define FFB_NSTATE 12" in src


def test_subflames_are_refused_where_not_built(native):
    """The differentiable render has no Jacobian for a subflame step; more
    than 8 subflames exceed the reference's MAX_SUBFLAMES."""
    c = json.dumps(plastic()).encode()
    n = ctypes.c_size_t()
    buf = ctypes.create_string_buffer(1 << 21)
    L = native.lib()
    assert L.ffb_diff_specialize(c, ctypes.c_size_t(len(c)), 16, 64, ctypes.byref(n), buf, ctypes.c_size_t(len(buf))) != 0
    assert "Jacobian" in L.ffb_last_error().decode()
    too_many = flame([parent()], [sierpinski()] * 9)
    with pytest.raises(EngineError, match="MAX_SUBFLAMES"):
        _native.specialize(json.dumps(too_many))


@pytest.mark.parametrize("rng", ["philox", "pcg"])
def test_constant_subflame_lights_its_placed_point(oracle, rng):
    """An inner transform that maps everything to (0.3, -0.2), placed by
    scale 2, angle 90 and offset (0.1, 0): every sample at q."""
    sub = {"transforms": [xf(a=0.0, b=0.0, c=0.0, d=0.0, e=0.3, f=-0.2)]}
    cfg = flame([parent(scale=2.0, angle=90.0, offset_x=0.1)], [sub])
    fl, inframe, cnt, _, lit = one_pixel(oracle, cfg, rng=rng)
    ang = np.float32(np.float32(90.0) * np.float32(0.017453292519943295))
    cs, sn = np.float32(math.cos(ang)), np.float32(math.sin(ang))
    x, y = np.float32(0.6), np.float32(-0.4)
    qx, qy = float(x * cs - y * sn + np.float32(0.1)), float(x * sn + y * cs)
    assert len(lit) == 1 and inframe == 500 * 130
    assert tuple(lit[0][::-1]) == fl.world_to_pixel(qx, qy)


def test_finals_map_the_walk_to_the_output(oracle):
    """subflame.wgsl:373-381: p -> 0.5 p + (1, 0) settles at (2, 0), and the
    final + (10, 0) gives q = (12, 0) without feeding the walk."""
    sub = {"transforms": [xf(a=0.5, d=0.5, e=1.0)], "final_transforms": [xf(e=10.0)]}
    cfg = flame([parent(scale=0.1)], [sub])
    fl, _, cnt, _, lit = one_pixel(oracle, cfg)
    assert len(lit) == 1
    assert tuple(lit[0][::-1]) == fl.world_to_pixel(float(np.float32(0.1) * np.float32(12.0)), 0.0)


def test_hidden_transform_moves_the_walk_but_never_outputs(oracle):
    sub = {"transforms": [xf(a=0.0, b=0.0, c=0.0, d=0.0, e=0.5, f=0.5, w=1.0),
                          xf(a=0.0, b=0.0, c=0.0, d=0.0, e=-0.5, f=-0.5, w=3.0, opacity=0.0)]}
    cfg = flame([parent()], [sub])
    fl, _, cnt, _, lit = one_pixel(oracle, cfg)
    assert len(lit) == 1 and tuple(lit[0][::-1]) == fl.world_to_pixel(0.5, 0.5)


def test_colour_mode_takes_the_subflames_colour(oracle):
    """color_mode 0 and direct colour 1: the parent's colour index is the
    subflame's, which settles at its transform's colour (speed 0)."""
    sub = {"transforms": [xf(a=0.0, b=0.0, c=0.0, d=0.0, e=0.2, f=0.1, col=0.75)]}
    t = parent(color_mode=0.0)
    t["direct_color"] = 1.0
    t["color"] = 0.1
    cfg = flame([t], [sub])
    fl, _, cnt, rgb, lit = one_pixel(oracle, cfg)
    px = tuple(lit[0])
    mean = rgb[px] / cnt[px]
    pal = fl.palette.reshape(-1, 3)
    np.testing.assert_allclose(mean, np.clip(pal[int(math.floor(0.75 * len(pal)))], 0, 1), rtol=1e-6)
    # color_mode -1 (the default): the parent's own colour flow (0.5 ci + 0.05 -> 0.1).
    t2 = parent()
    t2["color"] = 0.1
    fl, _, cnt, rgb, lit = one_pixel(oracle, flame([t2], [sub]))
    mean = rgb[tuple(lit[0])] / cnt[tuple(lit[0])]
    np.testing.assert_allclose(mean, np.clip(pal[int(math.floor(0.1 * len(pal)))], 0, 1), rtol=1e-6)


def test_an_empty_or_missing_subflame_outputs_the_origin(oracle):
    for cfg in (flame([parent()], [{"transforms": []}]), flame([parent(sub_id=3.0)], [sierpinski()])):
        fl, _, cnt, _, lit = one_pixel(oracle, cfg)
        assert len(lit) == 1 and tuple(lit[0][::-1]) == fl.world_to_pixel(0.0, 0.0)


# --------------------------------------------------------------------- GPU --

def gpu_vs_oracle(renderer, oracle, cfg, W, H, walkers, per, **job):
    rng = job.get("rng", "philox")
    ipt = job.get("iterations_per_thread", 1024)
    cnt, _, out = renderer.histogram(cfg, W, H, iterations=walkers * per, walkers=walkers, **job)
    fl = oracle.Flame(cfg, W, H)
    plotted, inframe, rc, _ = fl.render(walkers, per + 20, rng=rng, ipt=ipt, threads=8)
    assert out.total_iterations == plotted
    assert int(cnt.sum()) == out.inframe_samples == inframe > 0
    return cnt, rc


@pytest.mark.gpu
@pytest.mark.parametrize("rng_mode", ["philox", "pcg"])
@pytest.mark.parametrize("schedule", ["plain", "sorted"])
@pytest.mark.parametrize("which", ["plastic", "klein", "placed"])
def test_histogram_bit_exact_with_subflames(renderer, oracle, rng_mode, schedule, which):
    cfg = {"plastic": plastic, "klein": klein, "placed": placed}[which]()
    cnt, rc = gpu_vs_oracle(renderer, oracle, cfg, 96, 64, 2048, 400, rng=rng_mode, schedule=schedule,
                            iterations_per_thread=256, plot="inline")
    assert np.array_equal(cnt, rc)


@pytest.mark.gpu
@pytest.mark.parametrize("rng_mode", ["philox", "pcg"])
def test_subflame_state_survives_launches(renderer, oracle, rng_mode):
    """More iterations than one launch holds: the walk, its colour, q and
    klein_group's generator travel in the stored state."""
    cfg = klein()
    cnt, rc = gpu_vs_oracle(renderer, oracle, cfg, 64, 64, 256, 70_000, rng=rng_mode, iterations_per_thread=1024)
    assert np.array_equal(cnt, rc)


@pytest.mark.gpu
@pytest.mark.parametrize("rng_mode", ["philox", "pcg"])
def test_klein_group_in_the_parent(renderer, oracle, rng_mode):
    """klein_group as an ordinary variation: its state-init draw at every
    dispatch of the reference's stream (ipt 256 over 600 iterations)."""
    k = xf(v={"klein_group": 1.0, "linear": 0.2}, variation_params={"klein_group.recipe": 2.0,
                                                                   "klein_group.a_re": 1.9, "klein_group.b_re": 2.1})
    cfg = flame([k, xf(a=0.5, d=0.5, e=0.3, w=0.4)], [], zoom=0.6)
    cnt, rc = gpu_vs_oracle(renderer, oracle, cfg, 96, 64, 2048, 600, rng=rng_mode, iterations_per_thread=256)
    assert np.array_equal(cnt, rc)


@pytest.mark.gpu
def test_deferred_plot_with_subflames_is_the_same(renderer):
    cfg = placed()
    job = dict(iterations=20_000_000, walkers=16384, supersample=2)
    a, _, oa = renderer.histogram(cfg, 160, 120, plot="inline", **job)
    b, _, ob = renderer.histogram(cfg, 160, 120, plot="deferred", **job)
    assert oa.inframe_samples == ob.inframe_samples and np.array_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("inner", ["blob", "julian"])
def test_transcendental_subflame_within_monte_carlo_noise(renderer, oracle, inner):
    """The shape of the reference's subflame-blob / subflame-julian visual
    configs: a parametric variation beside two linear transforms."""
    v = {"blob": ({"blob": 1.0}, {"blob.high": 1.8, "blob.low": 0.3, "blob.waves": 8.0}, 0.6),
         "julian": ({"julian": 0.5}, {"julian.power": 5.0, "julian.dist": 2.5}, 0.5)}[inner]
    sub = {"transforms": [xf(a=0.8, d=0.8, w=v[2], col=0.0, v=v[0], variation_params=v[1]),
                          xf(a=0.5, d=0.5, e=0.5, col=0.5), xf(a=0.5, d=0.5, e=-0.5, col=1.0)]}
    cfg = flame([parent()], [sub], zoom=0.4)
    W = H = 128
    walkers, per = 8192, 400
    cnt, _, _ = renderer.histogram(cfg, W, H, iterations=walkers * per, walkers=walkers, seed=1001)
    fl = oracle.Flame(cfg, W, H)
    _, _, o1, _ = fl.render(walkers, per + 20, seed=1001, threads=8)
    _, _, o2, _ = fl.render(walkers, per + 20, seed=2002, threads=8)
    assert o1.sum() > 1000
    l1_go, p99_go = log_density_l1(cnt, o1)
    l1_oo, p99_oo = log_density_l1(o2, o1)
    assert l1_go <= 1.25 * l1_oo + 0.01, (l1_go, l1_oo)
    assert p99_go <= 1.25 * p99_oo + 0.05, (p99_go, p99_oo)


@pytest.mark.gpu
def test_subflames_are_refused_in_batches(renderer):
    from ffb200 import Batch
    with pytest.raises(EngineError, match="stateful"):
        Batch(renderer, [(plastic(), 32, 32, 10000)])
