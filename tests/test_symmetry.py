"""Post-symmetry (scene/transforms.rs:2093-2190; utilities.wgsl:470-568;
main_template.wgsl:747-755, 858-870): each kept sample is plotted once per
copy -- `order` rotations about the centre in point mode, the sample and its
reflection (after a pan of half the separation and a pre-rotation) in the
axis modes.  The sample density still counts iterations, not copies
(compute_kernel.rs:1796-1840).

A linear flame walks identical orbits on the GPU and in the oracle, and the
copies' cos/sin come from the same f32 host computation on both sides, so
the count planes agree bit for bit."""

import copy
import json

import numpy as np
import pytest

from ffb200 import synthetic

MODES = [
    {"ty": "point", "order": 3, "center_x": 0.0, "center_y": 0.0, "distance": 1.25, "rotation_deg": 6.0},
    {"ty": "point", "order": 6, "center_x": 0.25, "center_y": -0.125, "distance": 1.25, "rotation_deg": 6.0},
    {"ty": "xaxis", "order": 3, "center_x": 0.0, "center_y": 0.1, "distance": 0.5, "rotation_deg": 15.0},
    {"ty": "yaxis", "order": 3, "center_x": -0.2, "center_y": 0.0, "distance": 0.0, "rotation_deg": -30.0},
]


def with_sym(cfg, sym):
    c = copy.deepcopy(cfg)
    c["flame"]["post_symmetry"] = sym
    return c


def test_parse_errors(native):
    r = native
    base = synthetic.sierpinski()
    bad = with_sym(base, {"ty": "diagonal", "order": 3, "center_x": 0, "center_y": 0, "distance": 1, "rotation_deg": 0})
    with pytest.raises(r.EngineError, match="unknown variant"):
        r.specialize(json.dumps(bad))
    missing = with_sym(base, {"ty": "point", "center_x": 0, "center_y": 0, "distance": 1, "rotation_deg": 0})
    with pytest.raises(r.EngineError, match="missing field `order`"):
        r.specialize(json.dumps(missing))


@pytest.mark.parametrize("sym", MODES, ids=lambda s: f"{s['ty']}{s['order']}")
def test_symmetry_specialises(native, sym):
    n, src = native.specialize(json.dumps(with_sym(synthetic.sierpinski(), sym)))
    kind = {"point": 3, "xaxis": 1, "yaxis": 2}[sym["ty"]]
    assert n > 0 and f"#define FFB_SYM_KIND {kind}" in src


@pytest.mark.gpu
@pytest.mark.parametrize("sym", MODES, ids=lambda s: f"{s['ty']}{s['order']}")
@pytest.mark.parametrize("schedule", ["plain", "sorted"])
def test_symmetric_histogram_bit_exact(renderer, oracle, sym, schedule):
    cfg = with_sym(synthetic.sierpinski(), sym)
    W, H = 96, 80
    walkers, per = 2048, 300
    cnt, rgb, out = renderer.histogram(cfg, W, H, iterations=walkers * per, walkers=walkers, schedule=schedule)
    fl = oracle.Flame(cfg, W, H)
    plotted, inframe, rc, rr = fl.render(walkers, per + 20, threads=8)
    assert out.total_iterations == plotted == walkers * per          # iterations, not copies
    assert int(cnt.sum()) == out.inframe_samples == inframe
    copies = sym["order"] if sym["ty"] == "point" else 2
    assert inframe > plotted * (copies - 1) * 0.5                   # the copies landed
    assert np.array_equal(cnt, rc)
    tol = cnt[..., None].astype(np.float64) * 2.0 ** -24 * np.maximum(rr, 1.0) + 1e-6
    assert np.all(np.abs(rgb - rr) <= tol)


@pytest.mark.gpu
def test_point_symmetry_is_rotation_invariant(renderer):
    """Order 4 about the origin on a square frame: the count plane is
    invariant under a quarter turn up to the pixel grid's rounding."""
    cfg = with_sym(synthetic.plain_flame(2), {"ty": "point", "order": 4, "center_x": 0.0, "center_y": 0.0,
                                             "distance": 1.25, "rotation_deg": 6.0})
    W = 128
    cnt, _, _ = renderer.histogram(cfg, W, W, iterations=4096 * 500, walkers=4096)
    rot = np.rot90(cnt)
    b = lambda c: c.reshape(16, 8, 16, 8).sum(axis=(1, 3)).astype(np.float64)
    a, r = b(cnt), b(rot)
    assert np.abs(a - r).sum() <= 0.02 * a.sum()
