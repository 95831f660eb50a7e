"""Keyframe interpolation (src/animation/interpolation.rs) on the CPU, and
the batched animation render on the GPU."""

import math

import numpy as np
import pytest

from ffb200 import animation, synthetic


def test_interpolation_curves_match_the_reference_formulas():
    for t in (0.0, 0.25, 0.5, 0.75, 1.0):
        assert animation.apply("linear", t) == t
        assert animation.apply("step", t) == (0.0 if t < 0.5 else 1.0)
        assert animation.apply("smooth", t) == pytest.approx(t * t * (3 - 2 * t))
        assert animation.apply("sinusoidal", t) == pytest.approx((1 - math.cos(math.pi * t)) / 2)
    assert animation.geometric_lerp(1.0, 4.0, 0.5) == pytest.approx(2.0)
    assert animation.geometric_lerp(-1.0, 1.0, 0.5) == 0.0      # through zero: linear


def test_frames_blend_affines_and_keep_structure():
    a = synthetic.stress_flame(21, de_radius=0)
    b = synthetic.stress_flame(21, de_radius=0)
    for t in b["flame"]["transforms"]:
        t["a"] += 0.2
        t["e"] -= 0.1
    b["zoom"] = 2.0
    fr = animation.frames(a, b, 5)
    assert len(fr) == 5
    assert fr[0]["flame"]["transforms"][0]["a"] == pytest.approx(a["flame"]["transforms"][0]["a"])
    assert fr[-1]["flame"]["transforms"][0]["a"] == pytest.approx(b["flame"]["transforms"][0]["a"])
    assert fr[2]["flame"]["transforms"][3]["e"] == pytest.approx(a["flame"]["transforms"][3]["e"] - 0.05)
    assert fr[2]["zoom"] == pytest.approx(math.sqrt(2.0))   # zoom is a scale: equal ratios
    assert all(set(f["flame"]["transforms"][k]["variations"]) == set(a["flame"]["transforms"][k]["variations"])
               for f in fr for k in range(16))


def test_keyframes_of_different_structure_are_refused():
    a = synthetic.plain_flame(1)
    b = synthetic.plain_flame(1, n_xforms=4)
    with pytest.raises(ValueError):
        animation.interpolate(a, b, 0.5)


@pytest.mark.gpu
def test_animation_renders_as_one_batch(renderer):
    """Frames of one structure share a module: one launch, and each frame is
    the single render of the same walkers (2x supersampling, DE on)."""
    from ffb200 import Batch
    a = synthetic.stress_flame(21, de_radius=3.0)
    b = synthetic.stress_flame(21, de_radius=3.0)
    for t in b["flame"]["transforms"][:10]:
        t["a"] *= 0.9
    fr = animation.frames(a, b, 4)
    out = animation.render(renderer, fr, 96, 64, 400_000, supersample=2, threads=128, iterations_per_thread=256)
    assert len(out) == 4
    walkers, per = Batch.walkers_for(400_000, 128, 256)
    for cfg, (img, plotted) in zip(fr, out):
        assert plotted == walkers * per
        ref, o = renderer.render(cfg, 96, 64, iterations=walkers * per, walkers=walkers, supersample=2,
                                 seed=0, schedule="sorted")
        d = np.abs(img.astype(int) - ref.astype(int))
        assert d.max() <= 2 and (d > 0).mean() < 0.02
