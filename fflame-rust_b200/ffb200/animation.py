"""Keyframe animation of flames, rendered as one batch.

The interpolation vocabulary is the reference's (src/animation/
interpolation.rs:7-125): an `Interpolation` curve in time (step, linear,
smooth, sinusoidal, exponential) and, for exponential, equal-ratio
interpolation in value (`geometric_lerp`).  Two keyframe flames of the same
structure (same transforms and variations) are blended field by field; the
frames then share one compiled module, so a whole animation renders as one
persistent launch and one tone-map launch (`ffb200.Batch`).
"""

import copy
import math

INTERPOLATIONS = ("step", "linear", "smooth", "sinusoidal", "exponential")

# Numeric fields blended between keyframes.
TRANSFORM_FIELDS = ("a", "b", "c", "d", "e", "f", "post_a", "post_b", "post_c", "post_d", "post_e", "post_f",
                    "weight", "color", "color_speed", "opacity")
VIEW_FIELDS = ("zoom", "pan_x", "pan_y", "rotation")


def apply(mode, t):
    """Interpolation::apply (interpolation.rs:104-118): the time curve."""
    t = min(max(t, 0.0), 1.0)
    if mode == "step":
        return 0.0 if t < 0.5 else 1.0
    if mode in ("linear", "exponential"):
        return t
    if mode == "smooth":
        return t * t * (3.0 - 2.0 * t)
    if mode == "sinusoidal":
        return (1.0 - math.cos(t * math.pi)) / 2.0
    raise ValueError(f"unknown interpolation `{mode}`")


def geometric_lerp(a, b, t):
    """interpolation.rs:120-131: equal-ratio between same-sign values, else linear."""
    if (a > 0.0 and b > 0.0) or (a < 0.0 and b < 0.0):
        return a * (b / a) ** t
    return a + (b - a) * t


def _blend(a, b, t, mode):
    if mode == "exponential":
        return geometric_lerp(a, b, t)
    return a + (b - a) * t


def _blend_transform(ta, tb, t, mode):
    if set(ta["variations"]) != set(tb["variations"]):
        raise ValueError("keyframes differ in a transform's variations")
    out = copy.deepcopy(ta)
    for k in TRANSFORM_FIELDS:
        if k in ta or k in tb:
            d = {"post_a": 1.0, "post_d": 1.0, "weight": 1.0, "opacity": 1.0}.get(k, 0.0)
            out[k] = _blend(ta.get(k, d), tb.get(k, d), t, mode)
    out["variations"] = {n: _blend(ta["variations"][n], tb["variations"][n], t, mode) for n in ta["variations"]}
    pa, pb = ta.get("variation_params", {}), tb.get("variation_params", {})
    if pa or pb:
        out["variation_params"] = {k: _blend(pa.get(k, pb.get(k)), pb.get(k, pa.get(k)), t, mode) for k in set(pa) | set(pb)}
    return out


def interpolate(a, b, t, mode="linear"):
    """The flame between keyframes `a` (t = 0) and `b` (t = 1)."""
    s = apply(mode, t)
    fa, fb = a["flame"], b["flame"]
    if len(fa["transforms"]) != len(fb["transforms"]):
        raise ValueError("keyframes differ in their transform count")
    out = copy.deepcopy(a)
    out["flame"]["transforms"] = [_blend_transform(x, y, s, mode) for x, y in zip(fa["transforms"], fb["transforms"])]
    for key in ("final_transform",):
        if fa.get(key) and fb.get(key):
            out["flame"][key] = _blend_transform(fa[key], fb[key], s, mode)
    if fa.get("final_transforms"):
        out["flame"]["final_transforms"] = [_blend_transform(x, y, s, mode)
                                            for x, y in zip(fa["final_transforms"], fb["final_transforms"])]
    for k in VIEW_FIELDS:
        if k in a or k in b:
            d = 1.0 if k == "zoom" else 0.0
            out[k] = _blend(a.get(k, d), b.get(k, d), s, "exponential" if (mode == "exponential" or k == "zoom") else mode)
    return out


def frames(a, b, n, mode="linear"):
    """n frames from `a` to `b` inclusive."""
    if n == 1:
        return [copy.deepcopy(a)]
    return [interpolate(a, b, i / (n - 1), mode) for i in range(n)]


def render(renderer, configs, width, height, samples, tune=False, **job):
    """Render frames as one batch: [(RGBA8 [h, w, 4], plotted)] in order."""
    from ._native import Batch
    items = [(c, width, height, samples, 0) for c in configs]
    b = Batch(renderer, items, tune=tune, **job)
    b.run()
    out = [b.output(i) for i in range(len(configs))]
    b.close()
    return out
