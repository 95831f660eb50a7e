"""Seeded synthetic flames with the shapes of the benchmark configurations.

No public dataset is involved: each flame is drawn from a seeded generator
(numpy's PCG64), and the seed is part of the returned config's name.
Shapes follow the benchmark's configuration list:

* `plain_flame`  -- 3 transforms, affines ~U[-1,1], {linear, sinusoidal,
  spherical} at Dirichlet(1) weights, transform weights ~U[0.2,1], colours
  ~U[0,1], a 256-entry random RGB palette; gamma 4, vibrancy 1, brightness 4.
* `full_flame`   -- 8 transforms + 1 final, each with 3-5 of the twelve
  variations at weights ~U[0,1], affines ~U[-1.5,1.5]; density estimation
  radius 9 -> 0.
* `stress_flame` -- 16 transforms: 10 as the full flame's plus 6 rotations
  by k*60 degrees (6-fold rotational symmetry as ordinary transforms);
  density estimation radius 12 -> 0.
* `diff_flame`   -- 4 transforms for the differentiable render: the plain
  flame's distributions with each affine's linear part scaled by 0.6, so
  every transform contracts on average and a sample's sensitivity to
  iterations more than 16 back is below 1e-4 of its gradient;
* `batch_flames` -- 256 flames for the batched renderer: transform counts
  ~U{2..12}, variations as the plain flame, sizes ~{128,256,512,1024}^2,
  budgets ~U[50,2000] samples a pixel, a seed each.
"""

import numpy as np

TWELVE = ["linear", "swirl", "horseshoe", "polar", "julia", "bubble", "spherical", "sinusoidal",
          "disc", "ex", "cylinder", "curl"]


def random_palette(rng, n=256):
    cols = rng.integers(0, 256, size=(n, 3))
    return {"name": "synthetic", "indexed_colors": ",".join("%02X%02X%02X" % tuple(c) for c in cols)}


def _affine(rng, lo, hi):
    a, b, c, d, e, f = (float(v) for v in rng.uniform(lo, hi, 6))
    return {"a": a, "b": b, "c": c, "d": d, "e": e, "f": f}


def plain_flame(seed=1, n_xforms=3, variations=("linear", "sinusoidal", "spherical")):
    rng = np.random.default_rng(seed)
    xfs = []
    for _ in range(n_xforms):
        w = -np.log(rng.uniform(1e-12, 1.0, len(variations)))
        w = w / w.sum()                                            # Dirichlet(1)
        t = _affine(rng, -1.0, 1.0)
        t.update({"weight": float(rng.uniform(0.2, 1.0)), "color": float(rng.uniform(0, 1)),
                  "variations": {v: float(x) for v, x in zip(variations, w)}})
        xfs.append(t)
    return {
        "name": f"plain-{seed}", "flame": {"transforms": xfs}, "render_mode": "TwoD",
        "palette": random_palette(rng), "gamma": 4.0, "vibrancy": 1.0, "brightness": 4.0,
        "zoom": 1.0, "pan_x": 0.0, "pan_y": 0.0, "deterministic_rng": True,
    }


def full_flame(seed=7, n_xforms=8, de_radius=9.0):
    rng = np.random.default_rng(seed)

    def xform():
        k = int(rng.integers(3, 6))
        names = list(rng.choice(TWELVE, size=k, replace=False))
        t = _affine(rng, -1.5, 1.5)
        t.update({"weight": float(rng.uniform(0.2, 1.0)), "color": float(rng.uniform(0, 1)),
                  "color_speed": 0.0, "variations": {n: float(rng.uniform(0, 1)) for n in names}})
        return t

    xfs = [xform() for _ in range(n_xforms)]
    fin = xform()
    cfg = {
        "name": f"full-{seed}", "flame": {"transforms": xfs, "final_transform": fin}, "render_mode": "TwoD",
        "palette": random_palette(rng), "gamma": 4.0, "vibrancy": 1.0, "brightness": 4.0,
        "zoom": 1.0, "pan_x": 0.0, "pan_y": 0.0, "deterministic_rng": True,
    }
    if de_radius:
        cfg["density_estimation"] = {"radius": de_radius, "minimum": 0.0, "curve": 0.4}
    return cfg


def sierpinski():
    """A linear-only flame: no transcendental arithmetic, so the GPU and the
    oracle walk bit-identical orbits."""
    t = []
    for e, f in ((-0.5, -0.5), (0.5, -0.5), (0.0, 0.5)):
        t.append({"a": 0.5, "b": 0.0, "c": 0.0, "d": 0.5, "e": e, "f": f, "weight": 1.0, "color": (e + 1) / 2,
                  "color_speed": 0.3, "variations": {"linear": 1.0}})
    return {"name": "sierpinski", "flame": {"transforms": t}, "render_mode": "TwoD", "deterministic_rng": True,
            "zoom": 1.0}


def batch_flames(n=256, seed=3, spp=(50, 2000), sizes=(128, 256, 512, 1024)):
    """(config, width, height, samples, seed) tuples."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        k = int(rng.integers(2, 13))
        cfg = plain_flame(int(rng.integers(1, 2 ** 31)), n_xforms=k)
        side = int(rng.choice(sizes))
        samples = int(rng.uniform(*spp) * side * side)
        out.append((cfg, side, side, samples, 1000 + i))
    return out


def stress_flame(seed=21, de_radius=12.0):
    """The 4K stress flame: 10 random transforms + 6 rotation transforms."""
    import math
    base = full_flame(seed, n_xforms=10, de_radius=de_radius)
    rng = np.random.default_rng(seed + 1)
    for k in range(6):
        th = k * math.pi / 3.0
        base["flame"]["transforms"].append({
            "a": math.cos(th), "b": -math.sin(th), "c": math.sin(th), "d": math.cos(th), "e": 0.0, "f": 0.0,
            "weight": 0.5, "color": float(rng.uniform(0, 1)), "color_speed": 0.5, "variations": {"linear": 1.0}})
    base["name"] = f"stress-{seed}"
    return base


def diff_flame(seed=4, n_xforms=4):
    """The differentiable render's flame (4 transforms, contractive)."""
    cfg = plain_flame(seed, n_xforms=n_xforms)
    for t in cfg["flame"]["transforms"]:
        for k in "abcd":
            t[k] = float(np.float32(t[k] * 0.6))
    cfg["name"] = f"diff-{seed}"
    return cfg
