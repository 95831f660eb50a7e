"""Bad-value respawn (shaders/core/main_template.wgsl:449-479): when the
point after the transform leaves |x|, |y| <= 1e32 (NaN fails the test
too), the walker restarts at a fresh U[-1,1]^2 draw with its fuse back at
the burn-in, skips the colour update and plots nothing that iteration.

Each flame below is the linear Sierpinski flame plus one transform that
blows the orbit up: an offset of 1e33 (every pick respawns), a scale of
1e17 (two picks in a row respawn), or coefficients of +-3e38 (the products
overflow to infinities and their sum to NaN).  Linear flames carry no
transcendental arithmetic, so the GPU walks the oracle's orbits exactly:
the count planes must be identical pixel for pixel in both RNG modes, and
in the deferred plot path, and the plotted samples the oracle counts must
fall short of walkers x iterations by the burn-ins the respawns restarted.
"""

import numpy as np
import pytest

from ffb200 import synthetic

BLOWUPS = {
    "offset_1e33": dict(a=1.0, b=0.0, c=0.0, d=1.0, e=1e33, f=0.0),
    "scale_1e17": dict(a=1e17, b=0.0, c=0.0, d=1e17, e=0.0, f=0.0),
    "nan": dict(a=3e38, b=-3e38, c=3e38, d=-3e38, e=0.0, f=0.0),
}


def respawn_flame(kind):
    cfg = synthetic.sierpinski()
    t = dict(BLOWUPS[kind], weight=0.25, color=0.9, color_speed=0.3, variations={"linear": 1.0})
    cfg["flame"]["transforms"].append(t)
    return cfg


@pytest.mark.parametrize("kind", sorted(BLOWUPS))
def test_oracle_respawns(oracle, kind):
    """The oracle restarts orbits: plotted samples fall short of
    walkers x iterations, and every plotted point stays finite and in frame
    often enough to light the Sierpinski triangle (a 1e17 scale keeps a
    walker out of frame for the ~57 halvings that bring it back)."""
    cfg = respawn_flame(kind)
    fl = oracle.Flame(cfg, 64, 64)
    walkers, per = 256, 400
    plotted, inframe, cnt, _ = fl.render(walkers, per + 20, threads=4)
    assert plotted < walkers * per
    assert inframe == int(cnt.sum()) > 0.05 * plotted


@pytest.mark.gpu
@pytest.mark.parametrize("kind", sorted(BLOWUPS))
@pytest.mark.parametrize("path", ["pcg", "philox", "philox-deferred"])
def test_respawn_matches_oracle_bit_for_bit(renderer, oracle, kind, path):
    cfg = respawn_flame(kind)
    W, H = 96, 64
    rng = path.split("-")[0]
    walkers = 16384 if path.endswith("deferred") else 2048
    per = 300
    job = dict(iterations=walkers * per, walkers=walkers, rng=rng, iterations_per_thread=256)
    if path.endswith("deferred"):
        job["plot"] = "deferred"
    cnt, rgb, out = renderer.histogram(cfg, W, H, **job)
    fl = oracle.Flame(cfg, W, H)
    plotted, inframe, rc, rr = fl.render(walkers, per + 20, rng=rng, ipt=256, threads=8)
    # The host counts plotted samples as the reference does (OrbitFuses:
    # iterations past the first burn-in); the respawns' second burn-ins are
    # samples the oracle's walkers did not plot.
    assert out.total_iterations == walkers * per
    assert plotted < walkers * per
    assert out.inframe_samples == inframe == int(cnt.sum())
    assert np.array_equal(cnt, rc)
    tol = cnt[..., None].astype(np.float64) * 2.0 ** -24 * np.maximum(rr, 1.0) + 1e-6
    assert np.all(np.abs(rgb - rr) <= tol)
