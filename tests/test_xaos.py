"""Xaos (utilities.wgsl:106-137; main_template.wgsl:63-71, 163-211;
scene/xaos.rs): the next transform is picked with weight_i x
xaos[prev][i], a starting walker's previous transform is the unconditioned
pick at a Kronecker point of its index (walker * 2654435769 + seed), and a
chain whose walk (not the first pick) splits orbits between closed groups
gets the reference's orbit refresh: every dispatch restarts the walkers w
with (w + the dispatch's seed) % 4 == 0 (compute_kernel.rs:45-101).

CPU: parsing, the refresh decision, the oracle's walk on chains with known
answers (with refresh, each closed group's share of the samples tends to
its weight's share).
GPU: bit-identical count planes against the oracle for a linear flame with
xaos (both RNG modes, both schedules), with refresh across launches, and
the plotted-sample count the refresh leaves.
"""

import json

import numpy as np
import pytest

from ffb200 import EngineError, synthetic
from ffb200 import _native


def two_points(xaos, w=(1.0, 3.0)):
    """Two constant transforms (a = b = c = d = 0): every sample lands on
    one of two pixels, whichever transform the walker took."""
    t = [{"a": 0, "b": 0, "c": 0, "d": 0, "e": -1.0 + 0.01, "f": 0.01, "weight": w[0], "color": 0.0,
          "variations": {"linear": 1.0}},
         {"a": 0, "b": 0, "c": 0, "d": 0, "e": 1.0 + 0.01, "f": 0.01, "weight": w[1], "color": 1.0,
          "variations": {"linear": 1.0}}]
    return {"flame": {"transforms": t, "xaos": xaos}, "deterministic_rng": True}


def sierpinski_xaos():
    cfg = synthetic.sierpinski()
    cfg["flame"]["xaos"] = [[0.2, 1.0, 1.0], [1.0, 0.0, 2.0], [1.0, 1.0, 0.5]]
    return cfg


# --------------------------------------------------------------------- CPU --

def test_xaos_specializes_and_all_ones_is_plain():
    _, src = _native.specialize(json.dumps(sierpinski_xaos()))
    assert "#define FFB_XAOS 1" in src
    cfg = synthetic.sierpinski()
    cfg["flame"]["xaos"] = [[1, 1, 1], [1, 1, 1], [1, 1, 1]]
    _, src = _native.specialize(json.dumps(cfg))
    assert "#define FFB_XAOS" not in src


def test_a_walk_that_splits_orbits_is_refreshed(oracle):
    # Transform 0 leads to 1 and 2, each of which only returns to itself:
    # where an orbit ends is decided by the walk, not the first pick.
    cfg = synthetic.sierpinski()
    cfg["flame"]["xaos"] = [[0, 1, 1], [0, 1, 0], [0, 0, 1]]
    _, src = _native.specialize(json.dumps(cfg))
    assert "#define FFB_REFRESH 4" in src
    assert oracle.walk_splits_orbits([1.0, 1.0, 1.0], cfg["flame"]["xaos"])
    # Closed groups picked by the first transform alone need none (the stratified start).
    cfg["flame"]["xaos"] = [[1, 0, 0], [0, 1, 0], [0, 0, 1]]
    _, src = _native.specialize(json.dumps(cfg))
    assert "#define FFB_REFRESH" not in src
    assert not oracle.walk_splits_orbits([1.0, 1.0, 1.0], cfg["flame"]["xaos"])


def split_chain():
    """A start transform that leads to one of two absorbing constant
    transforms, weights 1 : 3."""
    cfg = two_points([[0, 1, 1], [0, 1, 0], [0, 0, 1]], w=(1.0, 3.0))
    cfg["flame"]["transforms"].insert(0, {"a": 0.5, "b": 0, "c": 0, "d": 0.5, "e": 0, "f": 0, "weight": 2.0,
                                          "color": 0.5, "variations": {"linear": 1.0}})
    return cfg


@pytest.mark.parametrize("rng", ["philox", "pcg"])
def test_refresh_shares_the_groups_by_weight(oracle, rng):
    """Without refresh an orbit stays in the group its walk first entered;
    with it a quarter restart each dispatch, and over many dispatches the
    two absorbing pixels split the samples as their weights (1 : 3) to
    within sampling noise."""
    cfg = split_chain()
    fl = oracle.Flame(cfg, 64, 32)
    walkers, ipt, per = 4000, 32, 32 * 60
    plotted, inframe, cnt, _ = fl.render(walkers, per + 20, rng=rng, ipt=ipt, threads=4)
    lit = sorted(int(v) for v in cnt[cnt > 0])
    assert len(lit) == 2
    share = lit[0] / (lit[0] + lit[1])
    assert abs(share - 0.25) < 0.02, share
    assert plotted < walkers * per                       # restarted walkers burn in again


def test_identity_xaos_keeps_each_walker_in_its_first_transform(oracle):
    """Each walker stays on its first transform's fixed point; the first
    picks are stratified, so the two pixels' counts split 1:3 to within a
    walker (the reference's stated purpose, main_template.wgsl:163-179)."""
    cfg = two_points([[1, 0], [0, 1]])
    fl = oracle.Flame(cfg, 64, 32)
    walkers = 4000
    plotted, inframe, cnt, _ = fl.render(walkers, 120, threads=4)
    lit = np.argwhere(cnt > 0)
    assert len(lit) == 2
    a, b = sorted(int(cnt[tuple(p)]) for p in lit)
    per = 120 - 20
    assert a + b == walkers * per
    assert abs(a / per - walkers / 4) <= 2 and abs(b / per - 3 * walkers / 4) <= 2


def test_alternating_xaos_alternates(oracle):
    """xaos [[0, 1], [1, 0]]: every step changes transform, so each walker
    splits its samples evenly between the two pixels."""
    cfg = two_points([[0, 1], [1, 0]])
    fl = oracle.Flame(cfg, 64, 32)
    walkers, per = 1000, 100
    plotted, inframe, cnt, _ = fl.render(walkers, per + 20, threads=4)
    lit = sorted(int(v) for v in cnt[cnt > 0])
    assert lit == [walkers * per // 2, walkers * per // 2]


def test_imported_chaos_renders_as_xaos():
    xml = ('<flames><flame name="X" size="64 48" center="0 0" scale="40">'
           '<xform weight="1" color="0" linear="1" coefs="0.5 0 0 0.5 -0.5 0" chaos="1 0.5" />'
           '<xform weight="1" color="1" linear="1" coefs="0.5 0 0 0.5 0.5 0" chaos="0 1" /></flame></flames>')
    cfg = _native.flame_import(xml)[0]
    assert cfg["flame"]["xaos"] == [[1, 0.5], [0, 1]]
    _, src = _native.specialize(json.dumps(cfg))
    assert "#define FFB_XAOS 1" in src


# --------------------------------------------------------------------- GPU --

@pytest.mark.gpu
@pytest.mark.parametrize("rng_mode", ["pcg", "philox"])
@pytest.mark.parametrize("schedule", ["plain", "sorted"])
def test_histogram_bit_exact_with_xaos(renderer, oracle, rng_mode, schedule):
    cfg = sierpinski_xaos()
    W, H, walkers, per = 96, 64, 2048, 600
    cnt, _, out = renderer.histogram(cfg, W, H, iterations=walkers * per, walkers=walkers, rng=rng_mode,
                                     iterations_per_thread=256, schedule=schedule)
    fl = oracle.Flame(cfg, W, H)
    plotted, inframe, rc, _ = fl.render(walkers, per + 20, rng=rng_mode, ipt=256, threads=8)
    assert out.total_iterations == plotted
    assert int(cnt.sum()) == inframe
    assert np.array_equal(cnt, rc)


@pytest.mark.gpu
@pytest.mark.parametrize("rng_mode", ["philox", "pcg"])
@pytest.mark.parametrize("schedule", ["plain", "sorted"])
def test_refresh_bit_exact(renderer, oracle, rng_mode, schedule):
    """Orbit refresh: the same restarts, orbits and plotted-sample count as
    the oracle, over launches of many dispatches."""
    cfg = split_chain()
    W, H, walkers, per, ipt = 64, 32, 2048, 70_000, 1024
    cnt, _, out = renderer.histogram(cfg, W, H, iterations=walkers * per, walkers=walkers, rng=rng_mode,
                                     iterations_per_thread=ipt, schedule=schedule)
    fl = oracle.Flame(cfg, W, H)
    plotted, inframe, rc, _ = fl.render(walkers, per + 20, rng=rng_mode, ipt=ipt, threads=8)
    assert out.total_iterations == plotted < walkers * per
    assert int(cnt.sum()) == out.inframe_samples == inframe
    assert np.array_equal(cnt, rc)


@pytest.mark.gpu
def test_xaos_state_survives_launches(renderer, oracle):
    """More iterations than one launch holds (65,536 a walker): the previous
    transform travels in the stored walker state."""
    cfg = sierpinski_xaos()
    W, H, walkers, per = 64, 64, 256, 70_000
    cnt, _, out = renderer.histogram(cfg, W, H, iterations=walkers * per, walkers=walkers, rng="philox")
    fl = oracle.Flame(cfg, W, H)
    _, inframe, rc, _ = fl.render(walkers, per + 20, threads=8)
    assert np.array_equal(cnt, rc)


@pytest.mark.gpu
def test_identity_xaos_on_the_gpu(renderer, oracle):
    cfg = two_points([[1, 0], [0, 1]])
    cnt, _, _ = renderer.histogram(cfg, 64, 32, iterations=4000 * 100, walkers=4000)
    fl = oracle.Flame(cfg, 64, 32)
    _, _, rc, _ = fl.render(4000, 120, threads=4)
    assert np.array_equal(cnt, rc)


@pytest.mark.gpu
def test_xaos_is_refused_in_batches(renderer):
    from ffb200 import Batch
    with pytest.raises(EngineError, match="xaos"):
        Batch(renderer, [(sierpinski_xaos(), 32, 32, 10000)])
