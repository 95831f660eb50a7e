"""Linked transforms and per-transform final chains (the attachments of
transforms.rs:470-480, gpu/buffers.rs:600-680; main_template.wgsl:320-360
and 663-717), and the solo transform (gpu/buffers.rs:523-536: every other
normal transform keeps moving the walk but plots nothing).

After the chaos game picks normal transform k, its linked chain runs in the
same iteration -- affine, variations, post-affine each, every output the
next one's input and the last the walker's next point, colour writes
reaching the register -- and at plot time k's own final chain shapes the
plotted point.  Attachment indices past their pool are dropped and a chain
holds at most 32 (the reference logs and does the same).

CPU: parsing and cleaning of the lists, the structure of the generated code
(one compiled chain when every normal shares it, the table otherwise), the
oracle's chains on known answers (a linked chain that feeds the walk to a
fixed point, differing final chains).
GPU: bit-identical count planes against the oracle for exactly rounded
chains, both RNG modes, both schedules, inline and deferred plotting;
chains with random draws within Monte-Carlo noise.
"""

import json

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


def chained():
    """Three normals with their own linked and final chains, exactly
    rounded bodies (spherical, bubble, curl, bent, horseshoe), a
    post-affine on a linked transform, an out-of-range attachment."""
    normals = [xf(a=0.5, d=0.5, e=0.0, f=0.5, col=0.0, v={"linear": 0.8, "spherical": 0.2},
                  linked_attachments=[0], final_attachments=[0]),
               xf(a=0.5, b=0.1, c=-0.1, d=0.5, e=-0.5, f=-0.5, col=0.5, v={"bubble": 0.5, "linear": 0.5},
                  final_attachments=[1, 2, 7]),
               xf(a=0.5, d=0.5, e=0.5, f=-0.5, w=0.7, col=1.0, v={"linear": 1.0},
                  linked_attachments=[1, 0, 5])]
    linked = [xf(a=0.9, b=0.05, c=-0.05, d=0.9, e=0.02, f=0.0, v={"curl": 0.3, "linear": 0.7},
                 variation_params={"curl.c1": 0.4, "curl.c2": 0.1}),
              xf(a=1.0, d=1.0, e=0.1, v={"bent": 0.6, "linear": 0.4}, post_affine_enabled=True,
                 post_a=0.8, post_b=0.1, post_c=-0.1, post_d=0.8, post_e=0.0, post_f=0.05)]
    finals = [xf(a=0.9, d=0.9, e=0.1, v={"horseshoe": 0.3, "linear": 0.7}),
              xf(a=1.0, d=1.0, f=-0.1, v={"spherical": 0.5, "linear": 0.5}),
              xf(a=0.8, b=0.2, c=-0.2, d=0.8, v={"linear": 1.0})]
    return {"flame": {"transforms": normals, "linked_transforms": linked, "final_transforms": finals},
            "deterministic_rng": True, "zoom": 0.7}


def drawing():
    """Chains whose transforms take random draws (blur, julia, noise)."""
    cfg = chained()
    fl = cfg["flame"]
    fl["linked_transforms"][0]["variations"] = {"blur": 0.1, "linear": 0.9}
    fl["final_transforms"][1]["variations"] = {"julia": 0.4, "linear": 0.6}
    fl["final_transforms"][2]["variations"] = {"noise": 0.2, "linear": 0.8}
    return cfg


def one_pixel(oracle, cfg, w=64, h=48):
    fl = oracle.Flame(cfg, w, h)
    _, inframe, cnt, _ = fl.render(400, 150, threads=4)
    return fl, inframe, cnt


# --------------------------------------------------------------------- CPU --

def test_attachments_specialize():
    n, src = _native.specialize(json.dumps(chained()))
    assert n > 0
    assert "#define FFB_NLNK 2" in src and "#define FFB_LCAP 2" in src and "#define FFB_FCAP 2" in src
    assert "ffb_linked_one(" in src and "T_ATT + k * FFB_ATT_STRIDE + 1 + FFB_LCAP" in src
    # Every normal on the same final chain: the chain is compiled in, no table.
    cfg = chained()
    for t in cfg["flame"]["transforms"]:
        t["final_attachments"] = [2, 0]
        t.pop("linked_attachments", None)
    _, src = _native.specialize(json.dumps(cfg))
    assert "#define FFB_NLNK 0" in src and "#define FFB_FCAP 0" in src
    body = src[src.index("void ffb_finals("):]
    body = body[:body.index("\n}\n")]
    assert "ffb_final_one(sm, 1, x, y, rng, ctx, true);\n    ffb_final_one(sm, 0, x, y, rng, ctx, true);" in body


def test_a_repeated_drawing_transform_needs_the_pcg_stream():
    cfg = drawing()
    cfg["flame"]["transforms"][0]["linked_attachments"] = [0, 0]
    with pytest.raises(EngineError, match="pcg stream"):
        _native.specialize(json.dumps(cfg))
    assert _native.specialize(json.dumps(cfg), rng="pcg")[0] > 0
    cfg = chained()
    cfg["flame"]["transforms"][0]["linked_attachments"] = [0, 0]            # no draws: fine
    assert _native.specialize(json.dumps(cfg))[0] > 0


def test_linked_chain_feeds_the_walk(oracle):
    """p -> 0.5 p (normal), then + (1, 0.3) (linked): the walk's map is
    0.5 p + (1, 0.3), fixed point (2, 0.6), where every sample lands."""
    cfg = {"flame": {"transforms": [xf(a=0.5, d=0.5, linked_attachments=[0])],
                     "linked_transforms": [xf(e=1.0, f=0.3)]}, "deterministic_rng": True, "zoom": 0.45}
    fl, inframe, cnt = one_pixel(oracle, cfg)
    lit = np.argwhere(cnt > 0)
    assert len(lit) == 1 and tuple(lit[0][::-1]) == fl.world_to_pixel(2.0, 0.6)


@pytest.mark.parametrize("rng", ["philox", "pcg"])
def test_each_normal_plots_through_its_own_finals(oracle, rng):
    """Two constant normals; the first's final moves its point, the second
    has none; an attachment past the pool is dropped."""
    cfg = {"flame": {"transforms": [xf(a=0, b=0, c=0, d=0, e=0.5, f=0.5, final_attachments=[0, 9]),
                                    xf(a=0, b=0, c=0, d=0, e=-0.5, f=-0.5)],
                     "final_transforms": [xf(e=0.25)]}, "deterministic_rng": True}
    fl = oracle.Flame(cfg, 64, 48)
    _, inframe, cnt, _ = fl.render(400, 150, rng=rng, threads=4)
    lit = sorted(tuple(p[::-1]) for p in np.argwhere(cnt > 0))
    assert lit == sorted([fl.world_to_pixel(0.75, 0.5), fl.world_to_pixel(-0.5, -0.5)])
    a, b = (int(cnt[p[1], p[0]]) for p in lit)
    assert a + b == inframe and abs(a - b) < 0.05 * inframe


def test_solo_transform_plots_alone(oracle):
    cfg = {"flame": {"transforms": [xf(a=0, b=0, c=0, d=0, e=0.5, f=0.5), xf(a=0, b=0, c=0, d=0, e=-0.5, f=-0.5)],
                     "solo_transform": 1}, "deterministic_rng": True}
    assert _native.specialize(json.dumps(cfg))[0] > 0
    fl, inframe, cnt = one_pixel(oracle, cfg)
    lit = np.argwhere(cnt > 0)
    assert len(lit) == 1 and tuple(lit[0][::-1]) == fl.world_to_pixel(-0.5, -0.5)
    cfg["flame"]["solo_transform"] = -1
    with pytest.raises(EngineError, match="solo_transform"):
        _native.specialize(json.dumps(cfg))


# --------------------------------------------------------------------- GPU --

@pytest.mark.gpu
def test_solo_transform_bit_exact(renderer, oracle):
    cfg = chained()
    cfg["flame"]["solo_transform"] = 1
    cnt, rc = gpu_vs_oracle(renderer, oracle, cfg, 96, 64, 2048, 300)
    assert np.array_equal(cnt, rc)



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
def test_chains_bit_exact(renderer, oracle, rng_mode, schedule):
    cnt, rc = gpu_vs_oracle(renderer, oracle, chained(), 96, 64, 2048, 400, rng=rng_mode, schedule=schedule,
                            iterations_per_thread=256, plot="inline")
    assert np.array_equal(cnt, rc)


@pytest.mark.gpu
def test_chains_deferred_plot_bit_exact(renderer, oracle):
    """The deferred plot finds each sample's final chain by the transform
    stored in its record."""
    cnt, rc = gpu_vs_oracle(renderer, oracle, chained(), 96, 64, 16384, 300, schedule="sorted", plot="deferred")
    assert np.array_equal(cnt, rc)


@pytest.mark.gpu
@pytest.mark.parametrize("rng_mode", ["philox", "pcg"])
def test_drawing_chains_within_monte_carlo_noise(renderer, oracle, rng_mode):
    cfg = drawing()
    W = H = 128
    walkers, per = 8192, 400
    cnt, _, _ = renderer.histogram(cfg, W, H, iterations=walkers * per, walkers=walkers, seed=1001, rng=rng_mode,
                                   iterations_per_thread=256)
    fl = oracle.Flame(cfg, W, H)
    _, _, o1, _ = fl.render(walkers, per + 20, seed=1001, rng=rng_mode, ipt=256, threads=8)
    _, _, o2, _ = fl.render(walkers, per + 20, seed=2002, rng=rng_mode, ipt=256, threads=8)
    assert o1.sum() > 1000
    l1_go, p99_go = log_density_l1(cnt, o1)
    l1_oo, p99_oo = log_density_l1(o2, o1)
    assert l1_go <= 1.25 * l1_oo + 0.01, (l1_go, l1_oo)
    assert p99_go <= 1.25 * p99_oo + 0.05, (p99_go, p99_oo)


@pytest.mark.gpu
def test_drawing_chains_deferred_equals_inline(renderer):
    cfg = drawing()
    job = dict(iterations=20_000_000, walkers=16384, supersample=2, schedule="sorted")
    a, _, oa = renderer.histogram(cfg, 160, 120, plot="inline", **job)
    b, _, ob = renderer.histogram(cfg, 160, 120, plot="deferred", **job)
    assert oa.inframe_samples == ob.inframe_samples and np.array_equal(a, b)
