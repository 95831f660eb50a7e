"""The variation registry beyond the benchmark configs' twelve: the
variations of the reference's ALL_VARIATIONS this build carries
(src/variations/defs/*.rs),
their parameters and init-derived values, several draws a body, bodies
that read their transform's affine or their own weight, and the Pre/Post
phases (pre_blur, flatten).

CPU: the registry the library reports against the oracle's, every
variation through NVRTC for sm_100a, the phases and draw slots in the
generated source, the differentiable render's refusal of a variation it
has no Jacobian for.

GPU (parity with the oracle, which tests/test_oracle_golden.py pins to the
reference's committed probe report):
* the 27-input probe of every variation: bit-identical where the body has
  no transcendental arithmetic, else within 4 ulp of the terms (the
  oracle's scale; near a floor/fract/comparison threshold the scale widens
  by the jump, see generic_scale in oracle/flame_oracle.cpp);
* with the SFU math mode, the reference report's class glyphs at every
  input where the oracle must match them (variations of at most one draw:
  later draws of the report came from an earlier stream);
* one step of transforms using every variation (non-default parameters,
  several draws, finals with Pre/Post variations) at 4096 points;
* whole renders: bit-identical count planes for a flame of exactly-rounded
  variations (both RNG modes), the sorted schedule walking the plain one's
  orbits with many draws an iteration, and log-density within Monte-Carlo
  noise of the oracle for a flame drawing 20 words an iteration.
"""

import ctypes
import json
import math

import numpy as np
import pytest

from ffb200 import Engine, EngineError, synthetic
from ffb200 import _native

from test_gpu_parity import within, bit_equal, log_density_l1
from test_oracle_golden import GOLDEN, LABELS, SFU_SIN, WIDER

PROBE_AFFINE = (1.0, 0.25, 0.1, -0.3, 0.9, -0.2)       # src/probe/flame.rs:4-12
# Bodies without transcendental arithmetic: +, -, *, /, sqrt, floor are
# correctly rounded on both sides, so the results are the same bits.
EXACT = {"linear", "spherical", "horseshoe", "bubble", "curl", "hyperbolic", "bent", "eyefish", "cross", "rings2",
         "rectangles", "splits", "butterfly", "fisheye", "stripes", "bent2", "linear3D", "flatten", "loonie", "scry",
         "separation", "mobius", "cell", "modulus", "square", "boarders",
         "blur_zoom", "blur_pixelize", "henon", "cylinder2", "flipcircle", "lozi", "bi_linear", "twoface", "flipy",
         "loonie3", "d_spherical", "hypertile3D", "voron", "minkQM", "poincare3D", "rosoni", "circleLinear",
         "plusrecip", "mobiq", "pointgrid_wf", "bubbleT3D", "cut_hexdots", "cut_fractal",
         "cut_snowflake"}


@pytest.fixture(scope="module")
def names(oracle):
    return sorted(oracle.REGISTRY, key=oracle.REGISTRY.get)


def wider(oracle):
    return [n for n in sorted(oracle.REGISTRY, key=oracle.REGISTRY.get) if n not in synthetic.TWELVE]


# --------------------------------------------------------------------- CPU --

def test_registry_is_the_oracles(oracle):
    """Names in registry order, and each variation's parameters."""
    lib = Engine().variations()
    assert list(lib) == sorted(oracle.REGISTRY, key=oracle.REGISTRY.get)
    for n, params in lib.items():
        assert params == [p for p, _ in oracle.PARAMS.get(n, [])], n


def test_every_variation_compiles_for_sm100a(oracle):
    """Flames using every variation of the registry between them (normal
    transforms, and a final chain holding Pre and Post ones; as many flames
    as keep each within the iteration's draw slots): NVRTC builds them (no
    device needed).  The subflame variations are a call of the subflame
    step, not a body of their own."""
    allv = sorted(oracle.REGISTRY, key=oracle.REGISTRY.get)
    parts, cur, d = [], [], 0
    for n in allv:                                   # at most 60 a flame, and 48 draws (the final takes more)
        k = oracle.var_meta(n)[0]
        if cur and (len(cur) == 60 or d + k > 48):
            parts.append(cur)
            cur, d = [], 0
        cur.append(n)
        d += k
    parts.append(cur)
    src = ""
    for part in parts:
        xfs = [{"a": 0.5, "b": 0.1, "c": -0.1, "d": 0.5, "e": 0.2, "f": -0.3, "weight": 1.0, "color": i / 10,
                "variations": {n: 0.3 for n in part[i:i + 6]}} for i in range(0, len(part), 6)]
        fin = {"a": 1, "b": 0, "c": 0, "d": 1, "e": 0, "f": 0, "weight": 1, "color": 0.5,
               "variations": {"pre_blur": 0.1, "linear": 1.0, "flatten": 1.0, "blur": 0.2}}
        cfg = {"flame": {"transforms": xfs, "final_transforms": [fin]}}
        n, part_src = _native.specialize(json.dumps(cfg))
        assert n > 0
        src += part_src
    for v in allv:
        if v in ("subflame_wf", "pre_subflame_wf"):
            assert f"ffb_subflame(sm, ctx, sq, " in src and f"}} }}   // {v}\n" in src, v
        else:
            assert f"v_{v}(" in src, v


def test_phases_and_draw_slots_in_the_generated_source():
    """pre_blur replaces the input before the weighted sum, flatten replaces
    the sum after it; a body's draws take consecutive slots from 2."""
    cfg = {"flame": {"transforms": [{"a": 1, "b": 0, "c": 0, "d": 1, "e": 0, "f": 0, "weight": 1, "color": 0,
                                     "variations": {"gaussian_blur": 0.5, "pre_blur": 0.2, "flatten": 1.0, "blur": 0.3}}]}}
    _, src = _native.specialize(json.dumps(cfg))
    body = src[src.index("void ffb_normal("):]
    body = body[:body.index("\n}\n")]
    pre, gb, bl, fl = (body.index(s) for s in ("v_pre_blur(tx, ty, rng, ", "v_gaussian_blur(tx, ty, rng, ",
                                               "v_blur(tx, ty, rng, ", "v_flatten(rx, ry"))
    assert pre < gb < fl and pre < bl < fl
    # local order: blur (30), gaussian_blur (31), pre_blur (54): slots 2-3, 4-8, 9-15
    assert "v_blur(tx, ty, rng, 2," in body and "v_gaussian_blur(tx, ty, rng, 4," in body
    assert "v_pre_blur(tx, ty, rng, 9," in body
    assert "#define FFB_NSLOTS 16" in src


def test_derived_values_are_the_oracles(oracle):
    """wgsl_init values the library packs beside the user parameters."""
    for name, user in (("julian", [3.0, 0.7]), ("wedge", [45.0, 0.1, 3.0, 0.2]), ("radial_blur", [30.0]),
                       ("perspective", [0.3, 1.5])):
        row = oracle.var_row(name, user)
        _, _, nd, _ = oracle.var_meta(name)
        assert nd > 0 and np.all(np.isfinite(row))
    assert oracle.var_row("julian", [2.0, 1.0])[2] == np.float32(0.25)           # dist / |power| / 2


def test_diff_refuses_a_variation_without_a_jacobian(native):
    cfg = {"flame": {"transforms": [{"a": 0.5, "b": 0, "c": 0, "d": 0.5, "e": 0, "f": 0, "weight": 1.0, "color": 0.3,
                                     "variations": {"linear": 0.5, "blur": 0.1}}]}}
    c = json.dumps(cfg).encode()
    n = ctypes.c_size_t()
    buf = ctypes.create_string_buffer(1 << 21)
    L = native.lib()
    st = L.ffb_diff_specialize(c, ctypes.c_size_t(len(c)), 16, 64, ctypes.byref(n), buf, ctypes.c_size_t(len(buf)))
    assert st != 0
    msg = L.ffb_last_error().decode()
    assert "blur" in msg and "Jacobian" in msg


def test_too_many_draws_are_refused():
    xf = {"a": 1, "b": 0, "c": 0, "d": 1, "e": 0, "f": 0, "weight": 1, "color": 0, "variations": {"pre_blur": 0.1}}
    cfg = {"flame": {"transforms": [dict(xf, final_attachments=list(range(8)))],
                     "final_transforms": [dict(xf) for _ in range(8)]}}   # 2 + 7 + 8 * 7 = 65 draws
    with pytest.raises(EngineError, match="random draws"):
        _native.specialize(json.dumps(cfg))


# --------------------------------------------------------------------- GPU --

def probe_cfg(name, copies=1, phase=1):
    t = {"a": PROBE_AFFINE[0], "b": PROBE_AFFINE[1], "c": PROBE_AFFINE[2], "d": PROBE_AFFINE[3], "e": PROBE_AFFINE[4],
         "f": PROBE_AFFINE[5], "weight": 1.0, "color": 0.5, "variations": {name: 1.0}}
    if phase in (0, 2):                              # the probe's `linear` carrier (src/probe/batch.rs:26-47)
        t["variations"] = {"linear": 1.0, name: 1.0}
        t["variation_order"] = ["linear", name]
    return {"flame": {"transforms": [t] * copies}, "deterministic_rng": True}


@pytest.fixture(scope="module")
def probe_pts():
    vals = []
    for x, y in [(0.0, 0.0), (0.0, -0.0), (-0.0, 0.0), (-0.0, -0.0), (1, 0), (-1, 0), (0, 1), (0, -1), (1, 1), (-1, 1),
                 (-1, -1), (1, -1), (0.5, 0.3), (0.12345679, -0.9876543), (2.5, -1.5), (math.pi, math.e), (1, 0),
                 (0.70710677, 0.70710677), (1e-20, -1e-20), (1.1754944e-38, 1.1754944e-38), (1e-40, -1e-40),
                 (1e20, -1e20), (9e31, -9e31), (1e33, -1e33), (1e30, 1e-30), (1.0, -0.0), (-0.0, 1.0)]:
        vals += [x, y]
    return np.array(vals, np.float32).reshape(-1, 2)


@pytest.mark.gpu
@pytest.mark.parametrize("name", [n for n in sorted(GOLDEN) if n not in synthetic.TWELVE])
def test_probe_matches_oracle(renderer, oracle, probe_pts, name):
    """The 27-input probe at transform 0, precise math: the oracle's values
    (its probe at slot 0, current stream), bit for bit for EXACT bodies."""
    draws_n, _, _, phase = oracle.var_meta(name)
    out = renderer.probe(probe_cfg(name, 1, phase), probe_pts, 1)[0]
    _, _, ref = oracle.probe(name, xform_slot=0, fold_first=False)
    ref = ref.reshape(27, 2)
    if name in EXACT:
        ok = bit_equal(out, ref)
    else:
        flushed = np.where(np.abs(probe_pts) < 1.17549435e-38, np.copysign(0.0, probe_pts), probe_pts).astype(np.float32)
        draws = np.array([oracle.probe_draws(i, max(draws_n, 1)) for i in range(27)], np.float32)
        if phase == 0:    # pre(p) feeds 0 + 1 * p: the pre variation's own scale
            sx, sy = oracle.variation_scale(name, flushed[:, 0], flushed[:, 1], draws, xf=PROBE_AFFINE)
        else:
            sx, sy = oracle.variation_scale(name, flushed[:, 0], flushed[:, 1], draws if draws_n else None, xf=PROBE_AFFINE)
        ok = within(out, ref, np.stack([sx, sy], axis=1))
    bad = [(LABELS[i], probe_pts[i].tolist(), out[i].tolist(), ref[i].tolist()) for i in range(27) if not ok[i].all()]
    assert not bad, f"{name}: {bad}"


@pytest.mark.gpu
@pytest.mark.parametrize("name", [n for n in sorted(GOLDEN) if n not in synthetic.TWELVE])
def test_sfu_probe_reproduces_the_reference_report(renderer, oracle, probe_pts, name):
    """With the approximate sin/cos/exp/log/tan of math = sfu, at the
    variation's batch slot: the reference report's glyph at every input
    where the oracle must match it (inputs listed in the oracle test's
    tables may differ).  Bodies of two or more draws are compared through
    the oracle only: the report's later draws came from an earlier stream."""
    draws_n, _, _, phase = oracle.var_meta(name)
    if draws_n > 1:
        pytest.skip("later draws of the report come from an earlier stream (test_oracle_golden.py)")
    gold, _, slot = GOLDEN[name]
    out = renderer.probe(probe_cfg(name, slot + 1, phase), probe_pts, slot + 1, math="sfu")[slot].reshape(-1)
    classes, _ = oracle.probe_digest(out)
    if slot == 0 or name == "flatten":
        # signed zeros: the reference compiler folded 0 + x into x for the batch's first variation
        # and for a Post variation's carrier
        gold, classes = gold.replace("o", "0"), classes.replace("o", "0")
    allowed = set(WIDER.get(name, {})) | set(SFU_SIN.get(name, {}))
    bad = [(LABELS[i], classes[2 * i:2 * i + 2], gold[2 * i:2 * i + 2]) for i in range(27)
           if classes[2 * i:2 * i + 2] != gold[2 * i:2 * i + 2] and LABELS[i] not in allowed]
    assert not bad, f"{name}: {bad}"


def wider_flames(oracle, budget=40):
    """The variations beyond the twelve split over flames whose draws fit
    the iteration's slots (a final chain takes 11 more)."""
    chunks, cur, d = [], [], 0
    for n in wider(oracle):
        k = oracle.var_meta(n)[0]
        if cur and d + k > budget:
            chunks.append(cur)
            cur, d = [], 0
        cur.append(n)
        d += k
    chunks.append(cur)
    return [wider_flame(oracle, c, 11 + j) for j, c in enumerate(chunks)]


def wider_flame(oracle, names, seed=11):
    """Transforms using `names` at random weights, non-default parameters;
    a final chain with Pre and Post variations."""
    rng = np.random.default_rng(seed)
    xfs = []
    for i in range(0, len(names), 5):
        group = names[i:i + 5]
        a = rng.uniform(-0.8, 0.8, 6)
        params = {}
        for n in group:
            for p, d in oracle.PARAMS.get(n, []):
                params[f"{n}.{p}"] = float(np.float32(d * rng.uniform(0.6, 1.4) + rng.uniform(-0.2, 0.2)))
        if "juliascope.power" in params:
            params["juliascope.power"] = 3.0
        if "julian.power" in params:
            params["julian.power"] = -3.0
        xfs.append({"a": a[0], "b": a[1], "c": a[2], "d": a[3], "e": a[4], "f": a[5], "weight": float(rng.uniform(0.3, 1)),
                    "color": float(rng.uniform()), "variations": {n: float(rng.uniform(0.1, 0.8)) for n in group},
                    "variation_params": params, "post_affine_enabled": i % 2 == 1, "post_a": 0.9, "post_b": 0.1,
                    "post_c": -0.1, "post_d": 0.9, "post_e": 0.05, "post_f": 0.0})
    fins = [{"a": 0.9, "b": 0.1, "c": -0.1, "d": 0.9, "e": 0.0, "f": 0.1, "weight": 1, "color": 0.2,
             "variations": {"pre_blur": 0.05, "linear": 0.8, "waves": 0.2, "flatten": 1.0}},
            {"a": 1.0, "b": 0.0, "c": 0.0, "d": 1.0, "e": 0.1, "f": 0.0, "weight": 1, "color": 0.7,
             "variations": {"rings": 0.3, "spherical": 0.4, "radial_blur": 0.2}, "variation_params": {"radial_blur.angle": 40.0}}]
    for t in xfs:
        t["final_attachments"] = [0, 1]
    return {"flame": {"transforms": xfs, "final_transforms": fins}, "deterministic_rng": True}


@pytest.mark.gpu
def test_apply_points_every_variation(renderer, oracle):
    n = 4096
    rng = np.random.default_rng(5)
    xs = rng.uniform(-2.5, 2.5, n).astype(np.float32)
    ys = rng.uniform(-2.5, 2.5, n).astype(np.float32)
    words = (rng.integers(0, 1 << 24, (n, 64)) / float(1 << 24)).astype(np.float32)
    for f, cfg in enumerate(wider_flames(oracle)):
        fl = oracle.Flame(cfg, 64, 64)
        n_all = len(cfg["flame"]["transforms"]) + len(cfg["flame"]["final_transforms"])
        for xi in range(n_all):
            for aff in (True, False):
                gx, gy = renderer.apply_points(cfg, xi, xs, ys, words, with_affine=aff)
                rx, ry, sx, sy = fl.apply_xform(xi, xs, ys, words, with_affine=aff, scales=True)
                ok = within(gx, rx, 4 * sx) & within(gy, ry, 4 * sy)
                bad = np.where(~ok)[0]
                names = list(cfg["flame"]["transforms"][xi]["variations"]) if xi < len(cfg["flame"]["transforms"]) else "final"
                assert len(bad) <= n // 1000, (f, xi, names, aff, len(bad),
                                               [(xs[i], ys[i], gx[i], rx[i], gy[i], ry[i], sx[i], sy[i]) for i in bad[:4]])


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(EXACT))
def test_exactly_rounded_bodies_are_bit_identical(renderer, oracle, name):
    """One step of a transform holding only `name` (weight 1, non-default
    parameters) at 65,536 points across magnitudes: the same bits."""
    rng = np.random.default_rng(REG_SEED + oracle.REGISTRY[name])
    n = 65536
    mag = 10.0 ** rng.uniform(-6, 6, n)
    xs = (rng.choice([-1, 1], n) * mag * rng.random(n)).astype(np.float32)
    ys = (rng.choice([-1, 1], n) * 10.0 ** rng.uniform(-6, 6, n) * rng.random(n)).astype(np.float32)
    params = {f"{name}.{p}": float(np.float32(d * 0.7 + 0.11)) for p, d in oracle.PARAMS.get(name, [])}
    t = {"a": 1, "b": 0, "c": 0, "d": 1, "e": 0, "f": 0, "weight": 1.0, "color": 0.5, "variations": {name: 1.0},
         "variation_params": params}
    cfg = {"flame": {"transforms": [t]}}
    words = (rng.integers(0, 1 << 24, (n, 64)) / float(1 << 24)).astype(np.float32)   # the draws of square, boarders, the blurs
    gx, gy = renderer.apply_points(cfg, 0, xs, ys, words, with_affine=False)
    rx, ry = oracle.Flame(cfg, 8, 8).apply_xform(0, xs, ys, words, with_affine=False)
    ok = bit_equal(gx, rx) & bit_equal(gy, ry)
    bad = np.where(~ok)[0]
    assert len(bad) == 0, (name, len(bad), [(xs[i], ys[i], gx[i], rx[i], gy[i], ry[i]) for i in bad[:4]])


REG_SEED = 900


def exact_flame():
    """A flame of correctly rounded bodies only."""
    def t(a, b, c, d, e, f, w, col, v, **kw):
        return dict(a=a, b=b, c=c, d=d, e=e, f=f, weight=w, color=col, variations=v, **kw)
    xfs = [t(0.5, 0.1, -0.1, 0.5, 0.3, 0.2, 1.0, 0.1, {"bent": 0.6, "hyperbolic": 0.3}),
           t(0.4, -0.3, 0.3, 0.4, -0.4, 0.1, 0.8, 0.4, {"eyefish": 0.7, "cross": 0.05, "linear3D": 0.2}),
           t(-0.5, 0.2, 0.1, 0.6, 0.1, -0.3, 0.6, 0.7, {"rectangles": 0.4, "splits": 0.3, "bent2": 0.3},
             variation_params={"rectangles.x": 0.3, "rectangles.y": 0.45, "bent2.x": 0.7, "bent2.y": 1.3}),
           t(0.3, 0.4, -0.4, 0.3, 0.2, 0.4, 0.7, 0.9, {"stripes": 0.5, "fisheye": 0.3, "butterfly": 0.2, "rings2": 0.1},
             variation_params={"rings2.val": 0.4}, final_attachments=[0]),
           ]
    for x in xfs:
        x["final_attachments"] = [0]
    fin = t(0.9, 0.0, 0.0, 0.9, 0.0, 0.0, 1, 0.5, {"linear": 1.0, "flatten": 1.0})
    return {"flame": {"transforms": xfs, "final_transforms": [fin]}, "deterministic_rng": True}   # seed 12345, the oracle's


@pytest.mark.gpu
@pytest.mark.parametrize("rng_mode", ["pcg", "philox"])
def test_histogram_bit_exact_for_exactly_rounded_variations(renderer, oracle, rng_mode):
    cfg = exact_flame()
    W, H = 96, 64
    job = dict(iterations=2048 * 500, walkers=2048, rng=rng_mode, iterations_per_thread=256)
    cnt, rgb, out = renderer.histogram(cfg, W, H, **job)
    fl = oracle.Flame(cfg, W, H)
    plotted, inframe, rc, rr = fl.render(2048, 500 + 20, rng=rng_mode, ipt=256, threads=8)
    assert out.total_iterations == plotted
    assert int(cnt.sum()) == out.inframe_samples == inframe > 0
    assert np.array_equal(cnt, rc)


def hide_flame():
    """Feature::CanHide on the exactly rounded flame: a transform of
    circlecrop at radius 0 (every point escapes: the iteration is dropped
    and the point reverts) and a final circlecrop of radius 0.8 (samples
    outside it are not plotted, the rest pass unchanged), and a transform
    whose circlecrop hides every point before a cut_hexdots stencil on the
    point (mode 0) assigns the flag again: the stencil's verdict stands."""
    cfg = exact_flame()
    xfs = cfg["flame"]["transforms"]
    xfs.append(dict(a=0.7, b=0.1, c=-0.2, d=0.6, e=0.1, f=0.1, weight=0.9, color=0.3, variations={"circlecrop": 1.0},
                    variation_params={"circlecrop.radius": 0.0}))
    xfs.append(dict(a=0.6, b=-0.2, c=0.2, d=0.7, e=-0.2, f=0.1, weight=0.7, color=0.8,
                    variations={"circlecrop": 0.5, "cut_hexdots": 0.9},
                    variation_params={"circlecrop.radius": 0.0, "cut_hexdots.mode": 0.0, "cut_hexdots.zoom": 3.0}))
    fin = dict(a=1.0, b=0.0, c=0.0, d=1.0, e=0.0, f=0.0, weight=1, color=0.5, variations={"circlecrop": 1.0},
               variation_params={"circlecrop.radius": 0.8})
    cfg["flame"]["final_transforms"].append(fin)
    for x in xfs:
        x["final_attachments"] = [0, 1]
    return cfg


@pytest.mark.gpu
@pytest.mark.parametrize("rng_mode", ["pcg", "philox"])
def test_canhide_drops_iterations_and_samples(renderer, oracle, rng_mode):
    """main_template.wgsl:389-400, 725-731: a hiding normal transform
    reverts the point and drops the iteration, a hiding final drops the
    sample; the orbits stay exact, so the count planes match bit for bit."""
    cfg = hide_flame()
    W, H = 96, 64
    job = dict(iterations=2048 * 300, walkers=2048, rng=rng_mode, iterations_per_thread=256)
    cnt, rgb, out = renderer.histogram(cfg, W, H, **job)
    fl = oracle.Flame(cfg, W, H)
    plotted, inframe, rc, rr = fl.render(2048, 300 + 20, rng=rng_mode, ipt=256, threads=8)
    assert int(cnt.sum()) == out.inframe_samples == inframe > 0
    assert np.array_equal(cnt, rc)
    # the hidden transform and the final's rim take samples away
    cfg_open = exact_flame()
    cnt_open, _, _ = renderer.histogram(cfg_open, W, H, **job)
    assert int(cnt.sum()) < int(cnt_open.sum())


@pytest.mark.gpu
def test_sorted_schedule_with_many_draws(renderer, oracle):
    """20 draw words an iteration (5 blocks of the counter stream): the
    regrouped walkers keep their streams.  The flames alternate between
    the two streams (each flame's four modules compile separately)."""
    job = dict(iterations=2_000_000, walkers=6000, supersample=1)
    for f, cfg in enumerate(wider_flames(oracle)):
        for rng in (("philox", "pcg")[f % 2],):
            a, _, oa = renderer.histogram(cfg, 160, 90, schedule="plain", rng=rng, iterations_per_thread=64, **job)
            b, _, ob = renderer.histogram(cfg, 160, 90, schedule="sorted", rng=rng, iterations_per_thread=64, **job)
            assert np.array_equal(a, b), (f, rng)
            assert oa.inframe_samples == int(a.sum()) > 0, (f, rng)


def drawing_flame():
    """Four transforms of the drawing and transcendental variations."""
    def t(a, w, col, v, p=None):
        d = dict(a=a[0], b=a[1], c=a[2], d=a[3], e=a[4], f=a[5], weight=w, color=col, variations=v)
        if p:
            d["variation_params"] = p
        return d
    xfs = [t((0.6, 0.1, -0.1, 0.6, 0.2, 0.1), 1.0, 0.1, {"julian": 0.7, "gaussian_blur": 0.1, "pre_blur": 0.05},
             {"julian.power": 3.0, "julian.dist": 0.8}),
           t((0.5, -0.3, 0.3, 0.5, -0.3, 0.2), 0.8, 0.5, {"juliascope": 0.6, "blur": 0.2, "noise": 0.1}),
           t((0.4, 0.2, -0.2, 0.4, 0.3, -0.3), 0.6, 0.8, {"pie": 0.3, "radial_blur": 0.3, "heart": 0.2, "waves": 0.2},
             {"radial_blur.angle": 60.0}),
           t((0.7, 0.0, 0.0, 0.7, -0.2, -0.2), 0.5, 0.3, {"spiral": 0.3, "ngon": 0.2, "fan2": 0.2, "wedge": 0.3},
             {"fan2.x": 0.6, "fan2.y": 0.3})]
    return {"flame": {"transforms": xfs}, "deterministic_rng": True}


@pytest.mark.gpu
@pytest.mark.parametrize("rng_mode", ["philox", "pcg"])
def test_histogram_with_draws_within_monte_carlo_noise(renderer, oracle, rng_mode):
    cfg = drawing_flame()
    W = H = 128
    walkers, per = 8192, 400
    cnt, _, out = renderer.histogram(cfg, W, H, iterations=walkers * per, walkers=walkers, seed=1001, rng=rng_mode,
                                     iterations_per_thread=256)
    fl = oracle.Flame(cfg, W, H)
    _, _, o1, _ = fl.render(walkers, per + 20, seed=1001, rng=rng_mode, ipt=256, threads=8)
    _, _, o2, _ = fl.render(walkers, per + 20, seed=2002, rng=rng_mode, ipt=256, threads=8)
    assert o1.sum() > 1000
    l1_go, p99_go = log_density_l1(cnt, o1)
    l1_oo, p99_oo = log_density_l1(o2, o1)
    assert l1_go <= 1.25 * l1_oo + 0.01, (l1_go, l1_oo)
    assert p99_go <= 1.25 * p99_oo + 0.05, (p99_go, p99_oo)
