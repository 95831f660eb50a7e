"""`.flame` XML import (fae_call "flame_import", ffb_flame_import): Apophysis
and JWildfire flames as configs of this path (src/flame_xml.rs:41-1130;
wasm/python/src/lib.rs:214-218).  The cases follow the reference's own
tests in src/flame_xml.rs:1882-2625, written here as fresh XML.  Import is
host work and needs no GPU; the `gpu` tests render an imported flame.
"""

import json

import numpy as np
import pytest

from ffb200 import Engine, EngineError
from ffb200 import _native

f32 = np.float32


def imp(xml):
    return _native.flame_import(xml)


def one(xml):
    cs = imp(xml)
    assert len(cs) == 1
    return cs[0]


def flame(body, attrs='size="800 600" center="0 0" scale="200"', name="T"):
    return f'<flames name="t"><flame name="{name}" {attrs}>{body}</flame></flames>'


def test_spherical_example():
    # flame_xml.rs:1883-1909
    c = one('''<flames name="spherical-apo">
<flame name="Spherical Test" version="Apophysis 7x Version 15D" size="1500 1000"
 center="0.12666568780208 0.0566529891945883" scale="208.227773031847" background="0 0 0" brightness="1" gamma="1">
   <xform weight="1" color="0" spherical="1" coefs="0.9 0 0 0.9 0 0" opacity="1" />
</flame>
</flames>''')
    assert c["name"] == c["flame"]["name"] == "Spherical Test"
    assert c["render_mode"] == "TwoD"
    (t,) = c["flame"]["transforms"]
    assert t["weight"] == 1.0
    assert f32(t["a"]) == f32(0.9) and f32(t["d"]) == f32(0.9)
    assert t["variations"] == {"spherical": 1.0}
    assert c["image_size"] == [1500, 1000]
    assert f32(c["zoom"]) == f32(f32(208.227773031847) / f32(200.0))
    assert (f32(c["pan_x"]), f32(c["pan_y"])) == (f32(0.12666568780208), f32(0.0566529891945883))
    assert c["gamma"] == 1.0 and c["brightness"] == 1.0


def test_coef_order_column_major():
    # "a c b d e f" (flame_xml.rs:1912-1937)
    t = one(flame('<xform weight="1" linear="1" coefs="0.34284 0.564847 -0.564847 0.34284 1.5 2.5" />'))["flame"]["transforms"][0]
    assert [f32(t[k]) for k in "acbdef"] == [f32(v) for v in (0.34284, 0.564847, -0.564847, 0.34284, 1.5, 2.5)]


def test_variation_order_follows_the_attributes():
    # flame_xml.rs:1940-1961: dispatch order is the XML attribute order.
    def order(attrs):
        return one(flame(f'<xform weight="1" color="0.5" {attrs} coefs="1 0 0 1 0 0"/>'))["flame"]["transforms"][0]["variation_order"]
    assert order('swirl="0.5" sinusoidal="0.9"') == ["swirl", "sinusoidal"]
    assert order('sinusoidal="0.9" swirl="0.5"') == ["sinusoidal", "swirl"]
    # Variations this build lacks keep their place too (and are refused at render).
    assert order('roundspher3D="0.5" waves2="0.9"') == ["roundspher3D", "waves2"]


def test_jwf_flame_layered_first_layer_only():
    # flame_xml.rs:1964-1994
    c = one('''<jwf-flame name="Layered" size="800 600" center="0 0" scale="200" brightness="4">
  <layer weight="1.0" visible="true">
    <xform weight="1" color="0.2" linear="1" coefs="1 0 0 1 0 0"/>
    <xform weight="0.5" color="0.7" spherical="1" coefs="1 0 0 1 0 0"/>
  </layer>
  <layer weight="0.5" visible="true">
    <xform weight="1" color="0.9" julian="1" julian_power="3" coefs="1 0 0 1 0 0"/>
    <palette count="256" format="RGB">''' + "FF0000" * 256 + '''</palette>
  </layer>
  <bgxform weight="1" color="0" linear="1" coefs="1 0 0 1 0 0"/>
</jwf-flame>''')
    assert c["name"] == "Layered"
    ts = c["flame"]["transforms"]
    assert len(ts) == 2
    names = {k for t in ts for k in t["variations"]}
    assert names == {"linear", "spherical"}
    assert c["image_size"] == [800, 600] and c["brightness"] == 4.0
    assert "palette" not in c, "a palette of the second layer is not read"


def test_color_read_as_written():
    # flame_xml.rs:1997-2020: `color` is the first number as written, with
    # or without a <palette>.
    body = ('<xform weight="1" color="0.7" linear="1" coefs="1 0 0 1 0 0" />'
            '<xform weight="1" color="0.123456 0" linear="1" coefs="1 0 0 1 0 0" />'
            '<finalxform color="0.3" linear="1" coefs="1 0 0 1 0 0" />')
    pal = '<palette count="256" format="RGB">' + "808080" * 256 + "</palette>"
    for b in (body, body + pal):
        fl = one(flame(b, 'size="64 64" center="0 0" scale="20"'))["flame"]
        assert f32(fl["transforms"][0]["color"]) == f32(0.7)
        assert f32(fl["transforms"][1]["color"]) == f32(0.123456)
        assert f32(fl["final_transforms"][0]["color"]) == f32(0.3)


def test_fx_priority_attributes_are_not_variations():
    # `<var>_fx_priority` (flame_xml.rs:913-955) is a phase override, never
    # a variation or a parameter.
    t = one(flame('<xform weight="1" color="0.5" linear="1" curl="0.5" curl_fx_priority="-1" '
                  'linear_fx_priority="0" coefs="1 0 0 1 0 0" />'))["flame"]["transforms"][0]
    assert t["variations"] == {"linear": 1.0, "curl": 0.5}
    assert "variation_params" not in t


def test_variation_parameters():
    # flame_xml.rs:2125-2176, 986-1010: "name_param" of a known variation
    # is its parameter; a variation this build lacks keeps its parameters
    # under the same key form.
    ts = one(flame(
        '<xform weight="0.5" color="1" bubble="0.2" pre_blur="10" coefs="1 0 0 1 0 0" opacity="1" />'
        '<xform weight="6" color="0" flatten="1" julian="1" coefs="0.707107 -0.707107 0.707107 0.707107 0 -0.3" '
        'julian_power="2" julian_dist="-1" opacity="1" />'
        '<xform weight="1" color="0.5" curl="0.5" curl_c1="0.3" curl_c2="-0.2" coefs="1 0 0 1 0 0" />'))["flame"]["transforms"]
    assert len(ts) == 3
    assert ts[0]["weight"] == 0.5
    assert {k: f32(v) for k, v in ts[0]["variations"].items()} == {"bubble": f32(0.2), "pre_blur": f32(10)}
    assert ts[1]["weight"] == 6.0 and ts[1]["variations"] == {"flatten": 1.0, "julian": 1.0}
    assert ts[1]["variation_params"] == {"julian.power": 2.0, "julian.dist": -1.0}
    assert {k: f32(v) for k, v in ts[2]["variation_params"].items()} == {"curl.c1": f32(0.3), "curl.c2": f32(-0.2)}


def test_post_affine_import():
    # flame_xml.rs:2206-2249
    fl = one(flame(
        '<xform weight="0.5" color="1" bubble="0.2" coefs="1 0 0 1 0 0" post="0.8 0 0 1 0 0" opacity="1" />'
        '<xform weight="1" color="0" linear="1" coefs="0.9 0 0 0.9 0 0" opacity="1" />'
        '<finalxform color="0" linear="1" coefs="1 0 0 1 0 0" post="0.5 0.1 -0.1 0.5 0.2 0.3" />'))["flame"]
    t0, t1 = fl["transforms"]
    assert t0["post_affine_enabled"] is True
    assert [f32(t0["post_" + k]) for k in "acbdef"] == [f32(v) for v in (0.8, 0, 0, 1, 0, 0)]
    assert "post_affine_enabled" not in t1
    fin = fl["final_transforms"][0]
    assert fin["post_affine_enabled"] is True
    assert [f32(fin["post_" + k]) for k in "acbdef"] == [f32(v) for v in (0.5, 0.1, -0.1, 0.5, 0.2, 0.3)]


def test_multiple_finalxforms_attach_to_every_normal():
    # flame_xml.rs:2252-2293, 404-425 (migrate_legacy_final)
    fl = one(flame(
        '<xform weight="1" color="0" linear="1" coefs="1 0 0 1 0 0" opacity="1" />'
        '<xform weight="2" color="1" swirl="1" coefs="1 0 0 1 0 0" opacity="1" />'
        '<finalxform weight="0" color="0.1" spherical="1" coefs="1 0 0 1 0 0" />'
        '<finalxform weight="0" color="0.5" linear="1" coefs="2 0 0 2 0 0" />'
        '<finalxform weight="0" color="0.9" bubble="1" coefs="1 0 0 1 3 4" />'))["flame"]
    f0, f1, f2 = fl["final_transforms"]
    assert f0["variations"] == {"spherical": 1.0}
    assert f1["variations"] == {"linear": 1.0} and f1["a"] == 2.0 and f1["d"] == 2.0
    assert f2["variations"] == {"bubble": 1.0} and (f2["e"], f2["f"]) == (3.0, 4.0)
    assert (f0["weight"], f0["opacity"]) == (1.0, 1.0), "a final's weight attribute is not read"
    for t in fl["transforms"]:
        assert t["final_attachments"] == [0, 1, 2]


def test_symmetry_is_color_speed():
    # flame_xml.rs:2429-2454
    t = one(flame('<xform weight="1" color="0" linear="1" coefs="1 0 0 1 0 0" symmetry="0.42" opacity="1" />'))
    assert abs(t["flame"]["transforms"][0]["color_speed"] - 0.42) < 1e-6


def test_alias_is_stored_canonically_and_summed():
    # flame_xml.rs:2549-2596: cylinder_apo is cylinder; both sum.
    t = one(flame('<xform weight="1" color="0" cylinder_apo="0.8" spherical="0.2" coefs="1 0 0 1 0 0" />'))["flame"]["transforms"][0]
    assert set(t["variations"]) == {"cylinder", "spherical"} and abs(t["variations"]["cylinder"] - 0.8) < 1e-6
    t = one(flame('<xform weight="1" color="0" cylinder="0.25" cylinder_apo="0.5" coefs="1 0 0 1 0 0" />'))["flame"]["transforms"][0]
    assert t["variations"] == {"cylinder": 0.75} and t["variation_order"] == ["cylinder"]


def test_radial_blur_angle_is_converted_from_half_turns():
    # flame_xml.rs:957-974: the .flame stores radial_blur's angle in half
    # turns (1 = pure spin); the config holds degrees.
    t = one(flame('<xform weight="1" radial_blur="0.5" radial_blur_angle="0.5" coefs="1 0 0 1 0 0" />'))["flame"]["transforms"][0]
    assert t["variation_params"] == {"radial_blur.angle": 90.0}


def test_zero_weight_variation_is_dropped():
    # flame_xml.rs:697-716: a variation is stored only with a non-zero weight.
    t = one(flame('<xform weight="1" linear="1" swirl="0" coefs="1 0 0 1 0 0" />'))["flame"]["transforms"][0]
    assert t["variations"] == {"linear": 1.0} and t["variation_order"] == ["linear"]


def test_flame_attributes():
    # flame_xml.rs:110-255 (attributes), 414-432 (zoom, rotation, gamma threshold)
    c = one(flame('<xform weight="1" linear="1" coefs="1 0 0 1 0 0" />',
                  'size="640 480" center="0.5 -0.25" scale="100" rotate="90" background="255 128 0" brightness="3" '
                  'gamma="4" vibrancy="0.5" gamma_threshold="0.01" white_level="180" saturation="1.5" cam_zoom="2"'))
    assert c["image_size"] == [640, 480]
    assert c["zoom"] == 1.0 and (c["pan_x"], c["pan_y"]) == (0.5, -0.25)
    assert f32(c["rotation"]) == f32(f32(90.0) * f32(np.pi) / f32(180.0))
    assert [f32(v) for v in c["background_color"]] == [f32(1.0), f32(128 / 255), f32(0.0)]
    assert (c["brightness"], c["gamma"], c["vibrancy"]) == (3.0, 4.0, 0.5)
    assert f32(c["gamma_threshold"]) == f32(f32(0.01) * f32(2000.0) + f32(50.0))
    assert (c["white_level"], c["saturation"]) == (180.0, 1.5)
    assert c["tonemap_mode"] == "Logarithmic" and c["highlight_mode"] == "Clip" and c["use_curve"] is True
    # Defaults: gamma 2.2, gamma_threshold 0.0025 -> 55, size 1920x1080, scale 100 -> zoom 0.5.
    d = one('<flames><flame name="d"><xform weight="1" linear="1" coefs="1 0 0 1 0 0"/></flame></flames>')
    assert f32(d["gamma"]) == f32(2.2) and f32(d["gamma_threshold"]) == f32(55.0)
    assert d["image_size"] == [1920, 1080] and d["zoom"] == 0.5 and d["name"] == "d"


def test_palette_hex():
    # flame_xml.rs:1014-1066: 256 RGB colours, 6 hex digits each, whitespace ignored.
    cols = [(i, 255 - i, (7 * i) & 255) for i in range(256)]
    hexs = "".join("%02x%02X%02x" % c for c in cols)
    text = "\n".join(hexs[i:i + 48] for i in range(0, len(hexs), 48))
    c = one(flame('<xform weight="1" linear="1" coefs="1 0 0 1 0 0" />'
                  f'<palette count="256" format="RGB">\n{text}\n</palette>'))
    got = c["palette"]["indexed_colors"].split(",")
    assert len(got) == 256
    assert [tuple(int(g[k:k + 2], 16) for k in (0, 2, 4)) for g in got] == cols


def test_bad_palette_is_refused():
    with pytest.raises(EngineError, match="1536 hex characters"):
        imp(flame('<xform weight="1" linear="1" coefs="1 0 0 1 0 0" /><palette count="256" format="RGB">'
                  + "00" * 700 + "</palette>"))
    with pytest.raises(EngineError, match="not hex"):
        imp(flame('<xform weight="1" linear="1" coefs="1 0 0 1 0 0" /><palette count="256" format="RGB">'
                  + "0G0000" + "000000" * 255 + "</palette>"))


def test_curves_sampled_from_the_rational_bezier():
    # flame_xml.rs:1084-1150: the first 12 numbers (4 points x, y, w) are
    # sampled at t = 1/4, 1/2, 3/4 between (0, 0) and (1, 1).
    d = [0, 0, 1, 0.25, 0.5, 1, 0.75, 0.9, 2, 1, 1, 1] + [0, 0, 1, 0, 0, 1, 1, 1, 1, 1, 1, 1] * 3
    c = one(flame('<xform weight="1" linear="1" coefs="1 0 0 1 0 0" />',
                  'size="64 64" center="0 0" scale="20" curves="' + " ".join(str(v) for v in d) + '"'))
    pts = c["tonemap_curve"]["points"]
    assert len(pts) == 5 and pts[0] == {"x": 0, "y": 0} and pts[-1] == {"x": 1, "y": 1}
    P = np.array(d[:12], np.float64).reshape(4, 3)
    for k, t in enumerate((0.25, 0.5, 0.75)):
        b = np.array([(1 - t) ** 3, 3 * (1 - t) ** 2 * t, 3 * (1 - t) * t * t, t ** 3]) * P[:, 2]
        x, y = (b @ P[:, 0]) / b.sum(), (b @ P[:, 1]) / b.sum()
        assert abs(pts[k + 1]["x"] - x) < 1e-6 and abs(pts[k + 1]["y"] - y) < 1e-6
    # Not 48 numbers: the linear curve.
    c = one(flame('<xform weight="1" linear="1" coefs="1 0 0 1 0 0" />', 'curves="0 0 1"'))
    assert c["tonemap_curve"]["points"] == [{"x": 0, "y": 0}, {"x": 1, "y": 1}]


def test_post_symmetry_and_chaos():
    # Post-symmetry attributes, axis names swapped on the wire
    # (scene/transforms.rs:2116-2146); chaos rows default to 1
    # (flame_xml.rs:353-375).
    c = one(flame('<xform weight="1" linear="1" coefs="1 0 0 1 0 0" chaos="1 0.5" />'
                  '<xform weight="1" swirl="1" coefs="1 0 0 1 0 0" />',
                  'post_symmetry_type="X_AXIS" post_symmetry_order="4" post_symmetry_centre_x="0.5" '
                  'post_symmetry_centre_y="-1"'))
    s = c["flame"]["post_symmetry"]
    assert s["ty"] == "yaxis" and s["order"] == 4 and (s["center_x"], s["center_y"]) == (0.5, -1.0)
    assert c["flame"]["xaos"] == [[1, 0.5], [1, 1]]
    p = one(flame('<xform weight="1" linear="1" coefs="1 0 0 1 0 0" />', 'post_symmetry_type="point" post_symmetry_order="5"'))
    assert p["flame"]["post_symmetry"]["ty"] == "point" and "xaos" not in p["flame"]


def test_several_flames_and_entities():
    cs = imp('<?xml version="1.0"?>\n<!-- two -->\n<flames>'
             '<flame name="A &amp; B"><xform weight="1" linear="1" coefs="1 0 0 1 0 0"/></flame>'
             '<flame name="empty"/>'
             '<flame name="C"><![CDATA[ ignored ]]><xform weight="1" swirl="1" coefs="1 0 0 1 0 0"/></flame>'
             '</flames>')
    assert [c["name"] for c in cs] == ["A & B", "C"], "an empty <flame/> carries nothing"


def test_errors():
    with pytest.raises(EngineError, match="No <flame>"):
        imp("<flames></flames>")
    with pytest.raises(EngineError, match="3-D camera"):
        imp(flame('<xform weight="1" linear="1" coefs="1 0 0 1 0 0" />', 'cam_pitch="0.5"'))
    with pytest.raises(EngineError):
        imp("<flames><flame name='x'><xform weight='1'</flame>")


def test_fae_call_and_engine_agree():
    xml = flame('<xform weight="1" color="0.25" spherical="1" coefs="0.9 0 0 0.9 0 0" />')
    texts = Engine().flame_import(xml)
    assert isinstance(texts, list) and all(isinstance(t, str) for t in texts)
    assert [json.loads(t) for t in texts] == imp(xml)
    with pytest.raises(EngineError, match="xml"):
        Engine()._data({"fn": "flame_import"})


def test_imported_configs_specialize_or_say_why():
    # An imported flame compiles for this path, or is refused naming what
    # this build lacks.
    ok = one(flame('<xform weight="1" color="0.25" spherical="1" coefs="0.9 0 0 0.9 0 0" />'
                   '<xform weight="1" color="0.75" curl="1" curl_c1="0.2" coefs="0.5 0 0 0.5 0.5 0" />'
                   '<finalxform color="0" linear="1" coefs="1 0 0 1 0 0" post="0.9 0 0 0.9 0 0"/>'))
    n, src = _native.specialize(json.dumps(ok))
    assert n > 0 and src
    bad = one(flame('<xform weight="1" synth="1" synth_power="0.3" coefs="1 0 0 1 0 0" />'))
    assert bad["flame"]["transforms"][0]["variation_params"] == {"synth.power": f32(0.3)}
    with pytest.raises(EngineError, match="synth"):
        _native.specialize(json.dumps(bad))
    chaos = one(flame('<xform weight="1" linear="1" coefs="1 0 0 1 0 0" chaos="1 0" />'
                      '<xform weight="1" swirl="1" coefs="1 0 0 1 0 0" />'))
    _, src = _native.specialize(json.dumps(chaos))      # xaos is built: the chain specializes
    assert "#define FFB_XAOS 1" in src


# ---------------------------------------------------------------- on the GPU

PAL = "".join("%02X%02X%02X" % (i, (i * 3) & 255, 255 - i) for i in range(256))
XML = flame('<xform weight="1" color="0.1" spherical="1" coefs="0.9 0 0 0.9 0 0" />'
            '<xform weight="0.5" color="0.9" swirl="0.6" linear="0.4" coefs="0.5 0.2 -0.2 0.5 0.4 0.1" symmetry="0.3" />'
            '<finalxform color="0.5" linear="1" coefs="1 0 0 1 0 0" post="0.8 0 0 0.8 0 0" />'
            f'<palette count="256" format="RGB">{PAL}</palette>',
            'size="96 64" center="0.1 0" scale="150" background="0 0 0" brightness="2" gamma="3"')


def hand_config():
    """The flame XML above as a config written by hand."""
    def xf(a, b, c, d, e, f, **kw):
        return dict(a=a, b=b, c=c, d=d, e=e, f=f, **kw)
    return {
        "name": "T", "render_mode": "TwoD",
        "flame": {
            "name": "T",
            "transforms": [
                xf(0.9, 0, 0, 0.9, 0, 0, weight=1, color=0.1, color_speed=0, variations={"spherical": 1},
                   variation_order=["spherical"], final_attachments=[0]),
                # coefs "0.5 0.2 -0.2 0.5 0.4 0.1" are a c b d e f
                xf(0.5, -0.2, 0.2, 0.5, 0.4, 0.1, weight=0.5, color=0.9, color_speed=0.3,
                   variations={"swirl": 0.6, "linear": 0.4}, variation_order=["swirl", "linear"], final_attachments=[0]),
            ],
            "final_transforms": [xf(1, 0, 0, 1, 0, 0, weight=1, color=0.5, color_speed=0, variations={"linear": 1},
                                    post_affine_enabled=True, post_a=0.8, post_b=0, post_c=0, post_d=0.8, post_e=0, post_f=0)],
        },
        "zoom": 0.75, "pan_x": 0.1, "pan_y": 0, "rotation": 0, "background_color": [0, 0, 0],
        "brightness": 2, "gamma": 3, "vibrancy": 1, "gamma_threshold": 55, "white_level": 200, "saturation": 1,
        "tonemap_mode": "Logarithmic", "highlight_mode": "Clip", "use_curve": True, "exposure": 1,
        "palette": {"indexed_colors": ",".join(PAL[6 * i:6 * i + 6] for i in range(256))},
    }


def test_imported_flame_specializes_like_the_hand_written_one():
    a = _native.specialize(Engine().flame_import(XML)[0])
    b = _native.specialize(json.dumps(hand_config()))
    assert a == b


@pytest.mark.gpu
def test_imported_flame_renders_as_the_same_flame_written_by_hand():
    imported = json.loads(Engine().flame_import(XML)[0])
    hand = hand_config()
    imported["deterministic_rng"] = hand["deterministic_rng"] = True       # the same seed for both
    e = Engine()
    a = e.render(json.dumps(imported), 96, 64, iterations=400_000, iterations_per_thread=256)
    b = e.render(json.dumps(hand), 96, 64, iterations=400_000, iterations_per_thread=256)
    assert a.rgba == b.rgba
    px = np.frombuffer(a.rgba, np.uint8).reshape(64, 96, 4)
    assert px[..., :3].max() > 0, "the flame lit some pixels"


@pytest.mark.gpu
def test_imported_flame_through_the_typed_api():
    cfg = imp(XML)[0]
    r = _native.Renderer()
    try:
        rgba, _ = r.render(json.dumps(cfg), 96, 64, iterations=200_000, iterations_per_thread=256)
        assert rgba.shape == (64, 96, 4) and rgba[..., :3].max() > 0
    finally:
        r.close()
