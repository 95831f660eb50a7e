"""Host-side checks of the C ABI that need no GPU: the library loads and
exports every function include/ffb200.h declares; the flame parser refuses
what the reference refuses; NVRTC specialises flames for sm_100a."""

import json
import os
import re

import pytest

from ffb200 import synthetic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "ffb200.h"), encoding="utf-8").read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b((?:fae|ffb)_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(native):
    L = native.lib()
    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    assert sorted(native.EXPORTS) == names


def test_version(native):
    assert b"sm_100a" in native.lib().ffb_version()


def _specialize_status(native, cfg):
    try:
        native.specialize(cfg)
        return native.OK, ""
    except native.EngineError as e:
        return e.status, str(e)


def test_unknown_variation_is_refused(native):
    cfg = synthetic.plain_flame(1)
    cfg["flame"]["transforms"][0]["variations"]["blob_not_here"] = 1.0
    st, msg = _specialize_status(native, cfg)
    assert st == native.ERR_CONFIG and "blob_not_here" in msg


def test_transform_cap(native):
    """compute_kernel.rs:6487-6499: 129 transforms -> TooLarge naming the count."""
    t = synthetic.plain_flame(1)["flame"]["transforms"][0]
    cfg = {"flame": {"transforms": [t] * 129}}
    st, msg = _specialize_status(native, cfg)
    assert st == native.ERR_CONFIG and "129" in msg


def test_missing_fields(native):
    for bad in ({}, {"flame": {}}, {"flame": {"transforms": [{"a": 1}]}}):
        st, msg = _specialize_status(native, bad)
        assert st == native.ERR_CONFIG, bad
    st, msg = _specialize_status(native, "{not json")
    assert st == native.ERR_CONFIG and "JSON" in msg


@pytest.mark.parametrize("make", [lambda: synthetic.plain_flame(3), lambda: synthetic.full_flame(7),
                                  synthetic.sierpinski])
@pytest.mark.parametrize("rng", ["pcg", "philox"])
def test_nvrtc_specialises_for_sm100a(native, make, rng):
    n, src = native.specialize(make(), rng=rng)
    assert n > 10000
    assert "ffb_chaos" in src and "#define FFB_RNG_MODE %d" % native.RNG[rng] in src


def test_specialisation_is_structural(native):
    """Flames of one structure share a compiled module: only the table differs."""
    a = synthetic.plain_flame(3)
    b = json.loads(json.dumps(a))
    for t in b["flame"]["transforms"]:
        t["a"] *= 0.5
        t["weight"] += 0.1
    assert native.specialize(a)[1] == native.specialize(b)[1]


def test_dispatch_order_follows_variation_order(native):
    """transforms.rs:668-682: `variation_order` first, then registry order."""
    t = {"a": 1, "b": 0, "c": 0, "d": 1, "e": 0, "f": 0, "weight": 1, "color": 0,
         "variations": {"spherical": 0.5, "linear": 0.5}}
    _, src = native.specialize({"flame": {"transforms": [t]}})
    body = src[src.index("ffb_normal(const"):]
    assert body.index("v_linear(") < body.index("v_spherical(")
    t2 = dict(t, variation_order=["spherical", "linear"])
    _, src = native.specialize({"flame": {"transforms": [t2]}})
    body = src[src.index("ffb_normal(const"):]
    assert body.index("v_spherical(") < body.index("v_linear(")


def test_fae_call_without_a_gpu_answers_data_calls(native):
    from ffb200 import Module
    m = Module()
    out, info = m.call({"fn": "variations"})
    names = [v["name"] for v in info["result"]]
    assert names[:3] == ["linear", "sinusoidal", "spherical"] and "curl" in names
    out, info = m.call({"fn": "info"})
    assert "version" in info["result"]
    with pytest.raises(native.EngineError):
        m.call({"fn": "flame_import", "xml": "<flame/>"})
    with pytest.raises(native.EngineError):
        m.call({"no": "fn"})


def test_struct_layouts_match_the_header(native):
    """The ctypes mirrors of ffb_job and ffb_output have the C layouts."""
    import ctypes
    jb, ob = ctypes.c_size_t(), ctypes.c_size_t()
    native.lib().ffb_struct_sizes(ctypes.byref(jb), ctypes.byref(ob))
    assert jb.value == ctypes.sizeof(native.Job) and ob.value == ctypes.sizeof(native.Output)


@pytest.mark.gpu
def test_progress_reports_and_cancel_stops(renderer, native):
    """RenderProgress (render.rs:293-301, 624-693): progress after each
    launch, rising to the render's total; a cancel before a launch ends the
    render with the Cancelled status."""
    cfg = synthetic.plain_flame(2)
    seen = []
    job = dict(iterations=1024 * 300_000, walkers=1024)             # five launches of 65,536 iterations
    renderer.histogram(cfg, 128, 128, progress=lambda c, t: seen.append((c, t)), **job)
    assert len(seen) == 5
    assert all(b[0] > a[0] for a, b in zip(seen, seen[1:]))
    assert seen[-1][0] == seen[-1][1] == 1024 * 300_000
    calls = []

    def cancel():
        calls.append(1)
        return len(calls) > 2
    with pytest.raises(native.EngineError) as e:
        renderer.histogram(cfg, 128, 128, cancel=cancel, **job)
    assert e.value.status == native.ERR_CANCELLED and len(calls) == 3
    # The renderer is usable after a cancel.
    cnt, _, out = renderer.histogram(cfg, 128, 128, **job)
    assert out.total_iterations == 1024 * 300_000
