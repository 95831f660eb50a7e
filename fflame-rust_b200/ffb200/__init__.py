"""ffb200 -- the B200-native fractal-flame render path of calibas/fflame-rust.

The Python face mirrors the reference's client (python/pyfae/__init__.py):
`Engine().render(config, width, height, iterations=..., ...)` -> Image.  It
drives the CUDA library through the reference's own boundary (`fae_call`,
a JSON request), so code written against pyfae runs unchanged apart from
the import.  `Renderer` is the typed API underneath (include/ffb200.h).
"""

import json

from ._module import Module, find_module
from ._native import Batch, EngineError, Output, Renderer, make_job, specialize  # noqa: F401

__all__ = ["Engine", "Image", "Module", "EngineError", "Renderer", "Batch", "specialize"]


def _text(config):
    if isinstance(config, str):
        if config.lstrip().startswith("{"):
            return config
        with open(config, encoding="utf-8") as f:
            return f.read()
    if hasattr(config, "data"):
        config = config.data
    return json.dumps(config)


class Image:
    """A render: RGBA8 bytes and the engine's note (pyfae's Image)."""

    def __init__(self, engine, rgba, info, config_text):
        self.engine = engine
        self.rgba = rgba
        self.info = info or {}
        self.config = config_text

    @property
    def width(self):
        return self.info.get("width")

    @property
    def height(self):
        return self.info.get("height")

    def array(self):
        import numpy as np
        return np.frombuffer(self.rgba, np.uint8).reshape(self.height, self.width, 4)

    def png(self):
        """The PNG the reference's CLI writes for this frame, its config and
        numbers in the metadata (python/pyfae/__init__.py:88-97)."""
        out, _ = self.engine._module.call({
            "fn": "encode_png", "config": self.config if isinstance(self.config, str) else self.config.decode(),
            "width": self.width, "height": self.height, "iterations": self.info.get("iterations", 0),
            "ms": self.info.get("ms", 0.0), "iterations_per_thread": self.info.get("iterations_per_thread", 1024),
        }, self.rgba)
        return out

    def save(self, path):
        with open(path, "wb") as f:
            f.write(self.png())


class Engine:
    """The engine (pyfae.Engine, python/pyfae/__init__.py:159-221)."""

    def __init__(self, module=None):
        self._module = Module(module)

    def _call(self, request, data=b""):
        return self._module.call(request, data)

    def _data(self, request, data=b""):
        return self._call(request, data)[1]["result"]

    def info(self):
        return self._data({"fn": "info"})

    def flame_import(self, xml):
        """`.flame` XML -> config JSON strings, one a flame (wasm/python/src/lib.rs:214-218)."""
        if isinstance(xml, (bytes, bytearray)):
            xml = bytes(xml).decode("utf-8")
        elif not (isinstance(xml, str) and xml.lstrip().startswith("<")):
            with open(xml, encoding="utf-8") as f:                 # a path
                xml = f.read()
        return self._data({"fn": "flame_import", "xml": xml})

    def variations(self):
        """{name: [parameter names]} in registration order."""
        return {v["name"]: v["params"] for v in self._data({"fn": "variations"})}

    def render(self, config, width, height, *, iterations=None, iterations_per_thread=None,
               transparent=False, premultiplied=False, sticky=False, sequence=False, supersample=None, walkers=None,
               exact=False, accumulate=None):
        """A config (dict, JSON, or a path) at `width` x `height` (python/pyfae/__init__.py:201-221).

        `iterations`: the flame's budget (default: the config's own).
        `iterations_per_thread`: default the CLI's, 1024.  `supersample` 2
        renders at twice the size and boxes it down with the firefly clamp;
        `walkers` fixes the number of concurrent orbits (default: sized to
        the budget); `exact` accumulates u64 counts and fixed-point colour
        sums (long renders, order-independent results); `accumulate`
        ("direct" or "tiled") picks how the sums are gathered.

        `sticky` and `sequence` are accepted for pyfae's signature and change
        nothing here.  The reference's `sticky` compiles a superset shader
        to save recompiles across flames, at the cost of the specialised
        shader's exact picture (wasm/python/src/render.rs:50-52, 155); this
        library always renders the specialised picture, and flames sharing a
        structure already share one compiled module.  `sequence` continues a
        simulation engine's state from the previous sequence frame
        (render.rs:185-199); a fractal flame carries no engine state between
        frames, so a sequence frame is the same render as a still.
        """
        text = _text(config)
        request = {"fn": "render", "config": text, "width": width, "height": height,
                   "transparent": transparent, "premultiplied": premultiplied,
                   "sticky": sticky, "sequence": sequence}
        if iterations:
            request["iterations"] = int(iterations)
        if iterations_per_thread:
            request["iterations_per_thread"] = int(iterations_per_thread)
        if supersample:
            request["supersample"] = int(supersample)
        if walkers:
            request["walkers"] = int(walkers)
        if exact:
            request["exact"] = True
        if accumulate:
            request["accumulate"] = accumulate
        out, info = self._call(request)
        return Image(self, out, info, text)
