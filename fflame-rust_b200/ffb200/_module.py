"""The engine module over the C ABI: pyfae's `Module` with libffb200.so in
place of the WASI module (python/pyfae/_module.py:33-62 of the reference).

One call crosses into it: `fae_call`, a JSON request and a block of bytes
beside it; back come a status, an output of bytes and a JSON note.
"""

import ctypes
import json

from . import _native
from ._native import EngineError


def find_module(path=None):
    """The library's file (pyfae's find_module, python/pyfae/_module.py:21-38)."""
    import os
    for c in (path, os.environ.get("FFB200_LIB"), _native.LIB_PATH):
        if c and os.path.exists(c):
            return os.path.abspath(c)
    raise FileNotFoundError("no engine library: run `python fflame-rust_b200/build.py`")


class Module:
    def __init__(self, path=None):
        find_module(path)
        self.lib = _native.lib()

    def _put(self, data):
        if not data:
            return None
        ptr = self.lib.fae_alloc(len(data))
        ctypes.memmove(ptr, data, len(data))
        return ptr

    def _get(self, ptr_fn, len_fn):
        n = len_fn()
        if not n:
            return b""
        return ctypes.string_at(ptr_fn(), n)

    def call(self, request, data=b""):
        """One call: `(output bytes, note)`, or EngineError."""
        req = json.dumps(request).encode()
        rp, dp = self._put(req), self._put(data)
        try:
            status = self.lib.fae_call(rp, len(req), dp, len(data))
        finally:
            self.lib.fae_free(rp, len(req))
            if dp:
                self.lib.fae_free(dp, len(data))
        out = self._get(self.lib.fae_output_ptr, self.lib.fae_output_len)
        if status != 0:
            raise EngineError(out.decode(errors="replace"))
        info = self._get(self.lib.fae_info_ptr, self.lib.fae_info_len)
        return out, (json.loads(info) if info else None)
