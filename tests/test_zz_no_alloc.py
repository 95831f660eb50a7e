"""Density estimation with its weight table in a static device array
(ffb_density_estimate_static), against the allocating entry point
(ffb_density_estimate) on the same histogram.

Collected last on purpose: it must pass after every other test has run in
the process as well as alone in a fresh one.
"""

import ctypes

import numpy as np
import pytest

from ffb200 import _native, synthetic


def _call(d_hist, w, h, max_radius, min_radius, curve, d_out, stream):
    L = _native.lib()
    return L.ffb_density_estimate_static(ctypes.c_void_p(d_hist), ctypes.c_uint32(w), ctypes.c_uint32(h),
                                         ctypes.c_float(max_radius), ctypes.c_float(min_radius), ctypes.c_float(curve),
                                         ctypes.c_void_p(d_out), ctypes.c_void_p(stream))


def test_table_beyond_the_static_array_is_refused():
    """curve 0.1 at radius 9 needs ~9^10 table entries: refused before any
    device work (so this runs without a GPU), with the limit in the message."""
    L = _native.lib()
    rc = _call(16, 8, 8, 9.0, 0.0, 0.1, 16, 0)
    assert rc == _native.ERR_TOO_LARGE
    assert b"65536" in L.ffb_last_error()


@pytest.mark.gpu
def test_static_scratch_matches_allocating_entry_point(renderer):
    import torch
    cfg = synthetic.plain_flame(3)
    W, H = 96, 80
    cnt, rgb, _ = renderer.histogram(cfg, W, H, iterations=150_000, seed=5)
    hist = np.empty((H, W, 4), np.float32)
    hist[..., :3] = rgb
    hist[..., 3] = cnt.view(np.float32)                   # u32 count bits, as ffb_chaos_device writes them
    dev = torch.device("cuda", 0)
    d_hist = torch.from_numpy(hist).to(dev)
    d_out = torch.empty_like(d_hist)
    stream = torch.cuda.Stream(dev)
    tables = ((9.0, 0.0, 0.4), (5.0, 0.5, 0.6))
    # The allocating entry point's answers first: it allocates, this one must not.
    refs = [renderer.density_estimate(cnt, rgb, *t) for t in tables]

    def static_call(t):
        d_out.fill_(float("nan"))
        torch.cuda.synchronize(dev)
        rc = _call(d_hist.data_ptr(), W, H, t[0], t[1], t[2], d_out.data_ptr(), stream.cuda_stream)
        assert rc == 0, _native.lib().ffb_last_error()
        stream.synchronize()
        return d_out.cpu().numpy()

    static_call(tables[1])                                # set-up: the array's address, the kernels loaded
    torch.cuda.synchronize(dev)
    free0, torch0 = torch.cuda.mem_get_info(dev)[0], torch.cuda.memory_allocated(dev)
    # Two calls in a row with different tables: the second overwrites the
    # first's entries in the shared array.
    for t, (ref_c, ref_rgb) in zip(tables, refs):
        o = static_call(t)
        gc, grgb = o[..., 3], o[..., :3]
        assert np.isfinite(o).all()
        # The DE parity tolerance: 1e-5 relative, floored at 1e-3 of the peak.
        assert np.max(np.abs(gc - ref_c) / np.maximum(np.abs(ref_c), 1e-3 * max(ref_c.max(), 1.0))) <= 1e-5
        assert np.max(np.abs(grgb - ref_rgb) / np.maximum(np.abs(ref_rgb), 1e-3 * max(ref_rgb.max(), 1.0))) <= 1e-5
    torch.cuda.synchronize(dev)
    # Nothing allocated on the device by the two calls: neither the driver's
    # free memory nor torch's allocator moved.
    assert torch.cuda.mem_get_info(dev)[0] == free0
    assert torch.cuda.memory_allocated(dev) == torch0


def test_nan_parameters_are_refused():
    """NaN fails every range comparison: it is refused with the out-of-range
    values, before any device work (so this runs without a GPU)."""
    L = _native.lib()
    nan = float("nan")
    for args in ((nan, 0.0, 0.4), (9.0, nan, 0.4), (9.0, 0.0, nan)):
        assert _call(16, 8, 8, *args, 16, 0) == _native.ERR_INVALID
        assert b"bad DE parameters" in L.ffb_last_error()
