"""ctypes binding of libffb200.so (include/ffb200.h).

The library is built in-tree by fflame-rust_b200/build.py.  Nothing here
computes anything on the CPU: every render call goes to the CUDA kernels,
and fails loudly (EngineError) when the library or a device is missing.
"""

import ctypes
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libffb200.so")

OK, ERR_INVALID, ERR_CONFIG, ERR_TOO_LARGE, ERR_OUT_OF_MEMORY, ERR_CUDA, ERR_COMPILE, ERR_CANCELLED, ERR_NO_DEVICE = range(9)
STATUS_NAMES = ["OK", "Invalid", "Config", "TooLarge", "OutOfMemory", "Cuda", "Compile", "Cancelled", "NoDevice"]
RNG = {"pcg": 0, "philox": 1}
MATH = {"precise": 0, "sfu": 1}

# Every symbol include/ffb200.h declares.
EXPORTS = [
    "fae_alloc", "fae_free", "fae_output_ptr", "fae_output_len", "fae_info_ptr", "fae_info_len", "fae_call",
    "ffb_last_error", "ffb_version", "ffb_renderer_create", "ffb_renderer_destroy", "ffb_render",
    "ffb_render_device", "ffb_histogram", "ffb_tonemap", "ffb_density_estimate", "ffb_probe",
    "ffb_apply_points", "ffb_specialize", "ffb_atomic_bench", "ffb_chaos_device", "ffb_hist_pack",
    "ffb_hist_unpack", "ffb_finish_device", "ffb_finish_band", "ffb_histogram_u64", "ffb_batch_create", "ffb_batch_run",
    "ffb_batch_output", "ffb_batch_info", "ffb_batch_destroy", "ffb_density_estimate_static",
    "ffb_diff_create", "ffb_diff_layout", "ffb_diff_theta", "ffb_diff_forward", "ffb_diff_backward", "ffb_diff_samples",
    "ffb_diff_jacobians", "ffb_diff_destroy", "ffb_diff_specialize", "ffb_encode_png",
    "ffb_flame_import", "ffb_histogram_f32", "ffb_hist_filter", "ffb_specialize_job", "ffb_struct_sizes",
    "ffb_plot_bench",
]


class EngineError(ValueError):
    """A call the engine refused or failed, with its reason (pyfae's EngineError)."""

    def __init__(self, msg, status=ERR_INVALID):
        super().__init__(msg)
        self.status = status


PROGRESS_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64)
CANCEL_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p)


class Job(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("iterations", ctypes.c_uint64),
        ("iterations_per_thread", ctypes.c_uint32), ("burn_in", ctypes.c_uint32), ("walkers", ctypes.c_uint32),
        ("supersample", ctypes.c_uint32), ("rng", ctypes.c_int32), ("math", ctypes.c_int32),
        ("transparent", ctypes.c_int32), ("threads", ctypes.c_int32), ("seed", ctypes.c_uint64),
        ("walker0", ctypes.c_uint32), ("schedule", ctypes.c_uint32), ("count_bits", ctypes.c_uint32),
        ("accumulate", ctypes.c_uint32), ("plot", ctypes.c_uint32),
        ("progress", PROGRESS_FN), ("cancelled", CANCEL_FN), ("progress_user", ctypes.c_void_p),
    ]


class Output(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("total_iterations", ctypes.c_uint64),
        ("inframe_samples", ctypes.c_uint64), ("render_time_ms", ctypes.c_double),
        ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64), ("kernel_launches", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


APPLY_WORDS = 64          # draw words a point of apply_points / diff jacobians


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built: run `python fflame-rust_b200/build.py`")
        L = ctypes.CDLL(LIB_PATH)
        L.ffb_last_error.restype = ctypes.c_char_p
        L.ffb_version.restype = ctypes.c_char_p
        L.fae_alloc.restype = ctypes.c_void_p
        L.fae_alloc.argtypes = [ctypes.c_size_t]
        L.fae_free.argtypes = [ctypes.c_void_p, ctypes.c_size_t]
        L.fae_output_ptr.restype = ctypes.c_void_p
        L.fae_info_ptr.restype = ctypes.c_void_p
        L.fae_output_len.restype = ctypes.c_size_t
        L.fae_info_len.restype = ctypes.c_size_t
        L.fae_call.restype = ctypes.c_int32
        L.fae_call.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t]
        L.ffb_renderer_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.ffb_renderer_destroy.argtypes = [ctypes.c_void_p]
        L.ffb_renderer_destroy.restype = None
        _lib = L
    return _lib


def _check(st):
    if st != OK:
        msg = lib().ffb_last_error().decode(errors="replace")
        raise EngineError(f"{STATUS_NAMES[st] if st < len(STATUS_NAMES) else st}: {msg}", st)


def _text(config):
    if isinstance(config, (bytes, bytearray)):
        return bytes(config)
    if isinstance(config, str):
        if config.lstrip().startswith("{"):
            return config.encode()
        with open(config, "rb") as f:
            return f.read()
    if hasattr(config, "data"):
        config = config.data
    return json.dumps(config).encode()


SCHEDULE = {"auto": 0, "plain": 1, "sorted": 2}


ACCUMULATE = {"auto": 0, "direct": 1, "tiled": 2}
PLOT = {"auto": 0, "inline": 1, "deferred": 2, "fused": 3}


def make_job(width=0, height=0, iterations=0, iterations_per_thread=0, burn_in=0, walkers=0, supersample=1,
             rng="philox", math="precise", transparent=0, threads=0, seed=0, walker0=0, schedule="auto", count_bits=32,
             accumulate="auto", plot="auto", progress=None, cancel=None):
    """The C job; `progress(current, total)` is called after each launch of
    the chaos game and `cancel()` returning true before one stops the render
    (RenderProgress, render.rs:293-301)."""
    j = Job()
    j.width, j.height, j.iterations = width, height, int(iterations or 0)
    j.iterations_per_thread, j.burn_in, j.walkers = iterations_per_thread, burn_in, walkers
    j.supersample = supersample
    j.rng = RNG[rng] if isinstance(rng, str) else rng
    j.math = MATH[math] if isinstance(math, str) else math
    j.transparent, j.threads, j.seed, j.walker0 = int(transparent), threads, int(seed), walker0
    j.schedule = SCHEDULE[schedule] if isinstance(schedule, str) else schedule
    j.count_bits = count_bits
    j.accumulate = ACCUMULATE[accumulate] if isinstance(accumulate, str) else accumulate
    j.plot = PLOT[plot] if isinstance(plot, str) else plot
    if progress is not None:
        j._progress_cb = PROGRESS_FN(lambda _u, cur, tot: progress(int(cur), int(tot)))
        j.progress = j._progress_cb
    if cancel is not None:
        j._cancel_cb = CANCEL_FN(lambda _u: 1 if cancel() else 0)
        j.cancelled = j._cancel_cb
    return j


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


class Renderer:
    """FlameRenderer: one CUDA device, its stream and the compiled-flame cache."""

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        _check(lib().ffb_renderer_create(device, ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().ffb_renderer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def render(self, config, width, height, **job):
        """config -> (RGBA8 [height, width, 4], Output)."""
        cfg = _text(config)
        j = make_job(width, height, **job)
        out = np.zeros((height, width, 4), np.uint8)
        o = Output()
        _check(lib().ffb_render(self._h, cfg, ctypes.c_size_t(len(cfg)), ctypes.byref(j), _p(out, ctypes.c_uint8), ctypes.byref(o)))
        return out, o

    def render_device(self, config, width, height, d_rgba, stream=None, sync=True, **job):
        """The render into device memory at `d_rgba` (an int pointer)."""
        cfg = _text(config)
        j = make_job(width, height, **job)
        o = Output()
        _check(lib().ffb_render_device(self._h, cfg, ctypes.c_size_t(len(cfg)), ctypes.byref(j), ctypes.c_void_p(d_rgba),
                                       ctypes.c_void_p(stream or 0), ctypes.c_int(1 if sync else 0), ctypes.byref(o)))
        return o

    def histogram(self, config, width, height, **job):
        """The chaos game alone: (counts u32 [H, W], rgb f32 [H, W, 3], Output) at the internal size."""
        cfg = _text(config)
        j = make_job(width, height, **job)
        ss = j.supersample or 1
        H, W = height * ss, width * ss
        cnt = np.zeros((H, W), np.uint32)
        rgb = np.zeros((H, W, 3), np.float32)
        o = Output()
        _check(lib().ffb_histogram(self._h, cfg, ctypes.c_size_t(len(cfg)), ctypes.byref(j), _p(cnt, ctypes.c_uint32),
                                   _p(rgb, ctypes.c_float), ctypes.byref(o)))
        return cnt, rgb, o

    def histogram_f32(self, config, width, height, **job):
        """config -> (counts [h, w] f32, rgb sums [h, w, 3], Output): also a filtered histogram."""
        cfg = _text(config)
        j = make_job(width, height, **job)
        ss = j.supersample or 1
        cnt = np.zeros((height * ss, width * ss), np.float32)
        rgb = np.zeros((height * ss, width * ss, 3), np.float32)
        o = Output()
        _check(lib().ffb_histogram_f32(self._h, cfg, ctypes.c_size_t(len(cfg)), ctypes.byref(j), _p(cnt, ctypes.c_float),
                                       _p(rgb, ctypes.c_float), ctypes.byref(o)))
        return cnt, rgb, o

    def hist_filter(self, counts, rgb, sigma, sigma_d):
        """The spatial filter of one batch histogram (counts u32 [h, w], rgb [h, w, 3]) -> [h, w, 4] (r, g, b, count)."""
        counts = np.ascontiguousarray(counts, np.uint32)
        rgb = np.ascontiguousarray(rgb, np.float32)
        h, w = counts.shape
        out = np.zeros((h, w, 4), np.float32)
        _check(lib().ffb_hist_filter(self._h, _p(counts, ctypes.c_uint32), _p(rgb, ctypes.c_float), ctypes.c_uint32(w),
                                     ctypes.c_uint32(h), ctypes.c_float(sigma), ctypes.c_float(sigma_d), _p(out, ctypes.c_float)))
        return out

    def histogram_u64(self, config, width, height, **job):
        """The chaos game with exact u64 counts: (counts u64 [H, W], rgb f32 [H, W, 3], Output)."""
        cfg = _text(config)
        j = make_job(width, height, **job)
        ss = j.supersample or 1
        H, W = height * ss, width * ss
        cnt = np.zeros((H, W), np.uint64)
        rgb = np.zeros((H, W, 3), np.float32)
        o = Output()
        _check(lib().ffb_histogram_u64(self._h, cfg, ctypes.c_size_t(len(cfg)), ctypes.byref(j), _p(cnt, ctypes.c_uint64),
                                       _p(rgb, ctypes.c_float), ctypes.byref(o)))
        return cnt, rgb, o

    def tonemap(self, config, counts, rgb, sample_density, ss=1, transparent=0, want_float=False):
        cfg = _text(config)
        counts = np.ascontiguousarray(counts, np.float32)
        rgb = np.ascontiguousarray(rgb, np.float32)
        h, w = counts.shape
        oh, ow = (h, w) if ss == 1 else (h // 2, w // 2)
        out = np.zeros((oh, ow, 4), np.uint8)
        f = np.zeros((h, w, 4), np.float32) if want_float else None
        _check(lib().ffb_tonemap(self._h, cfg, ctypes.c_size_t(len(cfg)), _p(counts, ctypes.c_float), _p(rgb, ctypes.c_float),
                                 ctypes.c_uint32(w), ctypes.c_uint32(h), ctypes.c_uint32(ss), ctypes.c_double(sample_density),
                                 ctypes.c_int32(transparent), _p(out, ctypes.c_uint8), _p(f, ctypes.c_float) if want_float else None))
        return (out, f) if want_float else out

    def density_estimate(self, counts, rgb, max_radius, min_radius=0.0, curve=0.4):
        counts = np.ascontiguousarray(counts, np.uint32)
        rgb = np.ascontiguousarray(rgb, np.float32)
        h, w = counts.shape
        oc = np.zeros((h, w), np.float32)
        orgb = np.zeros((h, w, 3), np.float32)
        _check(lib().ffb_density_estimate(self._h, _p(counts, ctypes.c_uint32), _p(rgb, ctypes.c_float), ctypes.c_uint32(w),
                                          ctypes.c_uint32(h), ctypes.c_float(max_radius), ctypes.c_float(min_radius),
                                          ctypes.c_float(curve), _p(oc, ctypes.c_float), _p(orgb, ctypes.c_float)))
        return oc, orgb

    def probe(self, config, pts, n_transforms, math="precise"):
        cfg = _text(config)
        pts = np.ascontiguousarray(pts, np.float32).reshape(-1, 2)
        out = np.zeros((n_transforms * len(pts), 2), np.float32)
        _check(lib().ffb_probe(self._h, cfg, ctypes.c_size_t(len(cfg)), _p(pts, ctypes.c_float), ctypes.c_uint32(len(pts)),
                               ctypes.c_int32(MATH[math] if isinstance(math, str) else math), _p(out, ctypes.c_float),
                               ctypes.c_uint32(len(out))))
        return out.reshape(n_transforms, len(pts), 2)

    def apply_points(self, config, xform, xs, ys, words, with_affine=True, math="precise"):
        cfg = _text(config)
        xs = np.ascontiguousarray(xs, np.float32)
        ys = np.ascontiguousarray(ys, np.float32)
        words = np.ascontiguousarray(words, np.float32)
        n = len(xs)
        assert words.size == n * APPLY_WORDS, "draw words: APPLY_WORDS a point"
        xo, yo = np.zeros(n, np.float32), np.zeros(n, np.float32)
        _check(lib().ffb_apply_points(self._h, cfg, ctypes.c_size_t(len(cfg)), ctypes.c_int32(xform), ctypes.c_uint32(n),
                                      _p(xs, ctypes.c_float), _p(ys, ctypes.c_float), _p(words, ctypes.c_float),
                                      ctypes.c_int32(1 if with_affine else 0), ctypes.c_int32(MATH[math] if isinstance(math, str) else math),
                                      _p(xo, ctypes.c_float), _p(yo, ctypes.c_float)))
        return xo, yo

    def chaos_device(self, config, width, height, d_hist, stream=None, **job):
        """The chaos game of the job's walker shard into a device histogram (int pointer)."""
        cfg = _text(config)
        j = make_job(width, height, **job)
        o = Output()
        _check(lib().ffb_chaos_device(self._h, cfg, ctypes.c_size_t(len(cfg)), ctypes.byref(j), ctypes.c_void_p(d_hist),
                                      ctypes.c_void_p(stream or 0), ctypes.byref(o)))
        return o

    def hist_pack(self, d_hist, pixels, d_counts, d_rgb, stream=None):
        _check(lib().ffb_hist_pack(self._h, ctypes.c_void_p(d_hist), ctypes.c_uint64(pixels), ctypes.c_void_p(d_counts),
                                   ctypes.c_void_p(d_rgb), ctypes.c_void_p(stream or 0)))

    def hist_unpack(self, d_counts, d_rgb, pixels, d_hist, stream=None):
        _check(lib().ffb_hist_unpack(self._h, ctypes.c_void_p(d_counts), ctypes.c_void_p(d_rgb), ctypes.c_uint64(pixels),
                                     ctypes.c_void_p(d_hist), ctypes.c_void_p(stream or 0)))

    def finish_device(self, config, width, height, d_hist, total_samples, row0, rows, d_rgba, stream=None, **job):
        cfg = _text(config)
        j = make_job(width, height, **job)
        _check(lib().ffb_finish_device(self._h, cfg, ctypes.c_size_t(len(cfg)), ctypes.byref(j), ctypes.c_void_p(d_hist),
                                       ctypes.c_uint64(total_samples), ctypes.c_uint32(row0), ctypes.c_uint32(rows),
                                       ctypes.c_void_p(d_rgba), ctypes.c_void_p(stream or 0)))

    def finish_band(self, config, width, height, d_hist, hist_row0, hist_rows, total_samples, row0, rows, d_rgba,
                    stream=None, **job):
        """finish_device from a window of the summed histogram: internal rows
        [hist_row0, hist_row0 + hist_rows), covering the band and the DE reach."""
        cfg = _text(config)
        j = make_job(width, height, **job)
        _check(lib().ffb_finish_band(self._h, cfg, ctypes.c_size_t(len(cfg)), ctypes.byref(j), ctypes.c_void_p(d_hist),
                                     ctypes.c_uint32(hist_row0), ctypes.c_uint32(hist_rows), ctypes.c_uint64(total_samples),
                                     ctypes.c_uint32(row0), ctypes.c_uint32(rows), ctypes.c_void_p(d_rgba),
                                     ctypes.c_void_p(stream or 0)))

    def atomic_bench(self, pixels, samples, kind=0):
        ms = ctypes.c_double()
        _check(lib().ffb_atomic_bench(self._h, ctypes.c_uint32(pixels), ctypes.c_uint64(samples), ctypes.c_int32(kind), ctypes.byref(ms)))
        return ms.value

    def plot_bench(self, config, width, height, **job):
        """The plot kernel alone (deferred plotting, each plot launch after
        its chaos launch on one stream): (plot ms, samples, in-frame splats)."""
        cfg = _text(config)
        j = make_job(width, height, **job)
        ms, n, inf = ctypes.c_double(), ctypes.c_uint64(), ctypes.c_uint64()
        _check(lib().ffb_plot_bench(self._h, cfg, ctypes.c_size_t(len(cfg)), ctypes.byref(j), ctypes.byref(ms), ctypes.byref(n),
                                    ctypes.byref(inf)))
        return ms.value, n.value, inf.value


class BatchItem(ctypes.Structure):
    _fields_ = [("config", ctypes.c_char_p), ("config_len", ctypes.c_size_t), ("width", ctypes.c_uint32),
                ("height", ctypes.c_uint32), ("iterations", ctypes.c_uint64), ("seed", ctypes.c_uint64)]


class Batch:
    """Many flames rendered by one persistent launch a structure group and
    one batched tone map, captured as a CUDA graph (ffb_batch_*).

    items: (config, width, height, samples[, seed]) tuples."""

    def __init__(self, renderer, items, tune=True, **common):
        self._r = renderer
        self._texts = [_text(it[0]) for it in items]
        arr = (BatchItem * len(items))()
        for k, (it, t) in enumerate(zip(items, self._texts)):
            arr[k].config, arr[k].config_len = t, len(t)
            arr[k].width, arr[k].height, arr[k].iterations = it[1], it[2], int(it[3])
            arr[k].seed = int(it[4]) if len(it) > 4 else 0
        self._items = arr
        self.sizes = [(it[1], it[2]) for it in items]
        j = make_job(**common)
        h = ctypes.c_void_p()
        L = lib()
        L.ffb_batch_destroy.argtypes = [ctypes.c_void_p]
        L.ffb_batch_destroy.restype = None
        _check(L.ffb_batch_create(renderer._h, arr, ctypes.c_uint32(len(items)), ctypes.byref(j), ctypes.c_int32(1 if tune else 0),
                                  ctypes.byref(h)))
        self._h = h

    def run(self, stream=None, sync=True):
        """Replay the batch; the device milliseconds when `sync`."""
        ms = ctypes.c_double()
        _check(lib().ffb_batch_run(self._h, ctypes.c_void_p(stream or 0), ctypes.c_int32(1 if sync else 0),
                                   ctypes.byref(ms) if sync else None))
        return ms.value if sync else None

    def output(self, index):
        w, h = self.sizes[index]
        out = np.zeros((h, w, 4), np.uint8)
        plotted = ctypes.c_uint64()
        _check(lib().ffb_batch_output(self._h, ctypes.c_uint32(index), _p(out, ctypes.c_uint8), ctypes.byref(plotted)))
        return out, plotted.value

    def info(self):
        t, th, it, g = ctypes.c_uint64(), ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        _check(lib().ffb_batch_info(self._h, ctypes.byref(t), ctypes.byref(th), ctypes.byref(it), ctypes.byref(g)))
        return {"samples": t.value, "threads": th.value, "iterations_per_walker": it.value, "groups": g.value}

    def close(self):
        if getattr(self, "_h", None):
            lib().ffb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def walkers_for(samples, threads, iters):
        """The walkers and per-walker iterations a batch gives a flame of `samples`."""
        w = max(-(-samples // iters), threads)
        w = -(-w // threads) * threads
        return w, -(-samples // w)


def specialize(config, rng="philox", math="precise"):
    """NVRTC-compile a config's chaos kernel for sm_100a (no device needed): (cubin bytes, source)."""
    cfg = _text(config)
    n = ctypes.c_size_t()
    buf = ctypes.create_string_buffer(1 << 20)
    _check(lib().ffb_specialize(cfg, ctypes.c_size_t(len(cfg)), ctypes.c_int32(RNG[rng]), ctypes.c_int32(MATH[math]),
                                ctypes.byref(n), buf, ctypes.c_size_t(len(buf))))
    return n.value, buf.value.decode()


def specialize_job(config, **job):
    """NVRTC-compile the module a render of `job` would use (no device needed): (cubin bytes, source)."""
    cfg = _text(config)
    j = make_job(**job)
    n = ctypes.c_size_t()
    buf = ctypes.create_string_buffer(1 << 21)
    _check(lib().ffb_specialize_job(cfg, ctypes.c_size_t(len(cfg)), ctypes.byref(j), ctypes.byref(n), buf,
                                    ctypes.c_size_t(len(buf))))
    return n.value, buf.value.decode()


def density_estimate_static(d_hist, width, height, max_radius, min_radius=0.0, curve=0.4, d_out=0, stream=None):
    """Density estimation of a device histogram (int pointer to width*height
    float4) into `d_out` (the same layout, counts as f32) that allocates
    nothing: the weight table lives in a fixed device array shared by every
    call on the device (ffb_density_estimate_static).  Queued on `stream`."""
    _check(lib().ffb_density_estimate_static(ctypes.c_void_p(d_hist), ctypes.c_uint32(width), ctypes.c_uint32(height),
                                             ctypes.c_float(max_radius), ctypes.c_float(min_radius), ctypes.c_float(curve),
                                             ctypes.c_void_p(d_out), ctypes.c_void_p(stream or 0)))


def encode_png(config, rgba, width, height, iterations=0, ms=0.0, iterations_per_thread=1024):
    """A frame (RGBA8 bytes or array) as the PNG the reference's CLI writes,
    the config and the render's numbers in its tEXt chunks (no GPU needed)."""
    cfg = _text(config)
    data = bytes(rgba) if not isinstance(rgba, np.ndarray) else np.ascontiguousarray(rgba, np.uint8).tobytes()
    if len(data) != width * height * 4:
        raise EngineError(f"{len(data)} bytes are not {width}x{height} RGBA")
    out, n = ctypes.POINTER(ctypes.c_uint8)(), ctypes.c_size_t()
    _check(lib().ffb_encode_png(cfg, ctypes.c_size_t(len(cfg)), data, ctypes.c_uint32(width), ctypes.c_uint32(height),
                                ctypes.c_uint64(int(iterations)), ctypes.c_double(ms), ctypes.c_uint32(iterations_per_thread),
                                ctypes.byref(out), ctypes.byref(n)))
    return ctypes.string_at(out, n.value)


def flame_import(xml):
    """Apophysis / JWildfire `.flame` XML (text or bytes) -> a list of config
    dicts, one a flame (2-D; a 3-D camera is refused with the reason)."""
    data = xml.encode() if isinstance(xml, str) else bytes(xml)
    out, n = ctypes.c_char_p(), ctypes.c_size_t()
    _check(lib().ffb_flame_import(data, ctypes.c_size_t(len(data)), ctypes.byref(out), ctypes.byref(n)))
    return json.loads(ctypes.string_at(out, n.value).decode())
