"""The differentiable render behind a torch.autograd.Function.

An addition beside the reference's render, which has no gradients.  The
forward pass is the chaos game with a bilinear splat and a linearly
interpolated palette, followed by the log tone map in linear light (alpha 1).
The backward pass is the adjoint kernel: every plotted sample is
differentiated through the last `window` iterations of its walker (16 by
default), recomputed from walker states checkpointed every `checkpoint`
iterations (64) instead of stored trajectories.  Gradients are taken with
respect to

    theta = [n_xf*6 affine a, b, c, d, e, f | n_xf*n_var variation weights,
             transform-major | n_xf colours]

with the transform choices (the Philox stream) held fixed, so two renders at
nearby theta share their random numbers (common random numbers).  With
`exact=True` the histogram is summed in integers (u64 fixed point), so a
render is the same bits whatever the order of the GPU's atomics.

    dr = DiffRenderer(config, 512, 512, samples=200_000_000)
    theta = dr.theta0().requires_grad_()
    img = dr.render(theta)                 # [512, 512, 4] float32, CUDA
    loss = ((img - target) ** 2).sum()
    loss.backward()                        # theta.grad via the adjoint kernel

Everything runs on the GPU through libffb200.so; without a device the
constructor raises EngineError.
"""

import ctypes

import torch

from ._native import EngineError, Renderer, _check, _text, lib, make_job  # noqa: F401


class DiffRenderer:
    """One flame set up for differentiable renders at width x height."""

    def __init__(self, config, width, height, samples, *, walkers=65536, window=16, checkpoint=64, seed=0,
                 burn_in=20, threads=128, exact=False, renderer=None, device=0):
        self.renderer = renderer or Renderer(device)
        self.width, self.height = width, height
        self.device = torch.device("cuda", device)
        cfg = _text(config)
        j = make_job(width, height, iterations=samples, walkers=walkers, seed=seed, burn_in=burn_in, threads=threads,
                     count_bits=64 if exact else 32)
        h = ctypes.c_void_p()
        _check(lib().ffb_diff_create(self.renderer._h, cfg, ctypes.c_size_t(len(cfg)), ctypes.byref(j),
                                     ctypes.c_uint32(window), ctypes.c_uint32(checkpoint), ctypes.byref(h)))
        self._h = h
        nx, nv, nw, it = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        names = ctypes.create_string_buffer(4096)
        _check(lib().ffb_diff_layout(h, ctypes.byref(nx), ctypes.byref(nv), ctypes.byref(nw), ctypes.byref(it), names,
                                     ctypes.c_size_t(len(names))))
        self.n_xforms, self.walkers, self.iterations = nx.value, nw.value, it.value
        self.variations = [n for n in names.value.decode().split(",") if n]
        self.n_params = self.n_xforms * (7 + len(self.variations))
        self.window, self.checkpoint = window, checkpoint
        self._serial = 0

    def close(self):
        if getattr(self, "_h", None):
            lib().ffb_diff_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def layout(self):
        """Slices of theta: affine [n_xf, 6], weights [n_xf, n_var], colours [n_xf]."""
        n, v = self.n_xforms, len(self.variations)
        return {"affine": slice(0, n * 6), "weights": slice(n * 6, n * (6 + v)), "colours": slice(n * (6 + v), n * (7 + v))}

    def theta0(self):
        """The config's own theta on the device (float32)."""
        t = torch.empty(self.n_params, dtype=torch.float32)
        _check(lib().ffb_diff_theta(self._h, ctypes.c_void_p(t.data_ptr())))
        return t.to(self.device)

    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def forward_raw(self, theta, hist=False):
        """Image [h, w, 4] (and the histogram [h, w, 4]: r, g, b sums, weight) at theta."""
        theta = theta.detach().to(self.device, torch.float32).contiguous()
        img = torch.empty(self.height, self.width, 4, dtype=torch.float32, device=self.device)
        hb = torch.empty_like(img) if hist else None
        self._serial += 1
        _check(lib().ffb_diff_forward(self._h, ctypes.c_void_p(theta.data_ptr()), ctypes.c_void_p(img.data_ptr()),
                                      ctypes.c_void_p(hb.data_ptr()) if hist else None, self._stream()))
        return (img, hb) if hist else img

    def backward_raw(self, grad_image, grad_hist=False):
        """dL/dtheta (float64) of the most recent forward, given dL/dimage
        (and dL/dhistogram [h, w, 4] with `grad_hist`)."""
        g = grad_image.detach().to(self.device, torch.float32).contiguous()
        out = torch.empty(self.n_params, dtype=torch.float64, device=self.device)
        gh = torch.empty(self.height, self.width, 4, dtype=torch.float32, device=self.device) if grad_hist else None
        _check(lib().ffb_diff_backward(self._h, ctypes.c_void_p(g.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                       ctypes.c_void_p(gh.data_ptr()) if grad_hist else None, self._stream()))
        return (out, gh) if grad_hist else out

    def samples(self):
        """(plotted, in-frame) samples of the most recent forward."""
        p, i = ctypes.c_uint64(), ctypes.c_uint64()
        _check(lib().ffb_diff_samples(self._h, ctypes.byref(p), ctypes.byref(i), self._stream()))
        return p.value, i.value

    def jacobians(self, xform, xs, ys, words):
        """Each variation's (vx, vy, J) at points (host arrays): [n, n_var, 6]."""
        import numpy as np
        xs = np.ascontiguousarray(xs, np.float32)
        ys = np.ascontiguousarray(ys, np.float32)
        words = np.ascontiguousarray(words, np.float32)
        assert words.size == len(xs) * 64, "draw words: 64 a point"
        out = np.zeros((len(xs), len(self.variations), 6), np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        _check(lib().ffb_diff_jacobians(self._h, ctypes.c_int32(xform), ctypes.c_uint32(len(xs)), xs.ctypes.data_as(fp),
                                        ys.ctypes.data_as(fp), words.ctypes.data_as(fp), out.ctypes.data_as(fp)))
        return out

    def render(self, theta):
        """The image at theta, differentiable with respect to theta."""
        return _Render.apply(theta, self)


class _Render(torch.autograd.Function):
    # The adjoint reads the histogram and checkpoints of the renderer's most
    # recent forward; a backward whose forward has since been replaced runs
    # that forward again first (the renders are deterministic apart from the
    # order of floating-point atomics).
    @staticmethod
    def forward(ctx, theta, dr):
        ctx.dr = dr
        ctx.dtype = theta.dtype
        ctx.save_for_backward(theta)
        img = dr.forward_raw(theta)
        ctx.serial = dr._serial
        return img

    @staticmethod
    def backward(ctx, grad_image):
        dr = ctx.dr
        if dr._serial != ctx.serial:
            (theta,) = ctx.saved_tensors
            dr.forward_raw(theta)
            ctx.serial = dr._serial
        g = dr.backward_raw(grad_image)
        return g.to(ctx.dtype), None


def render(dr, theta):
    """Functional form of DiffRenderer.render."""
    return dr.render(theta)
