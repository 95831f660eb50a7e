"""The differentiable render: the adjoint kernel against the FP64 oracle and
against central finite differences with common random numbers.

Tolerances:
* variation Jacobians: 2e-4 of max(|J|, 1) against the oracle's central
  differences in double;
* bilinear histogram of a linear-only flame (identical orbits): 1e-5
  relative (FP32 sums against double);
* tone map: 1e-4 relative of the FP64 oracle; its vector-Jacobian product:
  1e-3 of the pixel's largest component against central differences;
* gradient: 1e-3 relative (vector norm, and per parameter class) of the
  FP64 oracle's, same samples, also at the 512^2 size; the oracle's within
  1e-3 of central finite differences in FP64 for every class; at the
  512^2, 2e8-sample configuration on the GPU, per class 3e-3 (affine),
  5e-3 (weights), 8e-3 (colours) and 1e-3 along the gradient against
  central differences of deterministic FP32 renders.
"""

import ctypes
import json

import numpy as np
import pytest

from ffb200 import synthetic


def smooth_palette(cfg):
    cfg["palette"] = {"name": "ramp", "indexed_colors": ",".join("%02X%02X80" % (i, 255 - i) for i in range(256))}
    return cfg


def oracle_loss_grad(oracle, cfg, W, theta, walkers, iters, seed, target, window, f64=True):
    c = oracle.with_theta(cfg, theta)
    fl = oracle.DiffFlame(c, W, W)
    hist, n = fl.render(walkers, iters, seed=seed, f64=f64, threads=16)
    tm = oracle.tonemap_params_for(c, W, W, max(n / (W * W), 1e-6))
    img = oracle.diff_tonemap(tm, hist)
    loss = ((img[..., :3] - target[..., :3]) ** 2).sum()
    dimg = np.zeros_like(img)
    dimg[..., :3] = 2 * (img[..., :3] - target[..., :3])
    dh = oracle.diff_tonemap_vjp(tm, hist, dimg)
    return loss, img, fl.grad(dh, walkers, iters, seed=seed, window=window, f64=f64, threads=16)


def test_oracle_gradient_matches_finite_differences(oracle):
    """The oracle's adjoint (per-sample walk-back, FD Jacobians) against
    central differences of the whole render in double, common random
    numbers.  The loss is piecewise smooth (bilinear weights), so the
    difference quotient needs a small step; the 16-iteration window agrees
    with the untruncated gradient on this contractive flame."""
    cfg = smooth_palette(synthetic.diff_flame(1))
    W, walkers, iters, seed = 48, 128, 500, 99
    th = oracle.theta_of(cfg).astype(np.float64)
    _, img0, _ = oracle_loss_grad(oracle, cfg, W, th, walkers, iters, seed, np.zeros((W, W, 4)), 16)
    target = img0 + np.random.default_rng(0).normal(0, 0.05, img0.shape)
    _, _, g16 = oracle_loss_grad(oracle, cfg, W, th, walkers, iters, seed, target, 16)
    _, _, gall = oracle_loss_grad(oracle, cfg, W, th, walkers, iters, seed, target, 0)
    assert np.linalg.norm(g16 - gall) <= 1e-3 * np.linalg.norm(gall)
    fd = np.zeros_like(g16)
    for i in range(len(th)):
        # The flame's coefficients are f32: step to f32 neighbours and divide
        # by the step actually taken.
        tp, tm = th.copy(), th.copy()
        tp[i] = np.float32(th[i] + 1e-6)
        tm[i] = np.float32(th[i] - 1e-6)
        lp = oracle_loss_grad(oracle, cfg, W, tp, walkers, iters, seed, target, 16)[0]
        lm = oracle_loss_grad(oracle, cfg, W, tm, walkers, iters, seed, target, 16)[0]
        fd[i] = (lp - lm) / (tp[i] - tm[i])
    assert np.linalg.norm(gall - fd) <= 1e-3 * np.linalg.norm(fd), (np.linalg.norm(gall - fd) / np.linalg.norm(fd), gall, fd)
    # Every parameter class on its own, the 16-iteration gradient (the
    # render's definition) included: affine coefficients, variation weights,
    # colours, each within 1e-3 of the class's finite differences.
    n = len(cfg["flame"]["transforms"])
    v = len(th) // n - 7
    for name, sl in (("affine", slice(0, n * 6)), ("weights", slice(n * 6, n * (6 + v))), ("colours", slice(n * (6 + v), None))):
        for g in (g16, gall):
            rel = np.linalg.norm(g[sl] - fd[sl]) / np.linalg.norm(fd[sl])
            assert rel <= 1e-3, (name, rel)


def test_diff_module_compiles_for_every_variation(native):
    cfg = {"flame": {"transforms": [{"a": 0.5, "b": 0, "c": 0, "d": 0.5, "e": 0, "f": 0, "weight": 1.0, "color": 0.3,
                                     "variations": {n: 0.1 for n in synthetic.TWELVE}}]}}
    c = json.dumps(cfg).encode()
    n = ctypes.c_size_t()
    buf = ctypes.create_string_buffer(1 << 21)
    L = native.lib()
    assert L.ffb_diff_specialize(c, ctypes.c_size_t(len(c)), 16, 64, ctypes.byref(n), buf, ctypes.c_size_t(len(buf))) == 0, \
        L.ffb_last_error()
    src = buf.value.decode()
    assert n.value > 0 and "ffb_diff_adjoint" in src and "dj_julia" in src


# ------------------------------------------------------------------ GPU --

@pytest.fixture(scope="module")
def diff(renderer):
    from ffb200 import diff
    return diff


def make(diff, renderer, cfg, W, samples, walkers, seed, **kw):
    return diff.DiffRenderer(cfg, W, W, samples, walkers=walkers, seed=seed, renderer=renderer, **kw)


@pytest.mark.gpu
def test_variation_jacobians_against_central_differences(diff, renderer, oracle):
    cfg = {"flame": {"transforms": [{"a": 0.5, "b": 0, "c": 0, "d": 0.5, "e": 0, "f": 0, "weight": 1.0, "color": 0.3,
                                     "variations": {n: 0.1 for n in synthetic.TWELVE}}]}, "deterministic_rng": True}
    dr = make(diff, renderer, cfg, 32, 32 * 64, 32, 5)
    rng = np.random.default_rng(3)
    n = 512
    xs = rng.uniform(0.25, 1.5, n) * rng.choice([-1, 1], n)
    ys = rng.uniform(0.25, 1.5, n) * rng.choice([-1, 1], n)
    xs = np.where(np.abs(1 + xs) < 0.3, xs + 0.6, xs).astype(np.float32)    # away from curl's pole at x = -1
    ys = ys.astype(np.float32)
    words = rng.uniform(0, 1, (n, 64)).astype(np.float32)
    out = dr.jacobians(0, xs, ys, words)
    slots = {"julia": 2}
    for j, name in enumerate(dr.variations):
        draws = words[:, slots[name]] if name in slots else None
        ref = oracle.variation_jacobian(name, xs, ys, draws=draws)
        got = out[:, j, :].astype(np.float64)
        scale = np.maximum(np.abs(ref[:, 2:]).max(axis=1, keepdims=True), 1.0)
        err = np.abs(got[:, 2:] - ref[:, 2:]) / scale
        assert err.max() <= 2e-4, (name, err.max(), np.argmax(err.max(axis=1)))
        vs = np.maximum(np.abs(ref[:, :2]), 1.0)
        assert (np.abs(got[:, :2] - ref[:, :2]) / vs).max() <= 1e-5, name
    dr.close()


@pytest.mark.gpu
def test_forward_histogram_matches_oracle_linear(diff, renderer, oracle):
    """A linear-only flame walks identical orbits on both sides: the bilinear
    histogram agrees to FP32 summation error."""
    import torch
    cfg = synthetic.diff_flame(2)
    for t in cfg["flame"]["transforms"]:
        t["variations"] = {"linear": 1.0}
    W, walkers, per = 96, 2048, 300
    dr = make(diff, renderer, cfg, W, walkers * per, walkers, 41)
    img, hist = dr.forward_raw(dr.theta0(), hist=True)
    torch.cuda.synchronize()
    plotted, inframe = dr.samples()
    fl = oracle.DiffFlame(cfg, W, W)
    oh, n = fl.render(walkers, dr.iterations, seed=41, threads=16)
    assert plotted == n == walkers * per
    g = hist.cpu().numpy().astype(np.float64)
    scale = max(oh[..., 3].max(), 1.0)
    assert np.abs(g - oh).max() <= 1e-5 * scale + 1e-4
    assert abs(g[..., 3].sum() - oh[..., 3].sum()) <= 1e-5 * oh[..., 3].sum()
    dr.close()


@pytest.mark.gpu
def test_tonemap_and_its_vjp_match_oracle(diff, renderer, oracle):
    import torch
    cfg = synthetic.diff_flame(3)
    W, walkers, per = 128, 4096, 200
    dr = make(diff, renderer, cfg, W, walkers * per, walkers, 7)
    img, hist = dr.forward_raw(dr.theta0(), hist=True)
    plotted, _ = dr.samples()
    h = hist.cpu().numpy().astype(np.float64)
    tm = oracle.tonemap_params_for(cfg, W, W, max(plotted / (W * W), 1e-6))
    ref = oracle.diff_tonemap(tm, h)
    got = img.cpu().numpy().astype(np.float64)
    assert np.abs(got[..., :3] - ref[..., :3]).max() <= 1e-4 * max(ref[..., :3].max(), 1e-3) + 1e-7
    assert np.all(got[..., 3] == 1.0)
    # The vector-Jacobian product (the adjoint's first stage) on a random cotangent.
    rng = np.random.default_rng(5)
    dimg = rng.normal(0, 1, got.shape).astype(np.float32)
    dimg[..., 3] = 0
    dh_ref = oracle.diff_tonemap_vjp(tm, h, dimg.astype(np.float64))
    _, dh = dr.backward_raw(torch.from_numpy(dimg).cuda(), grad_hist=True)
    dh_gpu = dh.cpu().numpy().astype(np.float64)
    mask = h[..., 3] >= 1e-2
    scale = np.maximum(np.abs(dh_ref).max(axis=-1), 1e-6)
    err = (np.abs(dh_gpu - dh_ref).max(axis=-1) / scale)[mask]
    assert np.quantile(err, 0.999) <= 1e-3 and np.median(err) <= 1e-5, (np.quantile(err, 0.999), err.max())
    dr.close()


def gpu_loss_grad(dr, theta, target):
    import torch
    img = dr.forward_raw(theta)
    t = torch.from_numpy(target.astype(np.float32)).cuda()
    d = torch.zeros_like(img)
    d[..., :3] = 2 * (img[..., :3] - t[..., :3])
    g = dr.backward_raw(d)
    loss = ((img[..., :3].double() - t[..., :3].double()) ** 2).sum()
    return loss.item(), img.cpu().numpy(), g.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("linear_only", [True, False])
def test_gradient_matches_fp64_oracle(diff, renderer, oracle, linear_only):
    """Same flame, theta, seed and samples: the adjoint kernel's gradient
    against the oracle's FP64 per-sample walk-back (FP32 orbits, so the
    samples coincide: exactly for a linear-only flame, to a few ulp for the
    contractive three-variation one)."""
    cfg = smooth_palette(synthetic.diff_flame(5))
    if linear_only:
        for t in cfg["flame"]["transforms"]:
            t["variations"] = {"linear": 1.0}
    W, walkers, per, seed = 64, 1024, 300, 123
    dr = make(diff, renderer, cfg, W, walkers * per, walkers, seed)
    th = dr.theta0()
    assert np.array_equal(th.cpu().numpy(), oracle.theta_of(cfg))
    img0 = dr.forward_raw(th).cpu().numpy()
    target = img0 + np.random.default_rng(1).normal(0, 0.05, img0.shape)
    _, _, g = gpu_loss_grad(dr, th, target)
    _, _, go = oracle_loss_grad(oracle, cfg, W, th.cpu().numpy().astype(np.float64), walkers, dr.iterations, seed, target, 16,
                                f64=False)
    rel = np.linalg.norm(g - go) / np.linalg.norm(go)
    assert rel <= 1e-3, (rel, g, go)
    for name, sl in dr.layout().items():
        rel = np.linalg.norm(g[sl] - go[sl]) / np.linalg.norm(go[sl])
        assert rel <= 1e-3, (name, rel)
    dr.close()


@pytest.mark.gpu
def test_gradient_matches_fp64_oracle_c4_size(diff, renderer, oracle):
    """The C4 flame at its 512^2 size and 65,536 walkers (2e7 samples, the
    oracle's share of a test's time): the adjoint kernel's gradient against
    the oracle's per-sample FP64 walk-back on the same FP32 orbits, every
    parameter class within 1e-3 -- in FP32 and with the deterministic
    fixed-point histogram."""
    import torch
    cfg = synthetic.diff_flame(4)
    W, walkers, per, seed = 512, 65536, 300, 2024
    for exact in (False, True):
        dr = make(diff, renderer, cfg, W, walkers * per, walkers, seed, exact=exact)
        th = dr.theta0()
        noisy = th + torch.from_numpy(np.random.default_rng(2).normal(0, 0.05, th.numel()).astype(np.float32)).cuda()
        target = dr.forward_raw(noisy).cpu().numpy().astype(np.float64)
        _, _, g = gpu_loss_grad(dr, th, target)
        _, _, go = oracle_loss_grad(oracle, cfg, W, th.cpu().numpy().astype(np.float64), walkers, dr.iterations, seed, target,
                                    16, f64=False)
        for name, sl in dr.layout().items():
            rel = np.linalg.norm(g[sl] - go[sl]) / np.linalg.norm(go[sl])
            assert rel <= 1e-3, (exact, name, rel)
        dr.close()


@pytest.mark.gpu
def test_gradient_matches_finite_differences_c4(diff, renderer, oracle):
    """The differentiable configuration: 4 transforms at 512^2, 2e8 samples,
    loss = L2 between the image and the image at theta + N(0, 0.05).
    Central differences with common random numbers (the same Philox stream
    at theta +- eps) on renders summed in integers (the same bits whatever
    the atomics' order), the loss evaluated in FP64 on the host.  What is
    left is the FP32 rounding in the difference quotient: at eps = 2e-6 it
    bounds the agreement of each parameter class to a few 1e-3 (bounds
    below), while the directional derivative along the gradient (the whole
    gradient's signal against one quotient's noise) is held to 1e-3.  The
    gradient itself agrees with the FP64 oracle's to 1e-4 on every class
    at this size (test_gradient_matches_fp64_oracle_c4_size), and in FP64
    orbits with finite differences to 1e-3 on every class
    (test_oracle_gradient_matches_finite_differences)."""
    import torch
    cfg = synthetic.diff_flame(4)
    W, samples, seed = 512, 200_000_000, 2024
    dr = make(diff, renderer, cfg, W, samples, 65536, seed)
    dx = make(diff, renderer, cfg, W, samples, 65536, seed, exact=True)
    th = dr.theta0()
    noisy = th + torch.from_numpy(np.random.default_rng(2).normal(0, 0.05, th.numel()).astype(np.float32)).cuda()
    target = dr.forward_raw(noisy).cpu().numpy().astype(np.float64)
    _, _, g = gpu_loss_grad(dr, th, target)

    def loss64(theta):
        _, h = dx.forward_raw(theta, hist=True)
        p, _ = dx.samples()
        c = oracle.with_theta(cfg, theta.cpu().numpy().astype(np.float64))
        tm = oracle.tonemap_params_for(c, W, W, max(p / (W * W), 1e-6))
        im = oracle.diff_tonemap(tm, h.cpu().numpy().astype(np.float64))
        return ((im[..., :3] - target[..., :3]) ** 2).sum()

    fd = np.zeros(th.numel())
    for i in range(th.numel()):
        tp, tm = th.clone(), th.clone()
        tp[i] += 2e-6
        tm[i] -= 2e-6
        fd[i] = (loss64(tp) - loss64(tm)) / float(tp[i] - tm[i])
    # Each class against its difference quotients.  The quotients' own
    # noise sets the bounds: FP32 orbits (affine, weights) and FP32 colour
    # indices round differently at theta +- eps, so a quotient at 2e-6 is
    # good to a few 1e-3 (measured on this configuration: 1.6e-3 affine,
    # 2.6e-3 weights, 4.8e-3 colours; larger steps are worse, the bilinear
    # splat and the linearly interpolated palette being piecewise linear).
    bounds = {"affine": 3e-3, "weights": 5e-3, "colours": 8e-3}
    for name, sl in dr.layout().items():
        rel = np.linalg.norm(g[sl] - fd[sl]) / np.linalg.norm(fd[sl])
        assert rel <= bounds[name], (name, rel, g[sl], fd[sl])
    # Along the gradient: the loss difference against g . (theta+ - theta-),
    # the step actually taken in f32.
    v = torch.from_numpy((g / np.linalg.norm(g)).astype(np.float32)).cuda()
    tp, tm = th + 4e-6 * v, th - 4e-6 * v
    step = (tp.double() - tm.double()).cpu().numpy()
    dl = loss64(tp) - loss64(tm)
    pred = float(np.dot(g, step))
    assert abs(dl - pred) <= 1e-3 * abs(pred), (dl, pred)
    dr.close()
    dx.close()


@pytest.mark.gpu
def test_autograd_function(diff, renderer):
    import torch
    cfg = synthetic.diff_flame(6)
    dr = make(diff, renderer, cfg, 64, 1024 * 200, 1024, 9)
    theta = dr.theta0().requires_grad_()
    img = dr.render(theta)
    target = img.detach() * 0.9
    loss = ((img - target) ** 2).sum()
    loss.backward()
    g_ref = dr.backward_raw(2 * (img.detach() - target))
    assert theta.grad is not None and theta.grad.dtype == torch.float32
    assert torch.allclose(theta.grad.double(), g_ref, rtol=1e-5, atol=1e-8 * g_ref.abs().max().item())
    # A backward after another forward re-runs its own forward first.
    img2 = dr.render(theta.detach() * 1.01)
    theta.grad = None
    img = dr.render(theta)
    _ = dr.forward_raw(theta.detach() * 0.99)
    ((img - target) ** 2).sum().backward()
    assert torch.allclose(theta.grad.double(), g_ref, rtol=1e-4, atol=1e-6 * g_ref.abs().max().item())
    del img2
    dr.close()


@pytest.mark.gpu
def test_refusals(diff, renderer):
    from ffb200 import EngineError
    cfg = synthetic.full_flame(7)                         # has a final transform and DE
    with pytest.raises(EngineError):
        make(diff, renderer, cfg, 64, 1000, 32, 1)
    cfg = synthetic.diff_flame(1)
    cfg["highlight_mode"] = "filmic"
    with pytest.raises(EngineError):
        make(diff, renderer, cfg, 64, 1000, 32, 1)
    with pytest.raises(EngineError):
        make(diff, renderer, synthetic.diff_flame(1), 64, 1000, 32, 1, window=64)
