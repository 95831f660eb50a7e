"""Monte-Carlo parity of a CUDA render with the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Imported by tests/ and by bench.py's `parity` leg (run outside the timed
region), as the checker; the product never imports it.

A flame with transcendental arithmetic walks different orbits on the GPU
(CUDA's libm) and on the oracle (glibc's) after a few dozen steps, so two
renders of it agree only statistically.  The yardstick is the oracle
against itself: two oracle renders with independent seeds at the same
samples a pixel differ by Monte-Carlo noise alone, and the GPU render must
differ from one of them by no more than that (x 1.25, plus a small floor).
Three measures, each GPU-vs-oracle beside oracle-vs-oracle:

* normalised log-density: |log1p(a) - log1p(b)| over the pixels lit in
  either, its mean (L1) and 99th percentile;
* 16x16-block densities: the number of blocks whose difference exceeds 5
  standard errors (sqrt of the two blocks' summed counts);
* the tone-mapped image after density estimation: the mean absolute
  difference of the RGBA8 pixels (the oracle's histogram through its FP64
  density estimate, tone map and firefly downsample).

The three renders use three different seeds, so no pair shares its early
orbits.
"""

import numpy as np

from . import oracle as O


def log_density_l1(a, b):
    """(mean, 99th percentile) of |log1p(a) - log1p(b)| over pixels lit in either."""
    la, lb = np.log1p(np.asarray(a, np.float64)), np.log1p(np.asarray(b, np.float64))
    lit = (np.asarray(a) > 0) | (np.asarray(b) > 0)
    d = np.abs(la - lb)[lit]
    if d.size == 0:
        return 0.0, 0.0
    return float(d.mean()), float(np.percentile(d, 99))


def block_outliers(a, b, block=16):
    """Blocks of `block` x `block` pixels whose count sums differ by more than 5 standard errors."""
    h, w = a.shape
    hb, wb = h // block, w // block
    sa = np.asarray(a, np.float64)[:hb * block, :wb * block].reshape(hb, block, wb, block).sum(axis=(1, 3))
    sb = np.asarray(b, np.float64)[:hb * block, :wb * block].reshape(hb, block, wb, block).sum(axis=(1, 3))
    se = np.sqrt(np.maximum(sa + sb, 1.0))
    return int((np.abs(sa - sb) / se > 5).sum())


def oracle_image(cfg, cnt, rgb, plotted, ss):
    """The oracle's RGBA8 image of a histogram: FP64 density estimation (the
    config's radius x supersample), tone map, and the 2x2 firefly box at ss 2."""
    h, w = cnt.shape
    de = cfg.get("density_estimation")
    c, col = cnt.astype(np.float64), rgb.astype(np.float64)
    if de and de.get("radius", 0) > 0:
        c, col = O.density_estimate(c, col, w, h, de["radius"] * ss, de.get("minimum", 0.0) * ss, de.get("curve", 0.4))
    sd = plotted / float(w * h)
    _, u8 = O.tonemap(O.tonemap_params_for(cfg, w, h, sd), c, col)
    u8 = u8.reshape(h, w, 4)
    return O.downsample_firefly(u8, w // 2, h // 2) if ss == 2 else u8


def render_parity(renderer, cfg, width, height, ss, samples, walkers, seeds=(3003, 1001, 2002), threads=None, **job):
    """The GPU render (histogram and image, through the library with `job`)
    against two oracle replicates at the same samples a pixel.  Returns the
    measures (GPU vs oracle 1, oracle 2 vs oracle 1) and the render's facts."""
    import os
    threads = threads or max(1, min(len(os.sched_getaffinity(0)), 64))
    W, H = width * ss, height * ss
    per = -(-samples // walkers)
    gjob = dict(iterations=walkers * per, walkers=walkers, supersample=ss, seed=seeds[0], **job)
    cnt, _, out = renderer.histogram(cfg, width, height, **gjob)
    img, oimg = renderer.render(cfg, width, height, **gjob)
    fl = O.Flame(cfg, W, H)
    reps = []
    for s in seeds[1:]:
        plotted, inframe, c, rgb = fl.render(walkers, per + 20, seed=s, threads=threads)
        reps.append((plotted, inframe, c, rgb))
    (p1, i1, c1, r1), (p2, i2, c2, r2) = reps
    l1_go, p99_go = log_density_l1(cnt, c1)
    l1_oo, p99_oo = log_density_l1(c2, c1)
    im1 = oracle_image(cfg, c1, r1, p1, ss)
    im2 = oracle_image(cfg, c2, r2, p2, ss)
    img_go = float(np.abs(img.astype(np.int64) - im1.astype(np.int64)).mean())
    img_oo = float(np.abs(im2.astype(np.int64) - im1.astype(np.int64)).mean())
    return {
        "l1": l1_go, "p99": p99_go, "oracle_l1": l1_oo, "oracle_p99": p99_oo,
        "blocks_z5": block_outliers(cnt, c1), "oracle_blocks_z5": block_outliers(c2, c1),
        "image_mad": img_go, "oracle_image_mad": img_oo,
        "samples": int(out.total_iterations), "samples_per_px": out.total_iterations / float(W * H),
        "inframe": int(out.inframe_samples), "oracle_inframe": [int(i1), int(i2)],
        "size": [W, H], "walkers": walkers, "seeds": list(seeds), "kernel_launches": int(out.kernel_launches),
        "image_launches": int(oimg.kernel_launches),
    }


def within_noise(m):
    """The acceptance rule: GPU-vs-oracle within 1.25x oracle-vs-oracle (plus
    a floor) on every measure."""
    return (m["l1"] <= 1.25 * m["oracle_l1"] + 0.01 and m["p99"] <= 1.25 * m["oracle_p99"] + 0.05
            and m["blocks_z5"] <= max(2, m["oracle_blocks_z5"] + 2)
            and m["image_mad"] <= 1.25 * m["oracle_image_mad"] + 0.25)

