"""Multi-GPU rendering: one process a GPU, torch.distributed for the plumbing.

The path shards by walkers.  Rank r renders walkers [w0_r, w0_r + n_r) of the
flame into its own histogram; the walkers' streams are keyed by their global
ids, so the union of the shards is exactly the single-GPU render.  The one
exchange step is the histogram sum, as a reduce-scatter over row windows:
rank r owns a band of output rows, and its window is the band's internal
rows plus the density-estimation reach on either side (clamped to the
image), padded to one common length.  Each rank packs its histogram into a
u32 count plane and an f32 colour plane, lays the world's windows of each
plane side by side, and a reduce-scatter (NCCL over NVLink) leaves every
rank the sum of its own window -- about (world - 1) / world of the
histogram crosses the links, half of an all-reduce.  Each rank then runs
density estimation and the tone map on its band from its window, and the
bands are gathered.

The collective and banding logic is backend-neutral: `CudaBackend` drives the
CUDA kernels through the C ABI; tests supply a CPU backend and run the same
logic on `gloo` ranks.
"""

import contextlib
import math
import json

import torch
import torch.distributed as dist


def shard(total, world, rank):
    """Walkers [first, first + count) of rank `rank` (the remainder spread over the first ranks)."""
    base, extra = divmod(total, world)
    count = base + (1 if rank < extra else 0)
    first = rank * base + min(rank, extra)
    return first, count


def bands(height, world):
    """Output row bands (row0, rows), one a rank, covering [0, height)."""
    return [shard(height, world, r) for r in range(world)]


def de_reach(config, supersample):
    """Internal rows density estimation reads on either side of a band:
    ceil(radius x supersample), 0 without density estimation."""
    cfg = json.loads(config) if isinstance(config, str) else config
    de = cfg.get("density_estimation") or {}
    r = float(de.get("radius", 0.0) or 0.0)
    return int(math.ceil(r * supersample)) if r > 0 else 0


def windows(height, supersample, world, reach):
    """Each rank's histogram window: (first internal row, rows), one length
    for all ranks (a reduce-scatter's chunks are equal), holding the rank's
    band and `reach` rows on either side where the image has them."""
    H = height * supersample
    need = []
    for row0, rows in bands(height, world):
        lo = max(0, row0 * supersample - reach)
        hi = min(H, (row0 + rows) * supersample + reach)
        need.append((lo, hi))
    length = max(hi - lo for lo, hi in need)
    return [(min(lo, H - length), length) for lo, _ in need]


class CudaBackend:
    """The CUDA path: a Renderer of this rank's device, on one stream."""

    def __init__(self, renderer, device, stream=None):
        self.r = renderer
        self.device = device
        self.stream = stream or torch.cuda.current_stream(device)

    def empty(self, n, dtype):
        return torch.empty(n, dtype=dtype, device=self.device)

    def chaos(self, cfg, job, hist):
        o = self.r.chaos_device(cfg, job["width"], job["height"], hist.data_ptr(), stream=self.stream.cuda_stream,
                                **{k: v for k, v in job.items() if k not in ("width", "height")})
        return o.total_iterations

    def pack(self, hist, counts, rgb):
        self.r.hist_pack(hist.data_ptr(), counts.numel(), counts.data_ptr(), rgb.data_ptr(), stream=self.stream.cuda_stream)

    def unpack(self, counts, rgb, hist):
        self.r.hist_unpack(counts.data_ptr(), rgb.data_ptr(), counts.numel(), hist.data_ptr(), stream=self.stream.cuda_stream)

    def stream_context(self):
        """Torch's current stream is the backend's while a frame's kernels and
        collectives are queued, so NCCL orders against the library's work."""
        return torch.cuda.stream(self.stream)

    def finish_band(self, cfg, job, hist, hist_row0, hist_rows, samples, row0, rows, band):
        self.r.finish_band(cfg, job["width"], job["height"], hist.data_ptr(), hist_row0, hist_rows, samples, row0, rows,
                           band.data_ptr(), stream=self.stream.cuda_stream,
                           **{k: v for k, v in job.items() if k not in ("width", "height")})

    def finish(self, cfg, job, hist, samples, row0, rows, band):
        self.r.finish_device(cfg, job["width"], job["height"], hist.data_ptr(), samples, row0, rows, band.data_ptr(),
                             stream=self.stream.cuda_stream,
                             **{k: v for k, v in job.items() if k not in ("width", "height")})

    def sync(self):
        self.stream.synchronize()


def render(backend, config, width, height, iterations, walkers, supersample=1, group=None, gather=True, **job):
    """One frame over the ranks of `group`: RGBA8 [height, width, 4] (on every
    rank when `gather`), and the total plotted samples."""
    ctx = backend.stream_context() if hasattr(backend, "stream_context") else contextlib.nullcontext()
    with ctx:
        return _render(backend, config, width, height, iterations, walkers, supersample, group, gather, **job)


def _render(backend, config, width, height, iterations, walkers, supersample, group, gather, **job):
    cfg = config if isinstance(config, str) else json.dumps(config)
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    per_walker = -(-iterations // walkers)
    w0, nw = shard(walkers, world, rank)
    W, H = width * supersample, height * supersample
    npx = W * H
    base = dict(job, width=width, height=height, supersample=supersample)
    shard_job = dict(base, walkers=nw, walker0=w0 + base.get("walker0", 0), iterations=nw * per_walker)
    hist = backend.empty(npx * 4, torch.float32)
    # Each rank's plotted samples (its walkers past their burn-in, restarted
    # walkers of an orbit-refreshed flame burning in again), summed.
    samples = int(backend.chaos(cfg, shard_job, hist))
    if world > 1:
        total = backend.empty(1, torch.int64)
        total.fill_(samples)
        dist.all_reduce(total, op=dist.ReduceOp.SUM, group=group)
        samples = int(total.item())
    row0, rows = bands(height, world)[rank]
    if world > 1:
        wins = windows(height, supersample, world, de_reach(cfg, supersample))
        win0, L = wins[rank]
        counts = backend.empty(npx, torch.int32)
        rgb = backend.empty(npx * 3, torch.float32)
        backend.pack(hist, counts, rgb)
        # The world's windows side by side (they overlap by the halo).
        c_in = backend.empty(world * L * W, torch.int32)
        r_in = backend.empty(world * L * W * 3, torch.float32)
        for r, (a, _) in enumerate(wins):
            c_in[r * L * W:(r + 1) * L * W].copy_(counts[a * W:(a + L) * W])
            r_in[r * L * W * 3:(r + 1) * L * W * 3].copy_(rgb[a * W * 3:(a + L) * W * 3])
        c_out = backend.empty(L * W, torch.int32)
        r_out = backend.empty(L * W * 3, torch.float32)
        # u32 counts summed as int32: two's-complement addition is the same bits.
        dist.reduce_scatter_tensor(c_out, c_in, op=dist.ReduceOp.SUM, group=group)
        dist.reduce_scatter_tensor(r_out, r_in, op=dist.ReduceOp.SUM, group=group)
        win = backend.empty(L * W * 4, torch.float32)
        backend.unpack(c_out, r_out, win)
    else:
        win0, L, win = 0, H, hist
    band = backend.empty(max(rows, 1) * width * 4, torch.uint8)
    if rows:
        backend.finish_band(cfg, base, win, win0, L, samples, row0, rows, band)
    backend.sync()
    if not gather:
        return band[:rows * width * 4].view(rows, width, 4), samples
    if world == 1:
        return band.view(height, width, 4), samples
    most = max(r for _, r in bands(height, world))
    padded = backend.empty(most * width * 4, torch.uint8)
    padded.zero_()
    padded[:rows * width * 4].copy_(band[:rows * width * 4])
    parts = [backend.empty(most * width * 4, torch.uint8) for _ in range(world)]
    dist.all_gather(parts, padded, group=group)
    frame = torch.cat([p[:r * width * 4] for p, (_, r) in zip(parts, bands(height, world))])
    return frame.view(height, width, 4), samples
