"""Multi-GPU rendering: one process a GPU, torch.distributed for the plumbing.

The path shards by walkers.  Rank r renders walkers [w0_r, w0_r + n_r) of the
flame into its own histogram; the walkers' streams are keyed by their global
ids, so the union of the shards is exactly the single-GPU render.  The one
exchange step is the histogram sum (an all-reduce of the u32 count plane and
of the f32 colour plane, NCCL over NVLink), after which each rank runs density
estimation and the tone map on its own band of output rows (the DE halo comes
from the summed histogram) and the bands are gathered.

The collective and banding logic is backend-neutral: `CudaBackend` drives the
CUDA kernels through the C ABI; tests supply a CPU backend and run the same
logic on `gloo` ranks.
"""

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

    def finish(self, cfg, job, hist, samples, row0, rows, band):
        self.r.finish_device(cfg, job["width"], job["height"], hist.data_ptr(), samples, row0, rows, band.data_ptr(),
                             stream=self.stream.cuda_stream,
                             **{k: v for k, v in job.items() if k not in ("width", "height")})

    def sync(self):
        self.stream.synchronize()


def render(backend, config, width, height, iterations, walkers, supersample=1, group=None, gather=True, **job):
    """One frame over the ranks of `group`: RGBA8 [height, width, 4] (on every
    rank when `gather`), and the total plotted samples."""
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
    if world > 1:
        counts = backend.empty(npx, torch.int32)
        rgb = backend.empty(npx * 3, torch.float32)
        backend.pack(hist, counts, rgb)
        backend.sync()
        # u32 counts summed as int32: two's-complement addition is the same bits.
        dist.all_reduce(counts, op=dist.ReduceOp.SUM, group=group)
        dist.all_reduce(rgb, op=dist.ReduceOp.SUM, group=group)
        backend.unpack(counts, rgb, hist)
    row0, rows = bands(height, world)[rank]
    band = backend.empty(max(rows, 1) * width * 4, torch.uint8)
    if rows:
        backend.finish(cfg, base, hist, samples, row0, rows, band)
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
