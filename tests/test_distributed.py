"""The multi-GPU render logic (ffb200.distributed) on world_size-2 `gloo`
ranks, with an oracle-backed CPU backend in place of the CUDA kernels: walker
sharding, the histogram all-reduce of the count and colour planes, the
per-rank row bands (DE halo from the summed histogram) and the gather must
give exactly the single-rank frame."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


class OracleBackend:
    """The CPU oracle behind the backend interface of ffb200.distributed."""

    def __init__(self, O):
        self.O = O

    def empty(self, n, dtype):
        return torch.zeros(n, dtype=dtype)

    def chaos(self, cfg, job, hist):
        import json
        c = json.loads(cfg)
        ss = job.get("supersample", 1)
        W, H = job["width"] * ss, job["height"] * ss
        fl = self.O.Flame(c, W, H)
        per = job["iterations"] // job["walkers"]
        plotted, _, cnt, rgb = fl.render(job["walkers"], per + 20, seed=job.get("seed", 12345), walker0=job["walker0"],
                                         threads=2)
        h = hist.view(-1, 4)
        h[:, :3] = torch.from_numpy(rgb.reshape(-1, 3).astype(np.float32))
        h[:, 3] = torch.from_numpy(cnt.reshape(-1).view(np.float32))
        return plotted

    def pack(self, hist, counts, rgb):
        h = hist.view(-1, 4)
        counts.copy_(h[:, 3].contiguous().view(torch.int32))
        rgb.copy_(h[:, :3].reshape(-1))

    def unpack(self, counts, rgb, hist):
        h = hist.view(-1, 4)
        h[:, :3] = rgb.view(-1, 3)
        h[:, 3] = counts.view(torch.float32)

    def finish(self, cfg, job, hist, samples, row0, rows, band):
        import json
        c = json.loads(cfg)
        ss = job.get("supersample", 1)
        W, H = job["width"] * ss, job["height"] * ss
        h = hist.view(-1, 4).numpy()
        cnt = h[:, 3].copy().view(np.uint32).astype(np.float64).reshape(H, W)
        rgb = h[:, :3].astype(np.float64).reshape(H, W, 3)
        de = c.get("density_estimation")
        if de and de.get("radius", 0) > 0:
            cnt, rgb = self.O.density_estimate(cnt, rgb, W, H, de["radius"] * ss, de.get("minimum", 0.0) * ss, de.get("curve", 0.4))
        y0, y1 = row0 * ss, (row0 + rows) * ss
        P = self.O.tonemap_params_for(c, W, H, samples / (W * H), job.get("transparent", 0))
        _, u8 = self.O.tonemap(P, cnt[y0:y1], rgb[y0:y1])
        u8 = u8.reshape(y1 - y0, W, 4)
        if ss == 2:
            u8 = self.O.downsample_firefly(u8, job["width"], rows)
        band[:rows * job["width"] * 4] = torch.from_numpy(np.ascontiguousarray(u8).reshape(-1))

    def sync(self):
        pass


def _cfg():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "fflame-rust_b200"))
    from ffb200 import synthetic
    c = synthetic.plain_flame(4)
    c["density_estimation"] = {"radius": 2.0, "minimum": 0.0, "curve": 0.4}
    return c


def _worker(rank, world, port, out_path, width, height, ss):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "fflame-rust_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from oracle import oracle as O
    from ffb200 import distributed as D
    frame, samples = D.render(OracleBackend(O), _cfg(), width, height, iterations=600 * 300, walkers=600,
                              supersample=ss, seed=99)
    if rank == 0:
        np.save(out_path, frame.numpy())
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("ss", [1, 2])
def test_two_rank_render_equals_one_rank(oracle, tmp_path, ss):
    width, height = 40, 30
    out2 = str(tmp_path / "two.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out2, width, height, ss), nprocs=2, start_method="spawn")
    out1 = str(tmp_path / "one.npy")
    mp.start_processes(_worker, args=(1, _free_port(), out1, width, height, ss), nprocs=1, start_method="spawn")
    a, b = np.load(out2), np.load(out1)
    assert a.shape == (height, width, 4)
    assert (a[..., :3].max(axis=2) > 0).sum() > 50
    d = np.abs(a.astype(int) - b.astype(int))
    assert d.max() <= 1 and (d > 0).mean() < 0.01


def test_shards_and_bands_cover_everything():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "fflame-rust_b200"))
    from ffb200.distributed import shard, bands
    for total in (1, 7, 65536, 65537):
        for world in (1, 2, 3, 8):
            parts = [shard(total, world, r) for r in range(world)]
            assert parts[0][0] == 0
            for (a, n), (b, _) in zip(parts, parts[1:]):
                assert a + n == b
            assert sum(n for _, n in parts) == total
            assert max(n for _, n in parts) - min(n for _, n in parts) <= 1
    assert bands(1080, 8)[-1] == (945, 135)
