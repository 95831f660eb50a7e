"""The multi-GPU render logic (ffb200.distributed) on `gloo` ranks (world
sizes 2 and 3), with an oracle-backed CPU backend in place of the CUDA
kernels: walker sharding, the reduce-scatter of the count and colour planes
over row windows (each rank's band plus the density-estimation reach), the
per-rank bands finished from their windows and the gather must give the
single-rank frame.  A density-estimation radius wider than half a band puts
the halo across band edges.

On one GPU (marked gpu): the device building blocks the ranks call --
walker shards into separate histograms, the pack into planes and back, and
the band finish from a window -- assembled in one process against a single
render."""

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

    def finish_band(self, cfg, job, hist, hist_row0, hist_rows, samples, row0, rows, band):
        import json
        c = json.loads(cfg)
        ss = job.get("supersample", 1)
        W, H = job["width"] * ss, job["height"] * ss
        h = hist.view(-1, 4).numpy()
        cnt = h[:, 3].copy().view(np.uint32).astype(np.float64).reshape(hist_rows, W)
        rgb = h[:, :3].astype(np.float64).reshape(hist_rows, W, 3)
        de = c.get("density_estimation")
        if de and de.get("radius", 0) > 0:
            cnt, rgb = self.O.density_estimate(cnt, rgb, W, hist_rows, de["radius"] * ss, de.get("minimum", 0.0) * ss,
                                               de.get("curve", 0.4))
        y0, y1 = row0 * ss - hist_row0, (row0 + rows) * ss - hist_row0
        P = self.O.tonemap_params_for(c, W, H, samples / (W * H), job.get("transparent", 0))
        _, u8 = self.O.tonemap(P, cnt[y0:y1], rgb[y0:y1])
        u8 = u8.reshape(y1 - y0, W, 4)
        if ss == 2:
            u8 = self.O.downsample_firefly(u8, job["width"], rows)
        band[:rows * job["width"] * 4] = torch.from_numpy(np.ascontiguousarray(u8).reshape(-1))

    def sync(self):
        pass


def _cfg(radius=2.0):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "fflame-rust_b200"))
    from ffb200 import synthetic
    c = synthetic.plain_flame(4)
    c["density_estimation"] = {"radius": radius, "minimum": 0.0, "curve": 0.4}
    return c


def _worker(rank, world, port, out_path, width, height, ss, radius=2.0):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "fflame-rust_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    from oracle import oracle as O
    from ffb200 import distributed as D
    frame, samples = D.render(OracleBackend(O), _cfg(radius), width, height, iterations=600 * 300, walkers=600,
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


@pytest.mark.parametrize("world", [2, 3])
def test_halo_wider_than_half_a_band(oracle, tmp_path, world):
    """DE radius 9 against bands of 10-15 rows: every band's density estimate
    reads rows of its neighbours' bands, from the rank's own summed window."""
    width, height = 40, 30
    outn = str(tmp_path / "n.npy")
    mp.start_processes(_worker, args=(world, _free_port(), outn, width, height, 1, 9.0), nprocs=world, start_method="spawn")
    out1 = str(tmp_path / "one.npy")
    mp.start_processes(_worker, args=(1, _free_port(), out1, width, height, 1, 9.0), nprocs=1, start_method="spawn")
    a, b = np.load(outn), np.load(out1)
    d = np.abs(a.astype(int) - b.astype(int))
    assert (a[..., :3].max(axis=2) > 0).sum() > 50
    assert d.max() <= 1 and (d > 0).mean() < 0.01


def test_windows_hold_each_band_and_its_reach():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "fflame-rust_b200"))
    from ffb200.distributed import bands, windows
    for height, ss, world, reach in ((30, 1, 2, 9), (1080, 2, 8, 18), (7, 2, 3, 40), (100, 1, 4, 0)):
        H = height * ss
        wins = windows(height, ss, world, reach)
        assert len({L for _, L in wins}) == 1
        for (row0, rows), (a, L) in zip(bands(height, world), wins):
            assert 0 <= a and a + L <= H
            assert a <= max(0, row0 * ss - reach) and a + L >= min(H, (row0 + rows) * ss + reach)


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


@pytest.mark.gpu
@pytest.mark.parametrize("radius", [0.0, 9.0])
def test_device_building_blocks_assemble_the_single_render(renderer, radius):
    """On one GPU, in one process: two walker shards rendered by
    ffb_chaos_device into two histograms, each split by ffb_hist_pack, the
    planes summed, joined by ffb_hist_unpack, and the frame finished as two
    row bands (ffb_finish_device on the whole histogram and ffb_finish_band
    on each band's window) -- against one render of all the walkers: the
    count plane bit for bit, the image within 1 LSB."""
    import json as _json
    import sys
    sys.path.insert(0, os.path.join(ROOT, "fflame-rust_b200"))
    from ffb200 import distributed as D, synthetic
    cfg = synthetic.full_flame(6, de_radius=radius)
    text = _json.dumps(cfg)
    w, h, ss, walkers, per = 240, 135, 2, 32768, 300
    W, H = w * ss, h * ss
    job = dict(supersample=ss, seed=77)
    dev = torch.device("cuda", 0)
    hists, total = [], 0
    for w0, nw in (D.shard(walkers, 2, 0), D.shard(walkers, 2, 1)):
        hist = torch.zeros(W * H * 4, dtype=torch.float32, device=dev)
        o = renderer.chaos_device(text, w, h, hist.data_ptr(), walkers=nw, walker0=w0, iterations=nw * per, **job)
        total += o.total_iterations
        hists.append(hist)
    torch.cuda.synchronize(dev)
    counts = [torch.empty(W * H, dtype=torch.int32, device=dev) for _ in hists]
    rgbs = [torch.empty(W * H * 3, dtype=torch.float32, device=dev) for _ in hists]
    for hist, c, r in zip(hists, counts, rgbs):
        renderer.hist_pack(hist.data_ptr(), W * H, c.data_ptr(), r.data_ptr())
    torch.cuda.synchronize(dev)
    csum, rsum = counts[0] + counts[1], rgbs[0] + rgbs[1]
    summed = torch.empty(W * H * 4, dtype=torch.float32, device=dev)
    renderer.hist_unpack(csum.data_ptr(), rsum.data_ptr(), W * H, summed.data_ptr())
    torch.cuda.synchronize(dev)
    ref_cnt, _, ref_o = renderer.histogram(cfg, w, h, walkers=walkers, iterations=walkers * per, **job)
    assert total == ref_o.total_iterations
    got_cnt = summed.view(H, W, 4)[..., 3].contiguous().view(torch.int32).cpu().numpy().view(np.uint32)
    assert np.array_equal(got_cnt, ref_cnt)
    ref_img, _ = renderer.render(cfg, w, h, walkers=walkers, iterations=walkers * per, **job)
    wins = D.windows(h, ss, 2, D.de_reach(cfg, ss))
    for finish in ("device", "band"):
        parts = []
        for (row0, rows), (a, L) in zip(D.bands(h, 2), wins):
            band = torch.empty(rows * w * 4, dtype=torch.uint8, device=dev)
            if finish == "device":
                renderer.finish_device(text, w, h, summed.data_ptr(), total, row0, rows, band.data_ptr(), **job)
            else:
                win = summed[a * W * 4:(a + L) * W * 4].clone()
                renderer.finish_band(text, w, h, win.data_ptr(), a, L, total, row0, rows, band.data_ptr(), **job)
            torch.cuda.synchronize(dev)
            parts.append(band.cpu().numpy().reshape(rows, w, 4))
        img = np.concatenate(parts)
        d = np.abs(img.astype(int) - ref_img.astype(int))
        assert d.max() <= 1, (finish, d.max())
    # A window short of the DE reach is refused, not read past.
    if radius > 0:
        row0, rows = D.bands(h, 2)[1]
        win = summed[row0 * ss * W * 4:].clone()
        band = torch.empty(rows * w * 4, dtype=torch.uint8, device=dev)
        with pytest.raises(Exception) as e:
            renderer.finish_band(text, w, h, win.data_ptr(), row0 * ss, H - row0 * ss, total, row0, rows,
                                 band.data_ptr(), **job)
        assert "window" in str(e.value)
