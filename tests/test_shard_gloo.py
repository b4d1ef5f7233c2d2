"""Multi-process path on CPU (gloo, world size 2): photon-range sharding plus the
exact int64 film all-reduce reproduce the single-process film bit for bit.
The per-rank films come from the CPU oracle standing in for each rank's GPU."""
import ctypes as C
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from spectral_b200.shard import allreduce_film_, gather_bands, photon_range, row_band


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _scene():
    import oracle
    from helpers import obeam, ocam, oscene
    import spectral_b200 as sb
    scene, beam, cam = sb.dsotm_scene(1.0)
    return oscene(scene), obeam(beam), ocam(cam), oracle.vol_params(48, 40, 9, 0.5, 0.06, 0.5, 14.0, bins=16)


def _worker(rank, world, port, n, out_path):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    import oracle
    osc, ob, oc, p = _scene()
    b, e = photon_range(rank, world, n)
    _, _, fs = oracle.render_point(osc, oc, ob, p, b, e, f32=False, xyz=False, spec=True)
    t = torch.from_numpy(fs)
    allreduce_film_(t)
    if rank == 0:
        np.save(out_path, t.numpy())
    dist.barrier()
    dist.destroy_process_group()


def _tracer_scene():
    import oracle
    from helpers import ocam, oscene
    import spectral_b200 as sb
    s = sb.Scene(background=1.0)
    s.add_sphere((0, 0, -3), 1.0, sb.Dielectric(sb.SF11))
    cam = sb.Camera.look_at((0, 0.3, 0.5), (0, 0, -3), (0, 1, 0), 55.0, 1.5)
    return oracle, oscene(s), ocam(cam)


def _tracer_worker(rank, world, port, w, h, spp, out_path):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    oracle, osc, oc = _tracer_scene()
    b, e = row_band(rank, world, h)
    acc = np.zeros(3 * w * h, np.float32)
    oracle.lib.or_tracer_accumulate(C.byref(osc.c), C.byref(oc), w, h, 0, 5, spp, 0, 8, b, e, oracle.fp(acc))
    img = (acc / np.float32(spp)).reshape(h, w, 3)
    full = gather_bands(img[b:e], rank, world, h)
    np.save(out_path % rank, full)
    dist.barrier()
    dist.destroy_process_group()


class _OracleTracer:
    """Stand-in for GpuTracer on a gloo rank: the same dims / set_rows /
    accumulate / read_xyz calls, rendered by the CPU oracle."""

    def __init__(self, w, h, seed):
        self.oracle, self.osc, self.oc = _tracer_scene()
        self.w, self.h, self.seed = w, h, seed
        self.rows, self.samples = (0, h), 0
        self.sum = np.zeros(3 * w * h, np.float32)

    def dims(self):
        return self.w, self.h

    def set_rows(self, b, e):
        self.rows = (b, e)

    def accumulate(self, spp):
        self.oracle.lib.or_tracer_accumulate(C.byref(self.osc.c), C.byref(self.oc), self.w, self.h, 0, self.seed, spp,
                                             self.samples, 8, self.rows[0], self.rows[1], self.oracle.fp(self.sum))
        self.samples += spp

    def read_xyz(self):
        return self.sum / np.float32(max(self.samples, 1))


def _trace_rows_worker(rank, world, port, w, h, spp, out_path):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    from spectral_b200.shard import trace_rows_sharded
    np.save(out_path % rank, trace_rows_sharded(_OracleTracer(w, h, 5), spp))
    dist.barrier()
    dist.destroy_process_group()


def test_trace_rows_sharded_on_two_ranks(tmp_path):
    """shard.trace_rows_sharded end to end on two gloo ranks (set_rows,
    accumulate, read back, gather), the oracle standing in for each GPU."""
    w, h, spp, world = 20, 13, 3, 2
    out = str(tmp_path / "rows%d.npy")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_trace_rows_worker, args=(r, world, port, w, h, spp, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    whole = _OracleTracer(w, h, 5)
    whole.accumulate(spp)
    ref = whole.read_xyz().reshape(h, w, 3)
    assert ref.sum() > 0
    for r in range(world):
        assert np.load(out % r).tobytes() == ref.tobytes(), r


@pytest.mark.parametrize("world", [2, 3])
def test_tracer_row_bands_gather_to_the_full_image(tmp_path, world):
    """Pixel-row ownership for the camera tracer: each rank renders its band of
    rows (the CPU oracle standing in for its GPU) and the gathered image equals
    the single-process render bit for bit on every rank."""
    w, h, spp = 24, 17, 4
    out = str(tmp_path / "img%d.npy")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_tracer_worker, args=(r, world, port, w, h, spp, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    oracle, osc, oc = _tracer_scene()
    whole = np.zeros(3 * w * h, np.float32)
    oracle.lib.or_tracer_accumulate(C.byref(osc.c), C.byref(oc), w, h, 0, 5, spp, 0, 8, 0, h, oracle.fp(whole))
    whole = (whole / np.float32(spp)).reshape(h, w, 3)
    assert whole.sum() > 0
    for r in range(world):
        assert np.load(out % r).tobytes() == whole.tobytes(), r


def test_photon_range_partitions():
    for world in (1, 2, 3, 8):
        for n in (0, 1, 7, 1000, 2 ** 20 + 3):
            ranges = [photon_range(r, world, n, base=5) for r in range(world)]
            assert ranges[0][0] == 5 and ranges[-1][1] == 5 + n
            assert all(ranges[i][1] == ranges[i + 1][0] for i in range(world - 1))
    with pytest.raises(ValueError):
        photon_range(2, 2, 10)


def test_two_rank_film_reduce_is_exact(tmp_path):
    n = 6000
    out = str(tmp_path / "film.npy")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, n, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    import oracle
    osc, ob, oc, p = _scene()
    _, _, whole = oracle.render_point(osc, oc, ob, p, 0, n, f32=False, xyz=False, spec=True)
    assert (np.load(out) == whole).all() and whole.sum() > 0


def test_float_films_are_refused():
    with pytest.raises(TypeError):
        allreduce_film_(torch.zeros(4, dtype=torch.float32))


def test_tile_row_bands_cover_the_image_on_tile_boundaries():
    """The peer-band split gives every rank a band of whole 8-row tile rows:
    contiguous, covering [0, height), each starting on a multiple of 8."""
    from spectral_b200.shard import tile_row_band
    for height in (1, 7, 8, 9, 75, 80, 720, 1080):
        for world in (1, 2, 3, 5, 8, 16):
            bands = [tile_row_band(r, world, height) for r in range(world)]
            assert bands[0][0] == 0 and bands[-1][1] == height
            for (b0, e0), (b1, e1) in zip(bands, bands[1:]):
                assert e0 == b1
            for b, e in bands:
                assert b <= e and b % 8 == 0 and (e % 8 == 0 or e == height)
