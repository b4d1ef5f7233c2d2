"""The device leg of the photon-range split, on one GPU: two processes (gloo
ranks, both on cuda:0) each trace their photon range into their own device
film, trace_sharded sums the films through host memory and writes the sum
back into each device film, and the result must equal, bit for bit, one
process tracing every photon.  The code path is the one NCCL takes across
GPUs apart from where the sum is formed; the two ranks' kernels never wait on
each other (the exchange is on the host)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

W, H, BINS, N, SEED = 96, 80, 16, 300_001, 0x5AD


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _film(sb, ctx):
    scene, beam, cam = sb.dsotm_scene(W / H)
    return sb.GpuPhotonFilm(ctx, scene, cam, beam, W, H, N, SEED, 14.0, sb.VolWeights(), bins=BINS)


def _rank(rank, world, port, out_dir):
    import datetime
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist
    import spectral_b200 as sb
    from spectral_b200.shard import trace_sharded
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    ctx = sb.GpuContext(0)
    film = _film(sb, ctx)
    trace_sharded(film, N, SEED)
    np.save(os.path.join(out_dir, "raw%d.npy" % rank), film.read_raw())
    np.save(os.path.join(out_dir, "xyz%d.npy" % rank), film.accum())
    film.close()
    ctx.close()
    dist.barrier()
    dist.destroy_process_group()


def test_photon_range_split_device_films_sum_to_one_film(ctx, tmp_path):
    import spectral_b200 as sb
    world = 2
    mp.spawn(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    one = _film(sb, ctx)
    one.dispatch_photons(0, N, SEED)
    raw, xyz = one.read_raw(), one.accum()
    one.close()
    assert raw.sum() > 0
    for r in range(world):
        assert np.load(tmp_path / ("raw%d.npy" % r)).tobytes() == raw.tobytes(), r
        assert np.load(tmp_path / ("xyz%d.npy" % r)).tobytes() == xyz.tobytes(), r
