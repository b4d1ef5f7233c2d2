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


# ---- the split without an all-reduce: bands reduced from every rank's film ----

def _device_film(torch, _lib, ch):
    film = torch.zeros(_lib.lib.sc_film_bytes(W, H, ch) // 8, dtype=torch.int64, device="cuda")
    flags = torch.zeros(_lib.lib.sc_film_flag_bytes(W, H) // 4, dtype=torch.int32, device="cuda")
    return film, flags


def _trace(ctx, _lib, torch, desc, begin, end, film, flags):
    import ctypes as C
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(_lib.lib.sc_trace_photons_device(ctx.h, C.byref(desc), begin, end - begin,
                                                C.c_void_p(film.data_ptr()), C.c_void_p(flags.data_ptr()), stream))


def _one_film_image(ctx, bins):
    """The reference: one device film traced with every photon, reduced whole."""
    import ctypes as C
    import torch
    import spectral_b200 as sb
    from spectral_b200 import _lib
    from helpers import device_desc
    keep = []
    scene, beam, cam = sb.dsotm_scene(W / H)
    desc = device_desc(sb, _lib, torch, scene, cam, beam, W, H, SEED, bins, keep)
    ch = bins or 3
    film, flags = _device_film(torch, _lib, ch)
    _trace(ctx, _lib, torch, desc, 0, N, film, flags)
    xyz = torch.empty(3 * W * H, dtype=torch.float32, device="cuda")
    _lib.check(_lib.lib.sc_sensor_reduce_device(ctx.h, W, H, ch, 380.0, 730.0, 32, C.c_void_p(film.data_ptr()),
                                                C.c_void_p(flags.data_ptr()), C.c_void_p(xyz.data_ptr()), 0,
                                                C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    return xyz.cpu().numpy().reshape(H, W, 3)


@pytest.mark.parametrize("bins", [0, BINS])
def test_band_reduction_of_several_films_equals_one_film(ctx, bins):
    """Three device films, each holding a third of the photons, reduced band by
    band (whole tile rows) from their sum give the one-film image bit for bit."""
    import torch
    import spectral_b200 as sb
    from spectral_b200 import _lib
    from spectral_b200.shard import photon_range, reduce_band_peers, tile_row_band
    from helpers import device_desc
    keep = []
    scene, beam, cam = sb.dsotm_scene(W / H)
    desc = device_desc(sb, _lib, torch, scene, cam, beam, W, H, SEED, bins, keep)
    ch, world = bins or 3, 3
    films = []
    for r in range(world):
        film, flags = _device_film(torch, _lib, ch)
        _trace(ctx, _lib, torch, desc, *photon_range(r, world, N), film, flags)
        films.append(film)
    xyz = torch.full((3 * W * H,), float("nan"), dtype=torch.float32, device="cuda")
    for r in range(world):
        b, e = tile_row_band(r, world, H)
        reduce_band_peers(ctx, [f.data_ptr() for f in films], W, H, ch, desc.opts, b, e, xyz.data_ptr(),
                          torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    got = xyz.cpu().numpy().reshape(H, W, 3)
    ref = _one_film_image(ctx, bins)
    assert ref.sum() > 0 and got.tobytes() == ref.tobytes()
    with pytest.raises(_lib.SpectralError):  # a band must start on a tile row
        reduce_band_peers(ctx, [films[0].data_ptr()], W, H, ch, desc.opts, 4, 16, xyz.data_ptr())


def _peer_rank(rank, world, port, out_dir):
    import datetime
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist
    import spectral_b200 as sb
    from spectral_b200 import _lib
    from spectral_b200.shard import PeerFilms, photon_range, reduce_sharded_peers
    from helpers import device_desc
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    ctx = sb.GpuContext(0)
    keep = []
    scene, beam, cam = sb.dsotm_scene(W / H)
    desc = device_desc(sb, _lib, torch, scene, cam, beam, W, H, SEED, BINS, keep)
    film, flags = _device_film(torch, _lib, BINS)
    _trace(ctx, _lib, torch, desc, *photon_range(rank, world, N), film, flags)
    peers = PeerFilms(ctx, film)
    img = reduce_sharded_peers(peers, W, H, BINS, desc.opts)
    np.save(os.path.join(out_dir, "peer%d.npy" % rank), img)
    peers.close()
    dist.barrier()  # every rank has unmapped the others' films before they go
    del film, flags, keep
    ctx.close()
    dist.destroy_process_group()


def test_two_processes_reduce_bands_from_each_others_films(ctx, tmp_path):
    """Two processes (gloo ranks on cuda:0) trace their photon ranges into their
    own device films, map each other's film (CUDA IPC), each reduces its band of
    tile rows from the sum, and the gathered image equals one film's, bit for
    bit.  No kernel waits on another: the barriers are on the host."""
    world = 2
    mp.spawn(_peer_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    ref = _one_film_image(ctx, BINS)
    assert ref.sum() > 0
    for r in range(world):
        assert np.load(tmp_path / ("peer%d.npy" % r)).tobytes() == ref.tobytes(), r
