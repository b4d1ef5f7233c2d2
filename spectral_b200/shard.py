"""Multi-GPU sharding of one scene's photons (one process per GPU).

Photon i is keyed by its global index (its RNG stream is PathRng(i, seed)), so
a scene's photons split into contiguous index ranges, one per rank, with no
communication while tracing.  Each rank's 64-bit fixed-point film then holds
the exact sum of its photons' splats, and ONE all-reduce (sum) of the int64
films over NCCL (NVLink / NVSwitch) gives the film of the whole range,
bit-identical to a single-GPU trace and independent of the number of ranks or
the reduction order.  Batches and serving shard by whole scenes / requests and
need no collective at all.

Without the all-reduce (`PeerFilms`, `reduce_sharded_peers`): each rank maps
the other ranks' films into its process (CUDA IPC; peer memory over NVLink
between GPUs) and reduces its own band of tile rows straight from the sum of
all the films, so no film is summed into one or sent whole (each GPU reads
1/N of every film instead of moving two films' worth through an all-reduce),
and only the XYZ bands are gathered.  Same exact int64 sum, same image bits.

The camera tracer shards by pixels instead: each rank owns a contiguous band
of image rows (a pixel's samples are keyed by the pixel and sample index, so
a row renders the same on any rank), traces only that band, and the bands are
gathered into the full image.  Every pixel has one owner: no reduction.
"""
import ctypes as C

import numpy as np

from ._lib import check, lib


def photon_range(rank, world, n_photons, base=0):
    """Contiguous [begin, end) of photon indices owned by `rank`."""
    if not (0 <= rank < world):
        raise ValueError("rank %d outside world %d" % (rank, world))
    begin = base + (n_photons * rank) // world
    end = base + (n_photons * (rank + 1)) // world
    return begin, end


class _CudaArray:
    """__cuda_array_interface__ view of a device buffer (no copy)."""

    def __init__(self, ptr, nbytes, typestr, itemsize, stream):
        self.__cuda_array_interface__ = {"shape": (nbytes // itemsize,), "typestr": typestr,
                                         "data": (ptr, False), "version": 3, "strides": None,
                                         "stream": stream or 1}


def film_tensor(film):
    """int64 torch tensor aliasing a GpuPhotonFilm's device film (tile-major cells)."""
    import torch
    fp, fb, gp, gb, st = C.c_void_p(), C.c_size_t(), C.c_void_p(), C.c_size_t(), C.c_void_p()
    check(lib.sc_photon_film_device_buffers(film.h, C.byref(fp), C.byref(fb), C.byref(gp), C.byref(gb),
                                            C.byref(st)))
    return torch.as_tensor(_CudaArray(fp.value, fb.value, "<i8", 8, st.value), device="cuda")


def allreduce_film_(tensor, group=None):
    """Sum an int64 film tensor over every rank in place (exact; any backend)."""
    import torch.distributed as dist
    if tensor.dtype.is_floating_point:
        raise TypeError("films are int64 fixed point; a float all-reduce would not be exact")
    dist.all_reduce(tensor, op=dist.ReduceOp.SUM, group=group)
    return tensor


def row_band(rank, world, height):
    """Contiguous [begin, end) of image rows owned by `rank`."""
    return photon_range(rank, world, height)


def tile_row_band(rank, world, height):
    """Contiguous [begin, end) of image rows owned by `rank` when bands are
    whole 8-row tile rows of the film (the last band ends at the height)."""
    tiles = (height + 7) // 8
    b, e = photon_range(rank, world, tiles)
    return min(8 * b, height), min(8 * e, height)


def gather_bands(band, rank, world, height, group=None, device="cpu", bands=row_band):
    """All-gather every rank's band of rows (band: rows x width x 3 float32, the
    rows bands(rank, world, height)) into the full image on every rank."""
    import torch
    import torch.distributed as dist
    band = np.ascontiguousarray(band, dtype=np.float32)
    width = band.shape[1]
    rows = max(e - b for b, e in (bands(r, world, height) for r in range(world)))
    pad = torch.zeros((rows, width, 3), dtype=torch.float32, device=device)
    pad[: band.shape[0]] = torch.from_numpy(band).to(device)
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    out = np.empty((height, width, 3), np.float32)
    for r, t in enumerate(parts):
        b, e = bands(r, world, height)
        out[b:e] = t[: e - b].cpu().numpy()
    return out


def trace_rows_sharded(tracer, spp, group=None):
    """Accumulate spp samples of this rank's band of rows on its GPU, then gather
    the bands: every rank returns the full mean XYZ image (height x width x 3)."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    w, h = tracer.dims()
    b, e = row_band(rank, world, h)
    tracer.set_rows(b, e)
    tracer.accumulate(spp)
    img = tracer.read_xyz().reshape(h, w, 3)
    device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    return gather_bands(img[b:e], rank, world, h, group, device)


def trace_sharded(film, n_photons, seed, group=None):
    """Trace this rank's share of photons [0, n_photons) into `film`, then sum the
    films of all ranks into every rank's film: an int64 all-reduce of the
    device film in place over NCCL, or through host memory on a host backend
    (gloo).  The film's tiles are then all marked lit (other ranks lit some of
    them), so its reduction reads every tile."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    b, e = photon_range(rank, world, n_photons)
    film.dispatch_photons(b, e, seed)
    t = film_tensor(film)
    check(lib.sc_ctx_synchronize(film.ctx.h))  # the trace, on the film's stream, is done
    if dist.get_backend(group) == "nccl":
        allreduce_film_(t, group)
    else:
        host = t.cpu()
        allreduce_film_(host, group)
        t.copy_(host)
    torch.cuda.synchronize()
    check(lib.sc_photon_film_mark_all_dirty(film.h))
    return film


# ---- the split without an all-reduce: bands reduced from peer films ---------

def ipc_export(ctx, ptr):
    """(64-byte CUDA IPC handle, offset) of the device allocation holding ptr."""
    h = (C.c_ubyte * 64)()
    off = C.c_size_t()
    check(lib.sc_ipc_export(ctx.h, C.c_void_p(ptr), h, C.byref(off)))
    return bytes(h), off.value


def ipc_import(ctx, handle, offset):
    """Device pointer of another process's allocation mapped into ctx."""
    h = (C.c_ubyte * 64).from_buffer_copy(handle)
    p = C.c_void_p()
    check(lib.sc_ipc_import(ctx.h, h, offset, C.byref(p)))
    return p.value


def ipc_close(ctx, ptr, offset):
    check(lib.sc_ipc_close(ctx.h, C.c_void_p(ptr), offset))


def reduce_band_peers(ctx, film_ptrs, width, height, channels, opts, row_begin, row_end, xyz_ptr, stream=None):
    """The sensor reduction of the sum of the films at film_ptrs (device
    pointers, rank order) for rows [row_begin, row_end) into the XYZ image at
    xyz_ptr (3 * width * height floats); opts: an sc_film_options (band, scale)."""
    arr = (C.c_void_p * len(film_ptrs))(*film_ptrs)
    check(lib.sc_sensor_reduce_peers(ctx.h, width, height, channels, opts.lambda_min, opts.lambda_max,
                                     opts.scale_log2, arr, len(film_ptrs), row_begin, row_end,
                                     C.c_void_p(xyz_ptr), C.c_void_p(stream)))


class PeerFilms:
    """Every rank's device film, mapped into this process in rank order: its
    own (an int64 torch tensor) and the other ranks' through CUDA IPC.  Built
    once (the films are reused every step); close() before the films go."""

    def __init__(self, ctx, film, group=None):
        import torch.distributed as dist
        self.ctx, self.film = ctx, film
        rank, world = dist.get_rank(group), dist.get_world_size(group)
        mine = ipc_export(ctx, film.data_ptr())
        allh = [None] * world
        dist.all_gather_object(allh, mine, group=group)
        self.ptrs, self._opened = [], []
        for r, (h, off) in enumerate(allh):
            if r == rank:
                self.ptrs.append(film.data_ptr())
            else:
                p = ipc_import(ctx, h, off)
                self.ptrs.append(p)
                self._opened.append((p, off))

    def close(self):
        for p, off in self._opened:
            ipc_close(self.ctx, p, off)
        self._opened = []


def reduce_sharded_peers(peers, width, height, channels, opts, group=None):
    """After every rank traced its photon range into its film: this rank reduces
    its band of whole tile rows from the sum of all the films (reading the
    peers' films in place), and the bands are gathered.  Every rank returns
    the full XYZ image (height x width x 3), bit-identical to the reduction of
    one film holding every photon.  Barriers on both sides: the films are
    complete before anyone reads them, and read before anyone reuses them."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    torch.cuda.synchronize()
    dist.barrier(group=group)  # every rank's trace is done
    b, e = tile_row_band(rank, world, height)
    xyz = torch.empty(3 * width * height, dtype=torch.float32, device="cuda")
    reduce_band_peers(peers.ctx, peers.ptrs, width, height, channels, opts, b, e, xyz.data_ptr(),
                      torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    dist.barrier(group=group)  # every rank has read the films
    band = xyz.view(height, width, 3)[b:e].cpu().numpy()
    device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    return gather_bands(band, rank, world, height, group, device, bands=tile_row_band)
