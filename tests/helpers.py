"""Shared test helpers: hand one scene to both the CUDA library and the oracle,
and the film metrics the reference's gates use."""
import ctypes as C

import numpy as np

import oracle
import spectral_b200 as sb


def oscene(scene):
    """Oracle copy of a product Scene (same flat record bytes)."""
    prims, np_, planes, npl, mats, nm = scene.arrays()
    return oracle.OScene(bytes(prims), np_, bytes(planes), npl, bytes(mats), nm, scene.background, scene.horizon)


def obeam(beam):
    return oracle.or_beam.from_buffer_copy(bytes(beam.c))


def ocam(cam):
    return oracle.or_camera.from_buffer_copy(bytes(cam.c))


def rel_l1(gpu, cpu):
    gpu = np.asarray(gpu, np.float64)
    cpu = np.asarray(cpu, np.float64)
    den = np.abs(cpu).sum()
    return float(np.abs(gpu - cpu).sum() / den) if den > 0 else 0.0


def energy_delta(gpu_xyz, cpu_xyz):
    gy = float(np.asarray(gpu_xyz, np.float64)[1::3].sum())
    cy = float(np.asarray(cpu_xyz, np.float64)[1::3].sum())
    return abs(gy - cy) / cy if cy > 0 else 0.0


def axis_box(lo, hi):
    """ConvexSolid::axis_box (spectral-core/src/geom.rs:73-84)."""
    return [((1, 0, 0), -hi[0]), ((-1, 0, 0), lo[0]), ((0, 1, 0), -hi[1]), ((0, -1, 0), lo[1]),
            ((0, 0, 1), -hi[2]), ((0, 0, -1), lo[2])]


def triangular_prism(size, depth):
    """ConvexSolid::triangular_prism (spectral-core/src/geom.rs:89-103), f32 trig."""
    out = []
    for k in range(3):
        ang = np.float32(np.float32(np.pi / 2) + np.float32(k) * np.float32(2.0) * np.float32(np.pi) / np.float32(3.0))
        out.append(((float(np.cos(ang)), float(np.sin(ang)), 0.0), -size))
    out += [((0, 0, 1), -depth / 2.0), ((0, 0, -1), -depth / 2.0)]
    return out


def wedge(apex_deg, size, depth):
    """ConvexSolid::wedge (spectral-core/src/geom.rs:110-121)."""
    a = np.float32(apex_deg) * np.float32(np.float32(np.pi) / np.float32(180.0))
    return [((-1, 0, 0), -size), ((float(np.cos(a)), float(np.sin(a)), 0.0), -size), ((0, -1, 0), -size),
            ((0, 0, 1), -depth / 2.0), ((0, 0, -1), -depth / 2.0)]


def dsotm_params(width, height, seed, **kw):
    return oracle.vol_params(width, height, seed, **kw)


def oracle_job_xyz(job):
    """Spectral film of one sc_scene_job on the CPU, sensor-reduced like the
    library (bin-averaged CMF, f64 sums, / 2^32)."""
    prims = bytes(job.prims)[:32 * job.n_prims]
    planes = bytes(job.planes)[:16 * job.n_planes]
    mats = bytes(job.mats)[:16 * job.n_mats]
    sc = oracle.OScene(prims, job.n_prims, planes, job.n_planes, mats, job.n_mats, 0.0)
    cam = oracle.or_camera.from_buffer_copy(bytes(job.cam))
    beam = oracle.or_beam.from_buffer_copy(bytes(job.beam))
    o = job.opts
    p = oracle.vol_params(job.width, job.height, job.seed, job.weights.sigma_s, job.weights.sigma_t, job.weights.g,
                          job.max_dist, o.max_bounces, o.lambda_min, o.lambda_max, spectral=job.spectral,
                          bins=o.bins, estimator=o.estimator)
    _, _, fs = oracle.render_point(sc, cam, beam, p, 0, job.n_photons, f32=False, xyz=False, spec=True)
    w = oracle.bin_weights(o.bins, o.lambda_min, o.lambda_max).astype(np.float64)
    return (fs.reshape(-1, o.bins).astype(np.float64) @ w.T).reshape(-1) * 2.0 ** -32


def device_desc(sb, _lib, torch, scene, cam, beam, w, h, seed, bins, keep, estimator=0, scale_log2=32):
    """An sc_trace_desc for the device-pointer entry points, its scene records
    copied to the device (the tensors are appended to `keep`)."""
    prims, np_, planes, npl, mats, nm = scene.arrays()

    def dev(arr, n, size):
        t = torch.frombuffer(bytearray(bytes(arr)[: n * size] or b"\0"), dtype=torch.uint8).cuda()
        keep.append(t)
        return t.data_ptr()

    opts = _lib.sc_film_options(bins, 380.0, 730.0, 8, scale_log2, estimator)
    w8 = sb.VolWeights()
    return _lib.sc_trace_desc(dev(prims, np_, 32), np_, dev(planes, npl, 16), npl, dev(mats, nm, 16), nm, cam.c,
                              beam.c, _lib.sc_vol_weights(w8.sigma_s, w8.sigma_t, w8.g), w, h, seed, 1, 14.0, opts,
                              None)
