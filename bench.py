#!/usr/bin/env python
"""Benchmarks of the B200 spectral forward / volumetric / camera-tracer path.

    python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]
                    [--workload batch|prism|rainbow|tracer|beam|serve]

Prints one JSON line (rank 0).  Workloads (seeded synthetic scenes):

* batch (default): 256 uneven prism scenes (glass, apex, incidence, photons
  2^14-2^22, film side 128-1024, 32 bins) in one persistent graph-captured
  launch plus one drain/reduce; compared with plain per-scene launches and
  with the per-scene film-object API.
* prism: one SF11 prism, 2^20 photons, 640x360x64-bin film.
* rainbow: a water sphere in a wide beam, 2^26 photons, 1920x1080x64 bins.
* tracer: the hero-wavelength camera tracer, 1280x720, 64 spp.
* beam: the photon-beam estimator on the DSOTM scene, 800x800.
* serve: a Poisson request stream replayed against the continuous-batching
  server and against plain per-request launches (latency p50/p99).

value is device-timed (CUDA events on the launching stream, max over ranks,
weak scaling: every rank renders its own work, no data-path collective); e2e
is the same metric through the public ABI with host buffers; roofline and
cpu_baseline as described in each line.  ``--impl reference`` times the
reference's CPU path (the oracle restatement of spectral-core, all host
threads) on the same workload; the reference itself is Rust + wgpu and cannot
be built or run here.
"""
import argparse
import ctypes as C
import datetime
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # Plain prism pass: SF11 prism (apex 60, side 1), 0.02 beam at 45 deg, 2^20
    # photons, lambda U(380, 780), sigma_s 0.05, sigma_a 0, isotropic, 640x360x64.
    "prism": dict(width=640, height=360, bins=64, photons=1 << 20, sigma_s=0.05, sigma_t=0.05, g=0.0,
                  lambda_min=380.0, lambda_max=780.0, max_dist=6.0, max_bounces=8, seed=0xDED),
    # Rainbow: water sphere r=1, beam width 2.2, 2^26 photons, up to 4
    # internal bounces (6 surface interactions), sigma_s 0.02, 1920x1080x64.
    "rainbow": dict(width=1920, height=1080, bins=64, photons=1 << 26, sigma_s=0.02, sigma_t=0.02, g=0.0,
                    lambda_min=380.0, lambda_max=780.0, max_dist=8.0, max_bounces=6, seed=0x8A1B),
    # Photon-beam estimator (render_volumetric_scene) on the Dark-Side-of-the-Moon
    # composition of spectral-core/examples/prism_dsotm.rs: 800x800 XYZ film,
    # sigma_s 0.5, sigma_t 0.06, g 0.5, max_dist 14, seed 0xDED; 2^18 photons
    # per step (the example traces 50 M in total).
    "beam": dict(width=800, height=800, bins=0, photons=1 << 18, sigma_s=0.5, sigma_t=0.06, g=0.5,
                 lambda_min=380.0, lambda_max=730.0, max_dist=14.0, max_bounces=8, seed=0xDED, scale_log2=40,
                 estimator=2),
}


METRIC_POINT = "photons/s @<=0.5% film err (forward + volumetric single scatter)"
METRIC_BEAM = "photons/s (forward + photon-beam estimator, volumetric single scatter)"

# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of each workload's
# roofline region, per launch (per step for the tracer and batch), from one
# ncu capture of the default workload on a B200 (the profile summaries give the
# commands); reported only when the workload runs at its default size.
NCU_TRAFFIC = {
    "prism": (2092544, "photon_kernel, one capture"),
    "rainbow": (4839725056, "order_count + order_scan + order_scatter + photon_kernel, one capture"),
    "beam": (3842560, "beam_kernel, one capture"),
    "tracer": (6145474816, "all tracer wave kernels of one accumulate(64), one capture"),
    "batch": (3953000000, "batch_kernel + reduce_scan + reduce_list, scaled from a capture of the first 64 "
                          "scenes (4.4 GB of films): batch_kernel by photons, reduce_scan by film bytes, reduce_list by "
                          "lit-tile bytes"),
    "atomics": (24887296, "synthetic_splat_kernel, one capture"),
}


# Warp instructions the dominant kernel issues per unit of work (photon or path
# sample), from one ncu capture of smsp__inst_executed.sum and
# smsp__thread_inst_executed.sum (a single-pass metric pair), with the lanes
# active per instruction: the instruction-issue roofline of kernels whose films
# stay in L2.
NCU_INST = {
    "batch": (12734972130 / 2 / 48957886, 21.77, "batch_kernel<0, 4, 0, 0>: two launches on the first 64 scenes "
                                                  "(48,957,886 photons each), per photon"),
    "prism": (324289908 / 2 / (1 << 20), 25.60, "photon_kernel: two launches of 2^20 photons, per photon"),
    "rainbow": (5568513387 / (1 << 26), 23.90, "photon_kernel: one launch of 2^26 photons, per photon"),
    "tracer": (3642531467 / 58982400, 27.66, "tr_shade, tr_tail, tr_accumulate: the 60 launches of one "
                                             "accumulate(64), per path sample"),
}


def issue_roofline(workload, units, seconds, sms, sm_mhz, default_size=True):
    """Warp instructions issued per second (from the captured count per unit)
    against the issue peak: one warp instruction per clock on each of an SM's
    four schedulers."""
    if not default_size or workload not in NCU_INST:
        return None
    per_unit, lanes, what = NCU_INST[workload]
    achieved = per_unit * units / seconds / 1e9
    peak = sms * 4 * sm_mhz * 1e6 / 1e9
    return {"achieved": achieved, "peak": peak, "unit": "G warp instructions/s", "frac": achieved / peak,
            "inst_per_unit": per_unit, "lanes_per_inst": lanes,
            "source": "ncu smsp__inst_executed.sum of %s" % what,
            "peak_source": "%d SMs x 4 schedulers x 1 instruction per clock x %.0f MHz (sampled median)"
                           % (sms, sm_mhz)}


def ncu_traffic(workload, default_size=True):
    if not default_size or workload not in NCU_TRAFFIC:
        return None, None
    b, what = NCU_TRAFFIC[workload]
    return b, "ncu dram__bytes_read.sum + dram__bytes_write.sum of %s" % what


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["atomics", "batch", "serve", "split", "tracer"],
                    default="batch")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample length")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=0, help="0: same as --steps")
    ap.add_argument("--scenes", type=int, default=0,
                    help="scenes of the batch workload (0: 256; the first N of the same seeded draw)")
    ap.add_argument("--photons", type=int, default=0,
                    help="photons per step for prism/rainbow/beam (0: the workload's; smaller for profiling)")
    ap.add_argument("--serve-seconds", type=float, default=60.0,
                    help="window of the 200 req/s Poisson stream replayed in real time for the served numbers "
                         "(batch and serve workloads; 0: none)")
    ap.add_argument("--split-exchange", choices=["allreduce", "peer"], default="allreduce",
                    help="split workload: sum the films with one NCCL all-reduce, or reduce each rank's band of "
                         "tile rows from every rank's film mapped as peer memory (CUDA IPC) and gather the bands")
    ap.add_argument("--tracer-chains", type=int, default=0,
                    help="tracer schedule: waves in flight (0: the library's default, 3)")
    ap.add_argument("--tracer-wave-log2", type=int, default=0,
                    help="tracer schedule: paths per wave 2^k (0: the library's default, 22)")
    ap.add_argument("--tracer-wave-bounces", type=int, default=0,
                    help="tracer schedule: compacted bounces before the tail (0: the library's default, 2)")
    return ap.parse_args()


def build_scene(wl):
    import spectral_b200 as sb
    from spectral_b200.scenes import prism_workload, rainbow_workload
    cfg = WORKLOADS[wl]
    if wl == "prism":
        return prism_workload(cfg["width"], cfg["height"])
    if wl == "beam":
        return sb.dsotm_scene(cfg["width"] / cfg["height"])
    return rainbow_workload(cfg["width"], cfg["height"])


def load_specs():
    """spectral_b200/specs.py loaded by file path: the workload descriptions in
    plain Python, so that the CPU legs never load the CUDA library."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("spectral_specs", os.path.join(ROOT, "spectral_b200", "specs.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def oracle_scene(d, aspect):
    """(OScene, or_beam or None, or_camera) of a specs scene dict, in the record
    order the library's Scene flattens it (solids, then spheres)."""
    import oracle
    prims, planes, mats = [], [], []

    def mat(m):
        mats.append(oracle.or_mat(0.0, m[1], 1, 0) if m[0] == "glass" else oracle.or_mat(m[1], 0, 0, 0))
        return len(mats) - 1
    for pl, m in d["solids"]:
        start = len(planes)
        planes.extend(oracle.or_plane(oracle.F3(*n), dd) for n, dd in pl)
        prims.append(oracle.or_prim(oracle.F3(0.0, 0.0, 0.0), 0.0, start, len(pl), 1, mat(m)))
    for c, r, m in d["spheres"]:
        prims.append(oracle.or_prim(oracle.F3(*c), r, 0, 0, 0, mat(m)))
    sc = oracle.OScene(b"".join(bytes(x) for x in prims), len(prims), b"".join(bytes(x) for x in planes), len(planes),
                       b"".join(bytes(x) for x in mats), len(mats), 0.0)
    beam = oracle.or_beam(*[oracle.F3(*v) for v in d["beam"]]) if "beam" in d else None
    o, t, up, vfov = d["camera"]
    return sc, beam, oracle.camera_look_at(o, t, up, vfov, aspect)


def oracle_scene_of(wl):
    cfg = WORKLOADS[wl]
    specs = load_specs()
    d = {"prism": specs.prism_scene, "beam": specs.dsotm_scene, "rainbow": specs.rainbow_scene}[wl]()
    return oracle_scene(d, cfg["width"] / cfg["height"])


def oracle_prism_job(spec):
    """(OScene, or_camera, or_beam, or_vol_params) of a prism job dict (the
    sc_scene_job that spectral_b200.batch.job_from_spec makes of it)."""
    import oracle
    specs = load_specs()
    d = dict(solids=[(specs.prism_planes(spec["apex_deg"], 1.0, 1.0), ("glass", spec["glass"]))], spheres=[],
             beam=specs.prism_beam(spec["apex_deg"], 1.0, spec["incidence_deg"], 0.02), camera=specs.PRISM_CAMERA)
    sc, beam, cam = oracle_scene(d, spec["width"] / spec["height"])
    p = oracle.vol_params(spec["width"], spec["height"], spec["seed"], spec["sigma_s"], spec["sigma_t"], spec["g"],
                          6.0, 8, spec["lambda_min"], spec["lambda_max"], bins=spec["bins"])
    return sc, cam, beam, p


# ----------------------------------------------------------------------------
# CPU reference arm / baseline: the oracle's point estimator on all host cores
# ----------------------------------------------------------------------------
def run_cpu(wl, seconds, threads=None):
    """Photons/s of the CPU restatement on a bounded sample of the workload."""
    import oracle
    cfg = WORKLOADS[wl]
    osc, ob, oc = oracle_scene_of(wl)
    # the reference's XYZ film (per-thread int64 XYZ films merged exactly): a
    # 64-bin film per host thread would cost more to clear and merge than to trace
    p = oracle.vol_params(cfg["width"], cfg["height"], cfg["seed"], cfg["sigma_s"], cfg["sigma_t"], cfg["g"],
                          cfg["max_dist"], cfg["max_bounces"], cfg["lambda_min"], cfg["lambda_max"], bins=0)
    threads = threads or os.cpu_count() or 1
    if cfg.get("estimator", 0) == 2:
        # render_volumetric_scene: photon ranges on all host threads (ctypes
        # releases the GIL), one f32 image per thread as the reference's loop
        import concurrent.futures as cf
        imgs = [np.zeros(3 * cfg["width"] * cfg["height"], np.float32) for _ in range(threads)]

        def render(n):
            def part(i):
                lo, hi = n * i // threads, n * (i + 1) // threads
                oracle.lib.or_render_beam(C.byref(osc.c), C.byref(oc), C.byref(ob), C.byref(p), None, lo, hi,
                                          oracle.fp(imgs[i]))
            with cf.ThreadPoolExecutor(threads) as ex:
                list(ex.map(part, range(threads)))
    else:
        film = np.zeros(cfg["width"] * cfg["height"] * 3, np.int64)
        fp = film.ctypes.data_as(C.POINTER(C.c_int64))

        def render(n):
            oracle.lib.or_render_point_mt(C.byref(osc.c), C.byref(oc), C.byref(ob), C.byref(p), None, 0, n, fp,
                                          None, threads)
    # calibrate on a small sample, then size the timed sample to ~`seconds`
    n = 64 if cfg.get("estimator", 0) == 2 else 4096
    while True:
        t0 = time.perf_counter()
        render(n)
        dt = time.perf_counter() - t0
        if dt > 0.5 or n >= cfg["photons"]:
            break
        n *= 4
    n_s = int(min(cfg["photons"], max(n, n * seconds / max(dt, 1e-6))))
    # a whole step that ends early is repeated until ~`seconds` of work
    done, t0 = 0, time.perf_counter()
    while True:
        render(n_s)
        done += n_s
        dt = time.perf_counter() - t0
        if dt >= 0.8 * seconds or n_s < cfg["photons"]:
            break
    return done / dt, done, dt, threads


def cpu_serial(wl, seconds):
    """The restatement on ONE host thread, as the reference's serial photon loop
    (spectral-core/src/volume.rs:118): photons/s on a shorter sample."""
    rate, n_s, dt, _ = run_cpu(wl, max(1.0, seconds / 4), threads=1)
    return {"value": rate, "unit": "photons/s", "cores": 1,
            "sample": "%d photons from photon 0 on one thread, %.1f s" % (n_s, dt)}


def cpu_model():
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ----------------------------------------------------------------------------
# clocks during the timed region
# ----------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.uuid, self.proc, self.lines = uuid, None, []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.uuid, "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nme, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nme)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


# ----------------------------------------------------------------------------
# GPU arm
# ----------------------------------------------------------------------------
# Photons of the film-error sample per workload (the oracle's share of the run)
FILM_ERR_PHOTONS = {"prism": 1 << 20, "rainbow": 1 << 22, "beam": 1 << 12}


def rel_l1(got, ref):
    got, ref = np.asarray(got, np.float64), np.asarray(ref, np.float64)
    den = float(np.abs(ref).sum())
    return float(np.abs(got - ref).sum() / den) if den > 0 else 0.0


def oracle_xyz_from_spectral(fs, bins, lambda_min, lambda_max, scale_log2=32):
    """The library's sensor reduction on the host: spectral int64 film times the
    bin-averaged CMF (f64), / 2^scale."""
    import oracle
    w = oracle.bin_weights(bins, lambda_min, lambda_max).astype(np.float64)
    return (fs.reshape(-1, bins).astype(np.float64) @ w.T).reshape(-1) * 2.0 ** -scale_log2


def single_scene_film_err(wl, scene, beam, cam, cfg, n, gpu_xyz):
    """Relative L1 of a GPU XYZ image of photons [0, n) against the oracle's
    image of the same photons (the checker; never timed)."""
    import oracle
    prims, np_, planes, npl, mats, nm = scene.arrays()
    osc = oracle.OScene(bytes(prims), np_, bytes(planes), npl, bytes(mats), nm, scene.background)
    ob = oracle.or_beam.from_buffer_copy(bytes(beam.c))
    oc = oracle.or_camera.from_buffer_copy(bytes(cam.c))
    W, H, B = cfg["width"], cfg["height"], cfg["bins"]
    p = oracle.vol_params(W, H, cfg["seed"], cfg["sigma_s"], cfg["sigma_t"], cfg["g"], cfg["max_dist"],
                          cfg["max_bounces"], cfg["lambda_min"], cfg["lambda_max"], bins=B,
                          scale_log2=cfg.get("scale_log2", 32), estimator=cfg.get("estimator", 0))
    if cfg.get("estimator", 0) == 2:
        ref = oracle.render_beam(osc, oc, ob, p, 0, n)
    else:
        threads = max(1, min(os.cpu_count() or 1, 16 if W * H * max(B, 3) <= (1 << 24) else 4))
        _, _, fs = oracle.render_point(osc, oc, ob, p, 0, n, f32=False, xyz=False, spec=True, threads=threads)
        ref = oracle_xyz_from_spectral(fs, B, cfg["lambda_min"], cfg["lambda_max"], cfg.get("scale_log2", 32))
    return rel_l1(gpu_xyz, ref)


def run_gpu(args, rank, world, local_rank):
    import torch
    import spectral_b200 as sb
    from spectral_b200 import _lib
    dist = None
    if world > 1:
        import torch.distributed as dist
    cfg = dict(WORKLOADS[args.workload])
    if args.photons:
        cfg["photons"] = args.photons
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    ctx = sb.GpuContext(local_rank)
    scene, beam, cam = build_scene(args.workload)
    W, H, B, N = cfg["width"], cfg["height"], cfg["bins"], cfg["photons"]
    CH = B or 3  # film channels: spectral bins, or the reference's XYZ film
    SCALE, EST = cfg.get("scale_log2", 32), cfg.get("estimator", 0)
    prims, np_, planes, npl, mats, nm = scene.arrays()

    def dev_bytes(obj, n):
        t = torch.frombuffer(bytearray(bytes(obj)[: n * C.sizeof(obj._type_)] or b"\0"), dtype=torch.uint8).to(dev)
        return t

    d_prims, d_planes, d_mats = dev_bytes(prims, np_), dev_bytes(planes, npl), dev_bytes(mats, nm)
    opts = _lib.sc_film_options(B, cfg["lambda_min"], cfg["lambda_max"], cfg["max_bounces"], SCALE, EST)
    desc = _lib.sc_trace_desc(d_prims.data_ptr(), np_, d_planes.data_ptr(), npl, d_mats.data_ptr(), nm, cam.c, beam.c,
                              _lib.sc_vol_weights(cfg["sigma_s"], cfg["sigma_t"], cfg["g"]), W, H, cfg["seed"], 1,
                              cfg["max_dist"], opts, None)
    film = torch.zeros(_lib.lib.sc_film_bytes(W, H, CH) // 8, dtype=torch.int64, device=dev)
    flags = torch.zeros(_lib.lib.sc_film_flag_bytes(W, H) // 4, dtype=torch.int32, device=dev)
    xyz = torch.empty(3 * W * H, dtype=torch.float32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2
    stream = torch.cuda.current_stream(dev)
    sp = C.c_void_p(stream.cuda_stream)
    base = rank * N

    def trace():
        _lib.check(_lib.lib.sc_trace_photons_device(ctx.h, C.byref(desc), base, N, C.c_void_p(film.data_ptr()),
                                                    C.c_void_p(flags.data_ptr()), sp))

    def reduce():
        _lib.check(_lib.lib.sc_sensor_reduce_device(ctx.h, W, H, CH, cfg["lambda_min"], cfg["lambda_max"], SCALE,
                                                    C.c_void_p(film.data_ptr()), C.c_void_p(flags.data_ptr()),
                                                    C.c_void_p(xyz.data_ptr()), 1, sp))

    # algorithmic work of one launch (instrumented pass, outside the timed region)
    stats = torch.zeros(5, dtype=torch.int64, device=dev)
    _lib.check(_lib.lib.sc_trace_stats_device(ctx.h, C.byref(desc), base, N, C.c_void_p(stats.data_ptr()), sp))
    if EST == 2:  # photons, segments, march steps, in-frame steps, footprint deposits
        photons, segments, steps, in_frame, deposits = [int(x) for x in stats.cpu()]
        splats, scatters = deposits, 0
    else:
        photons, segments, splats, scatters = [int(x) for x in stats.cpu()[:4]]

    for _ in range(args.warmup):
        trace()
        reduce()
    # lit tiles of one pass (the drain reads and zeroes only those)
    trace()
    torch.cuda.synchronize()
    dirty_tiles = int(np.unpackbits(flags.cpu().numpy().view(np.uint8)).sum())
    reduce()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    with ClockSampler(uuid) as clk, torch.cuda.nvtx.range("timed"):  # nvtx range for ncu --nvtx-include
        for k in range(args.steps):
            flush.zero_()  # evict the film from L2 between steps (outside the events)
            ev[k][0].record(stream)
            trace()
            ev[k][1].record(stream)
            reduce()
            ev[k][2].record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms = [ev[k][0].elapsed_time(ev[k][2]) for k in range(args.steps)]
    trace_ms = [ev[k][0].elapsed_time(ev[k][1]) for k in range(args.steps)]
    reduce_ms = [ev[k][1].elapsed_time(ev[k][2]) for k in range(args.steps)]
    total_ms = sum(step_ms)
    if dist:
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = N * world * args.steps / (total_ms / 1e3)

    # film error against the oracle (outside the timed region): a prefix of
    # the workload's photons through the same device path, trace + reduce
    n_chk = min(N, FILM_ERR_PHOTONS[args.workload])
    film.zero_()
    flags.zero_()
    _lib.check(_lib.lib.sc_trace_photons_device(ctx.h, C.byref(desc), 0, n_chk, C.c_void_p(film.data_ptr()),
                                                C.c_void_p(flags.data_ptr()), sp))
    reduce()
    torch.cuda.synchronize()
    film_err = None
    if rank == 0:
        err = single_scene_film_err(args.workload, scene, beam, cam, cfg, n_chk, xyz.cpu().numpy())
        film_err = {"value": err, "bar": 5e-3, "photons": n_chk,
                    "sample": "photons [0, %d) of the workload (%s), GPU XYZ image vs the oracle's film%s"
                              % (n_chk, "all of them" if n_chk == N else "a prefix",
                                 " reduced by the bin-averaged CMF on the host" if B else "")}

    # end to end through the GpuPhotonFilm-shaped ABI object with host buffers
    e2e_steps = args.e2e_steps or args.steps
    pf = sb.GpuPhotonFilm(ctx, scene, cam, beam, W, H, N, cfg["seed"], cfg["max_dist"],
                          sb.VolWeights(cfg["sigma_s"], cfg["sigma_t"], cfg["g"]), bins=B,
                          lambda_min=cfg["lambda_min"], lambda_max=cfg["lambda_max"],
                          max_bounces=cfg["max_bounces"], scale_log2=SCALE, estimator=EST)
    host_xyz = torch.empty(3 * W * H, dtype=torch.float32, pin_memory=True).numpy()  # pinned read-back buffer
    h2d = C.sizeof(prims._type_) * np_ + C.sizeof(planes._type_) * npl + C.sizeof(mats._type_) * nm + \
        C.sizeof(cam.c) + C.sizeof(beam.c)

    def e2e_step():
        _lib.check(_lib.lib.sc_photon_film_set_scene(pf.h, prims, np_, planes, npl, mats, nm, C.byref(cam.c),
                                                     C.byref(beam.c)))
        _lib.check(_lib.lib.sc_photon_film_dispatch(pf.h, base, base + N, cfg["seed"]))
        _lib.check(_lib.lib.sc_photon_film_read_accum(pf.h, host_xyz.ctypes.data_as(C.POINTER(C.c_float))))
        _lib.check(_lib.lib.sc_photon_film_clear(pf.h))

    for _ in range(max(1, args.warmup)):
        e2e_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = N * world * e2e_steps / e2e_s
    pf.close()

    if rank != 0:
        return None

    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs")
    peak_note = "measured" if hbm else "fallback"
    hbm = hbm or 6650.0
    trace_s = statistics.mean(trace_ms) / 1e3
    reduce_s = statistics.mean(reduce_ms) / 1e3
    cl = clk.summary()
    sm_mhz = cl["sm_mhz"] or peaks.get("sm_max_mhz", 1965.0)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    fp32_peak = sms * 128 * 2 * sm_mhz * 1e6 / 1e12  # TFLOP/s at the sampled clock
    if EST == 2:
        # beam kernel: 8 B per film channel per footprint pixel deposited;
        # counted FP32 work: emission 20, intersect 14 per plane per segment,
        # 100 per in-frame march step (two projections, weight, radius), 16
        # per footprint pixel (two tent evaluations), 45 per scatter (segments
        # minus photons)
        kname = "beam_kernel"
        alg_bytes = deposits * 8 * CH
        alg_note = "8 B x %d channels per footprint pixel: %d deposits per launch" % (CH, deposits)
        flops = photons * 20 + segments * 14 * npl + in_frame * 100 + deposits * 16 + (segments - photons) * 45
    else:
        # photon kernel: one 8-byte fixed-point payload per in-frame haze
        # sample (its film atomic); counted FP32 work (exp/pow one op each):
        # emission 20, intersect 14 per plane per segment, 60 per haze sample,
        # 45 per scatter
        kname = "photon_kernel"
        alg_bytes = splats * 8 * (1 if B else 3)
        alg_note = "8 B per film channel per in-frame haze sample: %d samples per launch" % splats
        flops = photons * 20 + segments * 14 * npl + segments * 4 * 60 + scatters * 45
    lit_bytes = dirty_tiles * 64 * CH * 8
    # the library traces photons in film-bin order when a spectral film is larger than L2
    film_bytes = ((W + 7) // 8) * ((H + 7) // 8) * 64 * CH * 8
    ordered = (EST != 2 and B > 0 and N >= (1 << 16) and os.environ.get("SPECTRAL_CUDA_ORDER", "1") != "0"
               and film_bytes > torch.cuda.get_device_properties(dev).L2_cache_size)
    traffic, traffic_src = ncu_traffic(args.workload, not args.photons)
    workload_txt = {"prism": "SF11 prism apex 60 side 1, beam 0.02 @45deg, 2^20 photons, 640x360x64 bins",
                    "rainbow": "water sphere r=1, beam 2.2, 2^26 photons, 1920x1080x64 bins",
                    "beam": "photon-beam estimator, DSOTM prism scene, 2^18 photons, 800x800 XYZ film"}
    line = {
        "metric": METRIC_BEAM if EST == 2 else METRIC_POINT,
        "value": value, "unit": "photons/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 transport, int64 fixed-point film", "data": "synthetic (seeded scene)",
        "config": {"workload": "%s: %s%s" % (args.workload, workload_txt[args.workload],
                                             " [photons per step overridden: %d]" % N if args.photons else ""),
                   "photons_per_step": N * world, "film": [W, H, B], "band_nm": [cfg["lambda_min"], cfg["lambda_max"]],
                   "l2": "flushed between steps (256 MB write outside the timed events)",
                   "parallelism": "photon ranges per rank, no collective"},
        "e2e": {"value": e2e_value, "unit": "photons/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": 3 * W * H * 4,
                "path": "sc_photon_film_set_scene + dispatch + read_accum (host f32 XYZ) + clear"},
        # per step: the trace (3 wavelength-sort kernels first when ordered) and the drain
        "gpu_launches": args.steps * (2 + (3 if ordered else 0)),
        "kernels": {"trace_ms": statistics.mean(trace_ms), "reduce_ms": statistics.mean(reduce_ms),
                    "wavelength_ordered": ordered},
        "roofline": {"bound": "hbm", "achieved": alg_bytes / trace_s / 1e9, "peak": hbm, "unit": "GB/s",
                     "frac": alg_bytes / trace_s / 1e9 / hbm, "traffic": traffic, "traffic_source": traffic_src,
                     "kernel": kname + (" (after its wavelength sort)" if ordered else ""),
                     "peak_source": "%s hbm_gbs" % peak_note, "algorithmic": alg_note},
        "roofline_fp32": {"kernel": kname, "counted_flops": flops, "achieved_tflops": flops / trace_s / 1e12,
                          "peak_tflops": fp32_peak, "frac": flops / trace_s / 1e12 / fp32_peak,
                          "peak_source": "%d SMs x 128 FP32 lanes x 2 x %.0f MHz (sampled median)" % (sms, sm_mhz)},
        "roofline_issue": issue_roofline(args.workload, N, trace_s, sms, sm_mhz, not args.photons),
        "roofline_reduce": {"kernel": "reduce_kernel (drain)", "bound": "hbm",
                            "achieved": (2 * lit_bytes + 12 * W * H) / reduce_s / 1e9, "peak": hbm, "unit": "GB/s",
                            "frac": (2 * lit_bytes + 12 * W * H) / reduce_s / 1e9 / hbm,
                            "algorithmic": "read + zero the %d lit 8x8 tiles (%d B) + 12 B XYZ per pixel"
                                           % (dirty_tiles, lit_bytes)},
        "film_err": film_err,
        "work": ({"photons": photons, "segments": segments, "march_steps": steps, "in_frame_steps": in_frame,
                  "footprint_deposits": deposits} if EST == 2 else
                 {"photons": photons, "segments": segments, "in_frame_samples": splats, "scatters": scatters}),
        "clocks": cl,
    }
    if world == 1 and not args.no_cpu_baseline:
        rate, n_s, dt, th = run_cpu(args.workload, args.cpu_seconds)
        line["cpu_baseline"] = {"value": rate, "unit": "photons/s", "cores": th, "kind": "port",
                                "sample": "%d photons of the workload from photon 0 (whole steps repeated), %.1f s, %s"
                                          % (n_s, dt, cpu_model()),
                                "serial": cpu_serial(args.workload, args.cpu_seconds)}
    return line


# Camera-tracer workload: SF11 prism on a diffuse ground plane,
# spherical D65 emitter r=0.2 at (2,3,1), 1280x720, 64 spp per step, hero comb
# of 4 wavelengths, depth 8, Russian roulette after bounce 3.
TRACER = dict(width=1280, height=720, spp=64, seed=0x7ACE)
TRACER_WAVE_PATHS = 1 << 22  # paths per wavefront wave (the library's default queue size per chain)


def run_cpu_tracer(seconds, threads=None):
    """Path samples/s of the CPU restatement of CpuTracer (pixel-parallel, as
    the reference's rayon loop) with the emitter / roulette extensions, on
    whole frames at 1 spp until ~`seconds` of work."""
    import oracle
    W, H = TRACER["width"], TRACER["height"]
    d = load_specs().tracer_scene()
    osc, _, oc = oracle_scene(d, W / H)
    kw = d["tracer"]
    c, r, sc = kw["emitter"]
    ext = oracle.or_tracer_ext(oracle.F3(*c), r, sc, kw["rr_start"])
    threads = threads or os.cpu_count() or 1
    out = np.zeros(3 * W * H, np.float32)
    oracle.lib.or_tracer_set_ext(C.byref(ext))
    try:
        frames, t0 = 0, time.perf_counter()
        while True:
            oracle.lib.or_tracer_accumulate_mt(C.byref(osc.c), C.byref(oc), W, H, 0, TRACER["seed"], 1, frames,
                                               kw["max_depth"], oracle.fp(out), threads)
            frames += 1
            dt = time.perf_counter() - t0
            if dt >= seconds:
                break
    finally:
        oracle.lib.or_tracer_set_ext(None)
    return W * H * frames / dt, frames, dt, threads


def run_gpu_tracer(args, rank, world, local_rank):
    import torch
    import spectral_b200 as sb
    from spectral_b200 import _lib
    from spectral_b200.scenes import tracer_workload
    dist = None
    if world > 1:
        import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    ctx = sb.GpuContext(local_rank)
    W, H, SPP = TRACER["width"], TRACER["height"], TRACER["spp"]
    scene, cam, kw = tracer_workload(W, H)
    seed = TRACER["seed"] + rank  # each rank: its own independent 64-spp frame
    sched = dict(chains=args.tracer_chains, wave_paths_log2=args.tracer_wave_log2,
                 wave_bounces=args.tracer_wave_bounces)  # scheduling only: the image is the same
    tr = sb.GpuTracer(ctx, scene, cam, W, H, sb.D65, seed, **sched, **kw)
    sp = C.c_void_p()
    _lib.check(_lib.lib.sc_tracer_stream(tr.h, C.byref(sp)))
    st = torch.cuda.ExternalStream(sp.value, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        tr.accumulate(SPP)
    torch.cuda.synchronize()
    _, seg0 = tr.stats()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)]
    uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    with ClockSampler(uuid) as clk, torch.cuda.nvtx.range("timed"):  # nvtx range for ncu --nvtx-include
        for k in range(args.steps):
            with torch.cuda.stream(st):
                flush.zero_()  # evict queues and accumulators from L2 (outside the events)
            ev[k][0].record(st)
            tr.accumulate(SPP)
            ev[k][1].record(st)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms = [ev[k][0].elapsed_time(ev[k][1]) for k in range(args.steps)]
    total_ms = sum(step_ms)
    if dist:
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    paths, seg1 = tr.stats()
    segments = (seg1 - seg0) // args.steps
    samples = W * H * SPP
    value = samples * world * args.steps / (total_ms / 1e3)

    # end to end through the GpuTracer-shaped ABI object with host buffers: a new
    # camera, clear, 64 spp, mean XYZ back to the host, every step
    host = torch.empty(3 * W * H, dtype=torch.float32, pin_memory=True).numpy()  # pinned read-back buffer
    e2e_steps = args.e2e_steps or args.steps

    def e2e_step():
        tr.set_camera(cam)
        tr.clear_accum()
        tr.accumulate(SPP)
        _lib.check(_lib.lib.sc_tracer_read_xyz(tr.h, host.ctypes.data_as(C.POINTER(C.c_float))))

    for _ in range(max(1, args.warmup)):
        e2e_step()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = samples * world * e2e_steps / e2e_s
    tr.close()
    if rank != 0:
        return None

    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs")
    peak_note = "measured" if hbm else "fallback"
    hbm = hbm or 6650.0
    step_s = statistics.mean(step_ms) / 1e3
    cl = clk.summary()
    sm_mhz = cl["sm_mhz"] or peaks.get("sm_max_mhz", 1965.0)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    fp32_peak = sms * 128 * 2 * sm_mhz * 1e6 / 1e12
    n_planes = len(scene.planes)
    # counted FP32 work per path segment: 14 per plane (intersection), 20 for the
    # emitter sphere test, 60 for the shading step (Fresnel / refraction or
    # cosine sampling, 4-lane throughput and radiance update)
    flops = segments * (14 * n_planes + 20 + 60)
    # wavefront queue traffic: per segment after the first (the first bounce
    # makes its rays in place), the path state (44 B) written by the bounce
    # before and read by the one that intersects and shades it; per path, its
    # XYZ (12 B) written and read by the per-pixel sums
    qbytes = (segments - samples) * 2 * 44 + samples * 2 * 12
    wave_paths = 1 << args.tracer_wave_log2 if args.tracer_wave_log2 else TRACER_WAVE_PATHS
    wb = args.tracer_wave_bounces or 2
    waves = -(-(W * H) // max(1, wave_paths // SPP))
    line = {
        "metric": "path samples/s (hero-wavelength camera tracer, 4 lanes, depth 8)",
        "value": value, "unit": "samples/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene)",
        "config": {"workload": "tracer: SF11 prism on a diffuse ground (albedo 0.8), D65 sphere emitter r=0.2 at "
                               "(2,3,1), 1280x720, 64 spp, depth 8, roulette after bounce 3",
                   "samples_per_step": samples * world, "l2": "flushed between steps (256 MB write outside the events)",
                   "schedule": {"chains": args.tracer_chains or 3, "wave_paths": wave_paths, "wave_bounces": wb},
                   "parallelism": "independent frames per rank (own seed), no collective"},
        "e2e": {"value": e2e_value, "unit": "samples/s", "h2d_bytes_per_step": C.sizeof(cam.c),
                "d2h_bytes_per_step": 3 * W * H * 4,
                "path": "sc_tracer_set_camera + clear_accum + accumulate(64) + read_xyz (host f32 XYZ)"},
        # per wave: two shades (the first makes and intersects the primary rays
        # and intersects the second bounce's rays), the tail, per-pixel sums
        "gpu_launches": args.steps * waves * (min(kw["max_depth"], wb) + (1 if kw["max_depth"] > wb else 0) + 1),
        "kernels": {"accumulate_ms": statistics.mean(step_ms)},
        "roofline": {"bound": "hbm", "achieved": qbytes / step_s / 1e9, "peak": hbm, "unit": "GB/s",
                     "frac": qbytes / step_s / 1e9 / hbm, "traffic": ncu_traffic("tracer")[0],
                     "traffic_source": ncu_traffic("tracer")[1], "kernel": "tracer wave kernels (one accumulate)",
                     "peak_source": "%s hbm_gbs" % peak_note,
                     "algorithmic": "wavefront queue bytes: 88 B of path state per path segment after the first "
                                    "bounce, 24 B of XYZ per path (%d segments, %d paths per step)" % (segments, samples)},
        "roofline_fp32": {"kernel": "tr_intersect + tr_shade", "counted_flops": flops,
                          "achieved_tflops": flops / step_s / 1e12, "peak_tflops": fp32_peak,
                          "frac": flops / step_s / 1e12 / fp32_peak,
                          "peak_source": "%d SMs x 128 FP32 lanes x 2 x %.0f MHz (sampled median)" % (sms, sm_mhz)},
        "roofline_issue": issue_roofline("tracer", samples, step_s, sms, sm_mhz),
        "work": {"paths": samples, "segments": segments},
        "clocks": cl,
    }
    if world == 1 and not args.no_cpu_baseline:
        rate, frames, dt, th = run_cpu_tracer(args.cpu_seconds)
        line["cpu_baseline"] = {"value": rate, "unit": "samples/s", "cores": th, "kind": "port",
                                "sample": "%d frames of 1280x720 at 1 spp (%.1f s), %s" % (frames, dt, cpu_model())}
    return line


# Atomic-throughput workload: the AtomicFilm synthetic splat (vol_splat.wgsl
# semantics: random pixel, three u32 atomics x4096), 2^24 splats per step into a
# 1920x1080 film that stays in L2 -- the in-project measure of L2 atomic
# throughput, the ceiling of the splat kernels' film atomics.
ATOMICS = dict(width=1920, height=1080, splats=1 << 24, seed=0xA70)


def run_gpu_atomics(args, rank, world, local_rank):
    import torch
    import spectral_b200 as sb
    from spectral_b200 import _lib
    dist = None
    if world > 1:
        import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    ctx = sb.GpuContext(local_rank)
    W, H, N = ATOMICS["width"], ATOMICS["height"], ATOMICS["splats"]
    f = sb.AtomicFilm(ctx, W, H)
    sp = C.c_void_p()
    _lib.check(_lib.lib.sc_atomic_film_stream(f.h, C.byref(sp)))
    st = torch.cuda.ExternalStream(sp.value, device=dev)
    for k in range(args.warmup):
        f.splat(ATOMICS["seed"] + k, N)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)]
    uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    with ClockSampler(uuid) as clk, torch.cuda.nvtx.range("timed"):  # nvtx range for ncu --nvtx-include
        for k in range(args.steps):
            ev[k][0].record(st)
            f.splat(ATOMICS["seed"] + 1000 + k, N)
            ev[k][1].record(st)
        torch.cuda.synchronize()
    total_ms = sum(ev[k][0].elapsed_time(ev[k][1]) for k in range(args.steps))
    if dist:
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    atomics = 3 * N
    value = atomics * world * args.steps / (total_ms / 1e3)
    # end to end: splat, then the raw film back to the host, every step
    e2e_steps = args.e2e_steps or args.steps
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        f.splat(ATOMICS["seed"] + 2000 + k, N)
        f.read_film_raw()
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    f.close()
    if rank != 0:
        return None
    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs") or 6650.0
    step_s = total_ms / args.steps / 1e3
    line = {
        "metric": "L2 atomic throughput, u32 atomicAdd (AtomicFilm synthetic splat)",
        "value": value, "unit": "atomics/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32", "data": "synthetic (seeded splats)",
        "config": {"workload": "atomics: %d splats x 3 u32 atomics per step into a %dx%d film (resident in L2)"
                               % (N, W, H), "parallelism": "own film per rank, no collective"},
        "e2e": {"value": atomics * world * e2e_steps / e2e_s, "unit": "atomics/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 3 * W * H * 4,
                "path": "sc_atomic_film_splat + sc_atomic_film_read_raw (host u32 film)"},
        "gpu_launches": args.steps,
        "roofline": {"bound": "hbm", "achieved": atomics * 4 / step_s / 1e9, "peak": hbm, "unit": "GB/s",
                     "frac": atomics * 4 / step_s / 1e9 / hbm, "traffic": ncu_traffic("atomics")[0],
                     "traffic_source": ncu_traffic("atomics")[1], "kernel": "synthetic_splat_kernel",
                     "peak_source": "measured hbm_gbs" if peaks.get("hbm_gbs") else "fallback",
                     "algorithmic": "4 B payload per atomic (the film stays in L2: this is the L2 atomic rate)"},
        "clocks": clk.summary(),
    }
    if not args.no_cpu_baseline:
        rate, done, dt = run_cpu_atomics(min(args.cpu_seconds, 5.0))
        line["cpu_baseline"] = {"value": rate, "unit": "atomics/s", "cores": 1, "kind": "port",
                                "sample": "%d x 2^20 splats on one host thread (%.1f s), %s" % (done, dt, cpu_model())}
    return line


def run_cpu_atomics(seconds):
    """Atomics/s of the CPU restatement of the synthetic splat (serial, as the
    film it restates is one buffer), over batches of 2^20 splats."""
    import oracle
    W, H = ATOMICS["width"], ATOMICS["height"]
    film = np.zeros(3 * W * H, np.uint32)
    n_cpu, done, t0 = 1 << 20, 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        oracle.lib.or_synthetic_splat(W, H, ATOMICS["seed"] + done, n_cpu, film.ctypes.data_as(C.POINTER(C.c_uint32)))
        done += 1
    dt = time.perf_counter() - t0
    return 3 * n_cpu * done / dt, done, dt


# Serving workload: Poisson arrivals at 200 req/s (a 15 s window of
# the 60 s stream by default), prism scenes of the batch workload's distribution,
# 2^16-2^20 photons per frame, 30 % orbit sessions of 16-128 frames at 2 deg
# per frame, 40 GB HBM budget.
SERVE = dict(rate=200.0, budget_gb=40.0, seed=0x5E7E, sample_s=3.0)


def served_summary(ctx, seconds, rank, clk=None):
    """The serving numbers of the config-5 stream: a `seconds` window of the
    200 req/s Poisson stream replayed in real time against the continuous-
    batching server (latency from arrival to the XYZ image in host memory),
    then the stream's first SERVE["sample_s"] seconds of requests submitted at
    once to the server (capacity) and to the plain per-request path (a film
    object per request, frames traced and read back one by one), whose
    throughput ratio is served_over_plain."""
    from spectral_b200.serve import Server, poisson_requests, run_plain_stream, run_stream
    budget = int(SERVE["budget_gb"] * (1 << 30))
    warm = poisson_requests(SERVE["rate"], 0.5, SERVE["seed"] ^ 0xA5A5 ^ rank)
    srv = Server(ctx, budget_bytes=budget)
    run_stream(srv, warm, want_image=True)
    srv.close()
    run_plain_stream(ctx, warm[:20], time_scale=0.0)
    stream = poisson_requests(SERVE["rate"], seconds, SERVE["seed"] + rank)
    srv = Server(ctx, budget_bytes=budget)
    served = run_stream(srv, stream, want_image=True)
    srv.close()
    sample = [r for r in stream if r[0] < SERVE["sample_s"]]
    capacity, plain = None, None
    for _ in range(2):  # best of two: both are host-driven loops with run-to-run noise
        srv = Server(ctx, budget_bytes=budget)
        c = run_stream(srv, sample, time_scale=0.0, want_image=True)
        srv.close()
        p = run_plain_stream(ctx, sample, time_scale=0.0)
        capacity = c if capacity is None or c["photons_per_s"] > capacity["photons_per_s"] else capacity
        plain = p if plain is None or p["photons_per_s"] > plain["photons_per_s"] else plain
    return {
        "window_s": seconds, "rate_per_s": SERVE["rate"], "requests": len(stream),
        "sessions": sum(1 for r in stream if r[2] > 1), "frames": sum(r[2] for r in stream),
        "p50_ms": served["p50_ms"], "p99_ms": served["p99_ms"],
        "p50_first_frame_ms": served["p50_first_frame_ms"], "p99_first_frame_ms": served["p99_first_frame_ms"],
        "photons_per_s": served["photons_per_s"], "photons": served["photons"], "wall_s": served["wall_s"],
        "steps": served["steps"],
        "capacity_photons_per_s": capacity["photons_per_s"],
        "plain_per_request_photons_per_s": plain["photons_per_s"],
        "served_over_plain": capacity["photons_per_s"] / plain["photons_per_s"],
        "sample": "latency: the first %.0f s of the stream (seed 0x%X) replayed in real time; capacity and plain: "
                  "its first %.0f s (%d requests, %d frames) submitted at once to the server and to a film object "
                  "per request, best of two runs each" % (seconds, SERVE["seed"] + rank, SERVE["sample_s"],
                                                           len(sample), sum(r[2] for r in sample)),
        "what": "latency from arrival to the XYZ image in host memory; served_over_plain = capacity / plain on "
                "the same requests",
    }


def run_gpu_serve(args, rank, world, local_rank):
    import torch
    import spectral_b200 as sb
    torch.cuda.set_device(local_rank)
    ctx = sb.GpuContext(local_rank)
    seconds = args.serve_seconds or 15.0
    uuid = "GPU-" + str(torch.cuda.get_device_properties(torch.device("cuda", local_rank)).uuid)
    with ClockSampler(uuid) as clk, torch.cuda.nvtx.range("timed"):  # nvtx range for ncu --nvtx-include
        served = served_summary(ctx, seconds, rank)
    total_rate = served["photons_per_s"]
    if world > 1:  # every rank served its own stream: total photons over the longest replay
        import torch.distributed as dist
        dev = torch.device("cuda", local_rank)
        ph = torch.tensor([float(served["photons"])], dtype=torch.float64, device=dev)
        wall = torch.tensor([served["wall_s"]], dtype=torch.float64, device=dev)
        dist.all_reduce(ph, op=dist.ReduceOp.SUM)
        dist.all_reduce(wall, op=dist.ReduceOp.MAX)
        total_rate = float(ph.item()) / float(wall.item())
    if rank != 0:
        return None
    from spectral_b200.serve import poisson_requests
    stream = poisson_requests(SERVE["rate"], seconds, SERVE["seed"] + rank)
    in_bytes = sum(C.sizeof(r[1]) for r in stream)
    out_bytes = sum(3 * r[1].width * r[1].height * 4 for r in stream)
    return {
        "metric": "served photons/s with p50/p99 request latency (continuous batching vs plain per-request launch)",
        "value": total_rate, "unit": "photons/s", "n_gpus": world, "steps": 1,
        "warmup": args.warmup, "ms_per_step": served["wall_s"] * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 transport, int64 fixed-point film", "data": "synthetic (seeded stream)",
        "config": {"workload": "serve: Poisson %.0f req/s for %.0f s (%d requests, %d frames), prism scenes of the "
                               "batch distribution, 2^16-2^20 photons per frame, 30%% orbit sessions of 16-128 "
                               "frames at 2 deg, %.0f GB budget" % (SERVE["rate"], seconds, len(stream),
                                                                     served["frames"], SERVE["budget_gb"]),
                   "parallelism": "own request stream per rank, no collective",
                   "timing": "host clock over the whole stream replayed in real time (one step = the stream)"},
        "served": served,
        "e2e": {"value": total_rate, "unit": "photons/s", "h2d_bytes_per_step": in_bytes,
                "d2h_bytes_per_step": out_bytes,
                "path": "sc_server_submit per request, sc_server_step, sc_server_poll with the XYZ image to host"},
        "gpu_launches": served["steps"] * 3,  # per server step: batch_kernel, reduce_scan, reduce_list
        "clocks": clk.summary(),
    }


def run_gpu_split(args, rank, world, local_rank):
    """One scene split across the ranks (strong scaling): the rainbow workload's
    2^26 photons in contiguous ranges, one per rank, each traced into the rank's
    own int64 film, then ONE all-reduce (sum) of the 1.06 GB films over NCCL and
    the sensor reduction of the summed film on every rank.  The film of any
    number of ranks is bit-identical to one GPU's."""
    import torch
    import spectral_b200 as sb
    from spectral_b200 import _lib
    from spectral_b200.shard import photon_range, trace_sharded
    dist = None
    if world > 1:
        import torch.distributed as dist
    wl = "rainbow"
    cfg = dict(WORKLOADS[wl])
    if args.photons:
        cfg["photons"] = args.photons
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    ctx = sb.GpuContext(local_rank)
    scene, beam, cam = build_scene(wl)
    W, H, B, N = cfg["width"], cfg["height"], cfg["bins"], cfg["photons"]
    b0, b1 = photon_range(rank, world, N)
    prims, np_, planes, npl, mats, nm = scene.arrays()

    def dev_bytes(obj, n):
        return torch.frombuffer(bytearray(bytes(obj)[: n * C.sizeof(obj._type_)] or b"\0"), dtype=torch.uint8).to(dev)

    d_prims, d_planes, d_mats = dev_bytes(prims, np_), dev_bytes(planes, npl), dev_bytes(mats, nm)
    opts = _lib.sc_film_options(B, cfg["lambda_min"], cfg["lambda_max"], cfg["max_bounces"], 32, 0)
    desc = _lib.sc_trace_desc(d_prims.data_ptr(), np_, d_planes.data_ptr(), npl, d_mats.data_ptr(), nm, cam.c, beam.c,
                              _lib.sc_vol_weights(cfg["sigma_s"], cfg["sigma_t"], cfg["g"]), W, H, cfg["seed"], 1,
                              cfg["max_dist"], opts, None)
    film = torch.zeros(_lib.lib.sc_film_bytes(W, H, B) // 8, dtype=torch.int64, device=dev)
    flags = torch.zeros(_lib.lib.sc_film_flag_bytes(W, H) // 4, dtype=torch.int32, device=dev)
    xyz = torch.empty(3 * W * H, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = C.c_void_p(stream.cuda_stream)
    peer = args.split_exchange == "peer"
    if peer:
        from spectral_b200.shard import PeerFilms, reduce_band_peers, tile_row_band
        peers = PeerFilms(ctx, film) if dist else None
        ptrs = peers.ptrs if dist else [film.data_ptr()]
        rb, re_ = tile_row_band(rank, world, H)
        rows = max(e - b for b, e in (tile_row_band(r, world, H) for r in range(world)))
        band = torch.zeros((rows, W, 3), dtype=torch.float32, device=dev)
        bands = torch.empty((world, rows, W, 3), dtype=torch.float32, device=dev)
        ready = torch.zeros(1, dtype=torch.int32, device=dev)

    def step_peer(ev=None):
        # trace; a one-word all-reduce orders every rank's trace before any
        # band reads it; each rank reduces its band from all films; gathering
        # the bands orders every read before the films are cleared
        if ev:
            ev[0].record(stream)
        _lib.check(_lib.lib.sc_trace_photons_device(ctx.h, C.byref(desc), b0, b1 - b0, C.c_void_p(film.data_ptr()),
                                                    C.c_void_p(flags.data_ptr()), sp))
        if ev:
            ev[1].record(stream)
        if dist:
            dist.all_reduce(ready)
        reduce_band_peers(ctx, ptrs, W, H, B, opts, rb, re_, xyz.data_ptr(), stream.cuda_stream)
        if dist:
            band[: re_ - rb].copy_(xyz.view(H, W, 3)[rb:re_])
            dist.all_gather_into_tensor(bands, band)
            for r in range(world):
                b, e = tile_row_band(r, world, H)
                xyz.view(H, W, 3)[b:e].copy_(bands[r, : e - b])
        if ev:
            ev[2].record(stream)
        film.zero_()
        flags.zero_()
        if ev:
            ev[3].record(stream)

    def step(ev=None):
        if peer:
            return step_peer(ev)
        if ev:
            ev[0].record(stream)
        _lib.check(_lib.lib.sc_trace_photons_device(ctx.h, C.byref(desc), b0, b1 - b0, C.c_void_p(film.data_ptr()),
                                                    C.c_void_p(flags.data_ptr()), sp))
        if ev:
            ev[1].record(stream)
        if dist:
            dist.all_reduce(film, op=dist.ReduceOp.SUM)  # int64: exact
            flags.fill_(-1)                               # other ranks lit tiles too
        if ev:
            ev[2].record(stream)
        _lib.check(_lib.lib.sc_sensor_reduce_device(ctx.h, W, H, B, cfg["lambda_min"], cfg["lambda_max"], 32,
                                                    C.c_void_p(film.data_ptr()), C.c_void_p(flags.data_ptr()),
                                                    C.c_void_p(xyz.data_ptr()), 1, sp))
        if ev:
            ev[3].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    with ClockSampler(uuid) as clk:
        for k in range(args.steps):
            step(ev[k])
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    parts = [[ev[k][i].elapsed_time(ev[k][i + 1]) for k in range(args.steps)] for i in range(3)]
    total_ms = sum(ev[k][0].elapsed_time(ev[k][3]) for k in range(args.steps))
    if dist:
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = N * args.steps / (total_ms / 1e3)

    # end to end through the film object: trace_sharded (own range + the film
    # all-reduce) and the XYZ image back to the host, every step
    pf = sb.GpuPhotonFilm(ctx, scene, cam, beam, W, H, N, cfg["seed"], cfg["max_dist"],
                          sb.VolWeights(cfg["sigma_s"], cfg["sigma_t"], cfg["g"]), bins=B,
                          lambda_min=cfg["lambda_min"], lambda_max=cfg["lambda_max"], max_bounces=cfg["max_bounces"])
    host_xyz = torch.empty(3 * W * H, dtype=torch.float32, pin_memory=True).numpy()

    host_t = torch.from_numpy(host_xyz)

    def e2e_step():
        if peer:  # the device-pointer path with the peer-band exchange, the image back to the host
            step_peer()
            host_t.copy_(xyz)
            return
        if dist:
            trace_sharded(pf, N, cfg["seed"])
        else:
            pf.dispatch_photons(0, N, cfg["seed"])
        _lib.check(_lib.lib.sc_photon_film_read_accum(pf.h, host_xyz.ctypes.data_as(C.POINTER(C.c_float))))
        _lib.check(_lib.lib.sc_photon_film_clear(pf.h))

    e2e_steps = args.e2e_steps or max(3, args.steps // 2)
    e2e_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    pf.close()
    if peer and dist:
        torch.cuda.synchronize()
        dist.barrier()  # every rank is done with the others' films
        peers.close()
    if rank != 0:
        return None
    film_bytes = film.numel() * 8
    ar_ms = statistics.mean(parts[1])
    line = {
        "metric": METRIC_POINT + "; one scene split across GPUs",
        "value": value, "unit": "photons/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32 transport, int64 fixed-point film", "data": "synthetic (seeded scene)",
        "config": {"workload": "split: the rainbow scene (water sphere r=1, beam 2.2, 1920x1080x64 bins), %d photons "
                               "split into contiguous ranges over %d rank(s)" % (N, world),
                   "photons_per_step": N, "film": [W, H, B],
                   "parallelism": ("photon ranges per rank; each rank reduces its band of tile rows from every "
                                   "rank's film as peer memory, bands all-gathered" if peer else
                                   "photon ranges per rank + one int64 NCCL all-reduce of the film per step"),
                   "exchange": args.split_exchange},
        "kernels": ({"trace_ms": statistics.mean(parts[0]), "band_reduce_and_gather_ms": ar_ms,
                     "clear_ms": statistics.mean(parts[2])} if peer else
                    {"trace_ms": statistics.mean(parts[0]), "allreduce_ms": ar_ms,
                     "reduce_ms": statistics.mean(parts[2])}),
        "allreduce": None if peer else {"bytes": film_bytes, "ms": ar_ms,
                      "bus_gbs": (film_bytes * 2 * (world - 1) / world / (ar_ms / 1e3) / 1e9) if world > 1 and ar_ms > 0
                      else None},
        "e2e": {"value": N * e2e_steps / e2e_s, "unit": "photons/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 3 * W * H * 4,
                "path": ("sc_trace_photons_device (own range) + sc_sensor_reduce_peers (own band of every film) + "
                         "band all-gather + image to pinned host memory" if peer else
                         "shard.trace_sharded (own range + film all-reduce) + read_accum (host f32 XYZ) + clear")},
        "gpu_launches": args.steps * (2 + 3),  # per step: sort (3) + photon kernel, drain
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        rate, n_s, dt, th = run_cpu(wl, args.cpu_seconds)
        line["cpu_baseline"] = {"value": rate, "unit": "photons/s", "cores": th, "kind": "port",
                                "sample": "%d photons of the rainbow workload from photon 0, %.1f s, %s"
                                          % (n_s, dt, cpu_model())}
    return line


BATCH = dict(n_jobs=256, seed=0xB200, bins=32, lambda_min=380.0, lambda_max=780.0)


def batch_specs(rank, n_jobs=0):
    """The batch's job dicts (spectral_b200.specs.random_prism_jobs) of `rank`."""
    return load_specs().random_prism_jobs(n_jobs or BATCH["n_jobs"], seed=BATCH["seed"] + rank, bins=BATCH["bins"],
                                          lambda_min=BATCH["lambda_min"], lambda_max=BATCH["lambda_max"])


def run_cpu_batch(seconds, threads=None, rank=0, specs=None):
    """Photons/s of the CPU restatement over a bounded sample of the batch (or
    of the job dicts `specs`).  Scenes are rendered in parallel, one host thread
    per scene with its own film (the CPU oracle releases the GIL), taking scenes
    in job order and the first 2^18 photons of each, until `seconds` of wall
    time are used."""
    import threading
    import oracle
    if specs is None:
        specs = batch_specs(rank)
    threads = threads or os.cpu_count() or 1
    per_job = 1 << 18
    lock = threading.Lock()
    state = {"next": 0, "done": 0, "scenes": 0}
    t0 = time.perf_counter()

    def worker():
        while True:
            with lock:
                i = state["next"]
                if i >= len(specs) or time.perf_counter() - t0 >= seconds:
                    return
                state["next"] += 1
            sc, cam, beam, p = oracle_prism_job(specs[i])
            film = np.zeros(p.width * p.height * p.bins, np.int64)
            n = min(specs[i]["n_photons"], per_job)
            oracle.lib.or_render_point(C.byref(sc.c), C.byref(cam), C.byref(beam), C.byref(p), None, 0, n, None,
                                       None, film.ctypes.data_as(C.POINTER(C.c_int64)))
            with lock:
                state["done"] += n
                state["scenes"] += 1

    ts = [threading.Thread(target=worker) for _ in range(threads)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    dt = time.perf_counter() - t0
    return state["done"] / dt, state["done"], dt, threads, state["scenes"]


def batch_film_err(ctx, specs, cap=1 << 16):
    """Relative L1 of batch images against the oracle (the checker; never
    timed) on a sample: every scene of the batch with its own film, traced by
    the same batched launch on photons [0, cap) of its stream."""
    import concurrent.futures as cf
    import oracle
    from spectral_b200.batch import Batch, prism_jobs
    capped = [dict(s, n_photons=min(s["n_photons"], cap)) for s in specs]
    b = Batch(ctx, prism_jobs(capped))
    b.run()
    imgs = [b.read_xyz(i) for i in range(len(capped))]
    b.close()

    def ref(s):
        sc, cam, beam, p = oracle_prism_job(s)
        fs = np.zeros(p.width * p.height * p.bins, np.int64)
        oracle.lib.or_render_point(C.byref(sc.c), C.byref(cam), C.byref(beam), C.byref(p), None, 0, s["n_photons"],
                                   None, None, fs.ctypes.data_as(C.POINTER(C.c_int64)))
        return oracle_xyz_from_spectral(fs, s["bins"], s["lambda_min"], s["lambda_max"])
    with cf.ThreadPoolExecutor(max(1, min(16, os.cpu_count() or 1))) as ex:  # the oracle releases the GIL
        refs = list(ex.map(ref, capped))
    num = sum(float(np.abs(g.astype(np.float64) - r).sum()) for g, r in zip(imgs, refs))
    den = sum(float(np.abs(r).sum()) for r in refs)
    worst = max(rel_l1(g, r) for g, r in zip(imgs, refs))
    return {"value": num / den, "worst_scene": worst, "bar": 5e-3, "photons": sum(s["n_photons"] for s in capped),
            "sample": "every scene of the batch with its film, photons [0, %d) of each through one batched launch; "
                      "GPU XYZ images vs the oracle's spectral films reduced by the bin-averaged CMF on the host; "
                      "value = sum |diff| / sum |ref| over all scenes" % cap}


def run_gpu_batch(args, rank, world, local_rank):
    import torch
    import spectral_b200 as sb
    from spectral_b200.batch import Batch
    dist = None
    if world > 1:
        import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    ctx = sb.GpuContext(local_rank)
    from spectral_b200.batch import prism_jobs
    specs = batch_specs(rank, args.scenes)  # weak scaling: every rank renders its own scenes
    jobs = prism_jobs(specs)
    b = Batch(ctx, jobs)
    tuning = b.autotune()  # untimed: picks chunk size, register bound, splat aggregation
    stats = b.stats()      # untimed instrumented pass: work counters and dirty tiles
    stream = torch.cuda.Stream(dev)
    sp = stream.cuda_stream

    def timed(fn, steps):
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(steps)]
        for k in range(steps):
            ev[k][0].record(stream)
            fn(sp)
            ev[k][1].record(stream)
        torch.cuda.synchronize()
        return [ev[k][0].elapsed_time(ev[k][1]) for k in range(steps)]

    for _ in range(args.warmup):
        b.run(sp)
    b.run_plain(sp)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    with ClockSampler(uuid) as clk, torch.cuda.nvtx.range("timed"):  # nvtx range for ncu --nvtx-include
        ms = timed(b.run, args.steps)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with torch.cuda.nvtx.range("plain"):  # nvtx range for an ncu launch list of the plain path
        plain_ms = timed(b.run_plain, max(2, args.steps // 2))
    # plain per-scene launches through the drop-in object API (what a caller of
    # the reference's GpuPhotonFilm does per scene): create, trace, read back,
    # free.  The film's buffers come from the context's memory pool, so after
    # the first pass no pass allocates; best of two passes.
    plain_api_s = float("inf")
    for _ in range(2):
        t0 = time.perf_counter()
        for j in jobs:
            sc = sb.Scene(background=0.0)
            planes = [(tuple(j.planes[k].normal), j.planes[k].d) for k in range(j.n_planes)]
            sc.add_solid(planes, sb.Dielectric(j.mats[0].glass))
            f = sb.GpuPhotonFilm(ctx, sc, sb.Camera(j.cam), sb.Beam.from_c(j.beam), j.width, j.height,
                                 j.n_photons, j.seed, j.max_dist,
                                 sb.VolWeights(j.weights.sigma_s, j.weights.sigma_t, j.weights.g),
                                 bins=j.opts.bins, lambda_min=j.opts.lambda_min, lambda_max=j.opts.lambda_max,
                                 max_bounces=j.opts.max_bounces)
            f.trace_and_resolve(j.n_photons, j.seed)
            f.accum()
            f.close()
        plain_api_s = min(plain_api_s, time.perf_counter() - t0)
    total_ms = sum(ms)
    job_photons = b.total_photons  # photons of all ranks' batches (each rank draws its own scenes)
    if dist:
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        t = torch.tensor([b.total_photons], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        job_photons = float(t.item())
    value = job_photons * args.steps / (total_ms / 1e3)
    plain_value = b.total_photons * len(plain_ms) / (sum(plain_ms) / 1e3)

    # end to end: new job table each step (host -> device), one pass, every
    # scene's XYZ image back to pinned host memory
    # (the copy of pass k runs on the batch's copy stream while pass k+1 traces)
    host = torch.empty(b.xyz_floats, dtype=torch.float32, pin_memory=True).numpy()
    e2e_steps = args.e2e_steps or max(3, args.steps // 2)
    for _ in range(1):
        b.update_jobs(jobs)
        b.run(sp)
        b.read_all_xyz_async(host)
    b.synchronize()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        b.update_jobs(jobs)
        b.run(sp)
        b.read_all_xyz_async(host)
    b.synchronize()
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = job_photons * e2e_steps / e2e_s
    if rank != 0:
        served = None
        if args.serve_seconds > 0:  # every rank serves its own stream (the same work as rank 0)
            served_summary(ctx, args.serve_seconds, rank)
        return None
    film_err = batch_film_err(ctx, specs)
    served = served_summary(ctx, args.serve_seconds, rank) if args.serve_seconds > 0 else None

    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs") or 6650.0
    peak_note = "measured" if peaks.get("hbm_gbs") else "fallback"
    step_s = total_ms / args.steps / 1e3
    cl = clk.summary()
    film_gb = b.film_bytes / 1e9
    line = {
        "metric": "photons/s @<=0.5% film err; batched vs plain per-scene launch (forward + volumetric)",
        "value": value, "unit": "photons/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 transport, int64 fixed-point films", "data": "synthetic (PCG-seeded scene batch)",
        "config": {"workload": "batch: %d prism scenes, glass {BK7,SF11,fused silica}, apex U(30,75), incidence "
                               "U(30,60), photons log-U(2^14,2^22), square film side log-U(128,1024), 32 bins, "
                               "sigma_s U(0.01,0.1); one persistent graph-captured launch + one drain/reduce"
                               % len(jobs),
                   "photons_per_step": int(job_photons), "scenes_per_rank": len(jobs),
                   "film_gb_per_rank": film_gb, "l2": "films (%.1f GB) far larger than L2" % film_gb,
                   "autotuned": tuning, "parallelism": "scene batch per rank, no collective"},
        "plain": {"value": plain_value, "unit": "photons/s", "ms_per_step": sum(plain_ms) / len(plain_ms),
                  "what": "the same %d scenes as plain per-scene launches (trace + drain/reduce each), one GPU"
                          % len(jobs)},
        "plain_api": {"value": b.total_photons / plain_api_s, "unit": "photons/s", "s_per_step": plain_api_s,
                      "what": "per scene: GpuPhotonFilm create + trace_and_resolve + accum (host XYZ) + destroy; "
                              "best of two passes over the 256 scenes"},
        "batched_over_plain": value / job_photons * b.total_photons / plain_value,
        "batched_e2e_over_plain_api": e2e_value / job_photons * b.total_photons / (b.total_photons / plain_api_s),
        "e2e": {"value": e2e_value, "unit": "photons/s", "h2d_bytes_per_step": b.job_table_bytes,
                "d2h_bytes_per_step": b.xyz_floats * 4,
                "path": "sc_batch_update_jobs + sc_batch_run + sc_batch_read_all_xyz_async (pinned host; the "
                        "copy of a pass overlaps the next pass's tracing), all steps synchronised at the end"},
        "gpu_launches": args.steps * 3,  # per pass: batch_kernel, reduce_scan, reduce_list
        "film_err": film_err,
        "served": served,
        "work": stats,
        "roofline": {"bound": "hbm", "kernel": "batch_kernel + reduce_scan + reduce_list (one pass)",
                     "achieved": (stats["in_frame_samples"] * 8 + 2 * stats["dirty_tile_bytes"] +
                                  b.xyz_floats * 4) / step_s / 1e9,
                     "peak": hbm, "unit": "GB/s", "traffic": ncu_traffic("batch", not args.scenes)[0],
                     "traffic_source": ncu_traffic("batch", not args.scenes)[1],
                     "peak_source": "%s hbm_gbs" % peak_note,
                     "algorithmic": "8 B per in-frame haze sample + read and zero of every lit film tile + "
                                    "the f32 XYZ images"},
        "clocks": cl,
    }
    line["roofline"]["frac"] = line["roofline"]["achieved"] / hbm
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    sm_mhz = cl["sm_mhz"] or peaks.get("sm_max_mhz", 1965.0)
    flops = stats["photons"] * 20 + stats["segments"] * (14 * 5 + 4 * 60) + stats["scatters"] * 45
    fp32_peak = sms * 128 * 2 * sm_mhz * 1e6 / 1e12
    line["roofline_fp32"] = {"counted_flops": flops, "achieved_tflops": flops / step_s / 1e12,
                             "peak_tflops": fp32_peak, "frac": flops / step_s / 1e12 / fp32_peak,
                             "peak_source": "%d SMs x 128 FP32 lanes x 2 x %.0f MHz (sampled median)" % (sms, sm_mhz)}
    line["roofline_issue"] = issue_roofline("batch", stats["photons"], step_s, sms, sm_mhz, not args.scenes)
    if line["roofline_issue"]:
        line["roofline_issue"]["kernel"] = "batch_kernel, over the whole pass (drain included)"
    if world == 1 and not args.no_cpu_baseline:
        rate, n_s, dt, th, sc = run_cpu_batch(args.cpu_seconds)
        line["cpu_baseline"] = {"value": rate, "unit": "photons/s", "cores": th, "kind": "port",
                                "sample": "first %d photons of each of the first %d scenes (%d photons, %.1f s), %s"
                                          % (1 << 18, sc, n_s, dt, cpu_model())}
    b.close()
    return line


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return 0
        rates, serial = [], None
        per_step = max(1.0, args.cpu_seconds / max(1, args.steps))
        if args.workload == "atomics":
            th = 1
            for _ in range(args.steps):
                rate, done, dt = run_cpu_atomics(per_step)
                rates.append((3 * (1 << 20) * done, dt))
            sample = "per step batches of 2^20 splats on one host thread for ~%.1f s" % per_step
            metric = "L2 atomic throughput, u32 atomicAdd (AtomicFilm synthetic splat)"
            cfg_line = {"workload": "atomics (see the GPU arm)", "splats_per_step": ATOMICS["splats"]}
        elif args.workload == "serve":
            reqs = [r[1] for r in load_specs().poisson_request_specs(SERVE["rate"], args.serve_seconds or 15.0,
                                                                       SERVE["seed"])]
            run_cpu_batch(0.5, specs=reqs)
            for _ in range(args.steps):
                rate, n_s, dt, th, sc = run_cpu_batch(per_step, specs=reqs)
                rates.append((n_s, dt))
            sample = ("per step the first frame (up to 2^18 photons) of the stream's requests in arrival order, "
                      "one host thread per request, for ~%.1f s" % per_step)
            metric = ("served photons/s with p50/p99 request latency (continuous batching vs plain per-request "
                      "launch)")
            cfg_line = {"workload": "serve (see the GPU arm)", "rate_per_s": SERVE["rate"],
                        "seconds": args.serve_seconds or 15.0}
        elif args.workload == "tracer":
            run_cpu_tracer(0.5)
            for _ in range(args.steps):
                rate, frames, dt, th = run_cpu_tracer(per_step)
                rates.append((TRACER["width"] * TRACER["height"] * frames, dt))
            sample = "per step whole 1280x720 frames at 1 spp for ~%.1f s" % per_step
            metric = "path samples/s (hero-wavelength camera tracer, 4 lanes, depth 8)"
            cfg_line = {"workload": "tracer (see the GPU arm)", "samples_per_step": TRACER["width"] * TRACER["height"]
                        * TRACER["spp"]}
        elif args.workload == "batch":
            run_cpu_batch(0.5)
            for _ in range(args.steps):
                rate, n_s, dt, th, sc = run_cpu_batch(per_step)
                rates.append((n_s, dt))
            sample = ("per step the first 2^18 photons of each scene, scenes in job order rendered in parallel "
                      "(one host thread per scene) for ~%.1f s" % per_step)
            metric = "photons/s @<=0.5% film err; batched vs plain per-scene launch (forward + volumetric)"
            cfg_line = {"workload": "batch: 256 prism scenes (see the GPU arm)", "scenes": BATCH["n_jobs"]}
        else:
            wl = "rainbow" if args.workload == "split" else args.workload  # the split workload traces the rainbow
            cfg = WORKLOADS[wl]
            for _ in range(args.warmup):
                run_cpu(wl, 1.0)
            for _ in range(args.steps):
                rate, n_s, dt, th = run_cpu(wl, per_step)
                rates.append((n_s, dt))
            sample = "per step %d photons from photon 0 (the whole workload repeated when shorter)" % rates[0][0]
            serial = cpu_serial(wl, args.cpu_seconds)
            metric = METRIC_BEAM if wl == "beam" else METRIC_POINT
            if args.workload == "split":
                metric += "; one scene split across GPUs"
            cfg_line = {"workload": args.workload, "photons_per_step": cfg["photons"],
                        "film": [cfg["width"], cfg["height"], cfg["bins"]]}
        tot_n, tot_t = sum(n for n, _ in rates), sum(t for _, t in rates)
        value = tot_n / tot_t
        unit, what = {"atomics": ("atomics/s", "the synthetic splat of AtomicFilm"),
                      "tracer": ("samples/s", "CpuTracer::accumulate"),
                      "beam": ("photons/s", "render_volumetric_scene (beam estimator)")}.get(
            args.workload, ("photons/s", "render_volumetric_scene_point"))
        line = {"metric": metric, "value": value,
                "unit": unit, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": tot_t / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32 transport", "data": "synthetic (seeded scenes)", "impl": "reference",
                "config": cfg_line,
                "cpu_baseline": {"value": value, "unit": unit, "cores": th, "kind": "port",
                                 "sample": sample + "; CPU restatement of spectral-core %s, %s" % (what, cpu_model())},
                "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        if serial is not None:
            line["cpu_baseline"]["serial"] = serial
        print(json.dumps(line))
        return 0
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    line = {"atomics": run_gpu_atomics, "batch": run_gpu_batch, "serve": run_gpu_serve,
            "split": run_gpu_split, "tracer": run_gpu_tracer}.get(
        args.workload, run_gpu)(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
