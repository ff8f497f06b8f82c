"""Benchmark of the render path on the 1M-triangle, 1920x1080, 16 spp, depth-12 workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step renders the whole job: 16 samples per pixel of the 1920x1080 frame of the seeded
1M-triangle scene (200 instances of icospheres and displaced grids, random uber-shader
materials, 16 value-noise 1024^2 textures, a 2048x1024 HDRI), trace depth 12, NEE with
HDRI importance sampling (-dmis -emis). Rays are counted as traced: radiance plus shadow.

Reported (one JSON line, rank 0):
  value       Mrays/s of the device-timed render with the scene resident in HBM (all ranks)
  e2e         the same metric through the C-ABI from page-locked host buffers: lux_init (scene
              upload, device BVH build, light tables, textures), lux_render, lux_copy_image to
              host, lux_free
  e2e_resident_scene  the drop-in's per-reset cycle on a scene built once (lux_init_on_scene,
              lux_render, lux_copy_image, lux_free), as the reference builds its acceleration
              structures at load and reallocates only per-pixel state in pathtraceInit
  roofline    the traversal kernel (the dominant one): algorithmic bytes per launch over its
              CUDA-event duration against the measured HBM copy bandwidth; the shading kernel
              beside it
  cpu_baseline  the reference's own render-path sources built for the host (oracle/_ref),
              OpenMP over pixel rows, on a bounded crop of the same workload
  batched     (one GPU) the batching form: 64 seeded jobs over 8 resident scenes of 10k-2M
              triangles, mixed resolutions / spp / depths, rendered in one shared wavefront by the
              job engine, against the same 64 jobs through single-job contexts on the same
              resident scenes: one lux_render_iter per sample (the reference's plain wavefront)
              and lux_render (many samples per wave); images compared bitwise
  served      (one GPU) the serving form: 256 Poisson requests at 50, 150 and 400 per second
              against 16 resident scenes of 50k-4M triangles (binary16 HDRIs) under a 150 GB HBM
              budget, continuous batching in the engine, against first-come-first-served
              single-job contexts on the same resident scenes; p50/p95/p99 latency and throughput
  precision   (one GPU) the precision form (4M triangles, binary16 textures and HDRI, FP64 CDFs,
              compensated accumulation, 1080p at 1024 spp) against the plain FP32 path on the
              same scene and RNG streams; and both against the FP64 integrator (the oracle in
              double on the host cores) at 4096 spp on a crop of a 256x256 view
With --impl reference only that CPU arm runs (rank 0). --no-forms skips batched, served, precision.
Under torchrun every rank renders its own 16 samples (disjoint iterations, weak scaling) and
the FP32 images are summed with one NCCL all-reduce per step.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mrays/s + served-job p50/p99 vs plain wavefront, 1 B200, equal relMSE"
SPP = 16
WORKLOAD = "1M tris / 200 instances, 1920x1080, 16 spp, depth 12, NEE + HDRI MIS (-dmis -emis), seed 0"
# algorithmic bytes per path-bounce (fixed figures): trace I/O and shade
TRACE_BYTES_PER_BOUNCE = 68.0  # radiance + shadow ray I/O of one path-bounce
SHADE_BYTES_PER_BOUNCE = 244.0


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _with_camera(sc, cam):
    """The host scene's description with another camera (restored by the caller)."""
    d = sc.desc
    saved = type(d.camera).from_buffer_copy(d.camera)
    d.camera = cam
    return saved


def run_batched(seed: int = 0):
    """The batching form: 64 jobs in one shared wavefront of the job engine, against the same 64
    jobs rendered one after another by single-job contexts on resident scenes (scenes built
    once, as the reference builds its acceleration structures at load):
      plain_wavefront  lux_init_on_scene, then one lux_render_iter per sample -- the
                       reference's pathtrace() loop, one iteration per call -- then the image
      plain_waves      the same contexts with lux_render (many samples per wave)
    and, for reference, one lux_init per job (scene upload and BVH build per job, cold).
    Every arm is host wall time from the first submit/context to the last image on the host;
    scene builds are outside it for every arm. Images are compared bitwise with the engine's."""
    import luxion_b200 as lx
    from luxion_b200 import workloads
    from luxion_b200._ffi import default_options
    t0 = time.perf_counter()
    scenes, tris = workloads.batch_scenes(seed)
    jobs = workloads.batch_jobs(len(scenes), seed=seed)
    t_gen = time.perf_counter() - t0
    base = dict(direct_light_sampling=1, env_importance_sampling=1)
    opt = default_options(**base)
    t0 = time.perf_counter()
    E = lx.Engine(scenes, opt)
    t_create = time.perf_counter() - t0
    t0 = time.perf_counter()
    ids = [E.submit(j["scene"], j["spp"], trace_depth=j["depth"], camera=j["camera"]) for j in jobs]
    E.run()
    imgs = [E.image(i) for i in ids]
    t_batch = time.perf_counter() - t0
    st = E.stats()
    E.close()
    samples = sum(j["camera"].width * j["camera"].height * j["spp"] for j in jobs)
    t0 = time.perf_counter()
    res = [lx.ResidentScene(sc, opt) for sc in scenes]
    t_res = time.perf_counter() - t0
    arms = {}
    for arm in ("plain_wavefront", "plain_waves"):
        t0 = time.perf_counter()
        same = 0
        for j, img in zip(jobs, imgs):
            r = lx.Renderer(res[j["scene"]], default_options(**base, trace_depth=j["depth"]), camera=j["camera"])
            if arm == "plain_wavefront":
                for it in range(1, j["spp"] + 1):
                    r.render_iter(it)
            else:
                r.render(1, j["spp"])
            ref = r.image_sum()
            r.close()
            same += int(np.array_equal(ref.view(np.uint32), img.view(np.uint32)))
        el = time.perf_counter() - t0
        arms[arm] = {"s": el, "samples_per_s": samples / el, "batched_speedup": el / t_batch,
                     "identical_images": f"{same}/{len(jobs)}"}
    for r in res:
        r.close()
    # per-job scene builds (cold), on a subset: the first 16 jobs
    sub = jobs[:16]
    t0 = time.perf_counter()
    for j in sub:
        saved = _with_camera(scenes[j["scene"]], j["camera"])
        try:
            r = lx.Renderer(scenes[j["scene"]], default_options(**base, trace_depth=j["depth"]))
        finally:
            scenes[j["scene"]].desc.camera = saved
        r.render(1, j["spp"])
        r.image_sum()
        r.close()
    t_cold = time.perf_counter() - t0
    for sc in scenes:
        sc.close()
    return {"workload": "64 jobs over 8 seeded scenes of %d-%d tris; res {128^2,256^2,512^2,1024^2,1920x1080}, "
                        "spp {1,4,16,64}, depth 4..16, -dmis -emis" % (min(tris), max(tris)),
            "samples": samples, "batched_s": t_batch, "batched_samples_per_s": samples / t_batch,
            "batched_mrays_per_s": st["rays"] / t_batch / 1e6, "waves": st["waves"],
            "autotuned": {"max_paths": st["max_paths"], "trace_blocks": st["trace_blocks"]},
            "plain": arms, "speedup_vs_plain_wavefront": arms["plain_wavefront"]["s"] / t_batch,
            "speedup_vs_plain_waves": arms["plain_waves"]["s"] / t_batch,
            "cold_per_job_scene_build_first16_s": t_cold, "engine_create_s": t_create, "resident_scenes_s": t_res,
            "scene_gen_s": t_gen,
            "timing": "host wall clock, first submit (or context) to the last image on the host, scenes resident"}


def fcfs_latencies(arrival_ms, service_ms):
    """Latencies of a first-come-first-served single server with the given service times."""
    t, out = 0.0, []
    for a, s in zip(arrival_ms, service_ms):
        t = max(t, a) + s
        out.append(t - a)
    return out


def run_served(seed: int = 0, requests: int = 256, rates=(50.0, 150.0, 400.0)):
    """The serving form: continuous batching in the job engine at several Poisson rates, against
    first-come-first-served single-job contexts on the same resident scenes. The same requests
    (scene, camera, spp) arrive at each rate, so the plain path's service time of each request is
    measured once and its latencies at every rate follow from the FCFS recurrence."""
    import luxion_b200 as lx
    from luxion_b200 import serving, workloads
    from luxion_b200._ffi import SCHED_SHORTEST_FIRST, default_options
    scenes, tris = workloads.serving_scenes(seed)
    base = workloads.request_stream(len(scenes), requests, rates[0], seed=seed)
    opt = default_options(direct_light_sampling=1, env_importance_sampling=1)
    E = lx.Engine(scenes, opt, hbm_budget_bytes=150 * 10**9, schedule=SCHED_SHORTEST_FIRST)
    out = {"workload": "%d Poisson requests per rate over 16 seeded scenes of %d-%d tris (binary16 2048x1024 HDRI); "
                       "log-normal res 256^2..1920x1080, spp 4..256, depth 12, random camera azimuth, -dmis -emis, "
                       "150 GB HBM budget" % (requests, min(tris), max(tris)), "rates": {}}
    eng_images = None
    for rate in rates:
        reqs = [dict(r, arrival_ms=r["arrival_ms"] * rates[0] / rate) for r in base]
        eng = serving.serve_engine(E, reqs, keep_images=(eng_images is None))
        if eng_images is None:
            eng_images = eng.pop("images")
        out["rates"][str(int(rate))] = {"engine": eng}
    E.close()
    res = [lx.ResidentScene(sc, opt) for sc in scenes]
    service, same, samples = [], 0, 0.0
    t_all = time.perf_counter()
    for i, r in enumerate(sorted(base, key=lambda q: q["arrival_ms"])):
        t0 = time.perf_counter()
        rr = lx.Renderer(res[r["scene"]], default_options(direct_light_sampling=1, env_importance_sampling=1,
                                                          trace_depth=r["depth"]), camera=r["camera"])
        rr.render(1, r["spp"])
        img = rr.image_sum()
        rr.close()
        service.append((time.perf_counter() - t0) * 1e3)
        same += int(np.array_equal(img.view(np.uint32), eng_images[i].view(np.uint32)))
        samples += r["camera"].width * r["camera"].height * r["spp"]
    busy = time.perf_counter() - t_all
    for rr in res:
        rr.close()
    for sc in scenes:
        sc.close()
    arr = sorted(q["arrival_ms"] for q in base)
    for rate in rates:
        a = [x * rates[0] / rate for x in arr]
        lat = fcfs_latencies(a, service)
        p = serving.percentiles(lat)
        wall = max(x + l for x, l in zip(a, lat))
        p.update(samples_per_s=samples / (wall * 1e-3), wall_ms=wall)
        d = out["rates"][str(int(rate))]
        d["plain_fcfs"] = p
        d["p99_ratio_plain_over_engine"] = p["p99_ms"] / d["engine"]["p99_ms"]
        d["throughput_ratio"] = d["engine"]["samples_per_s"] / p["samples_per_s"]
    out["plain_service_ms_mean"] = float(np.mean(service))
    out["plain_busy_s"] = busy
    out["identical_images"] = f"{same}/{len(base)}"
    out["capacity_req_per_s"] = {"plain": 1000.0 / float(np.mean(service))}
    return out


def run_precision(spp: int = 1024, fp64_spp: int = 4096, crop: int = 32):
    """The precision form on its own workload: the 1M-triangle generator scaled to 4M triangles,
    binary16 textures and HDRI, FP64 light CDFs, compensated accumulation.
      * throughput: 1920x1080 at 1024 spp, precision form and plain FP32 path on the same scene;
      * error against the FP64 integrator (the oracle run in double on the host cores):
        a 256x256 view of the same scene (the generator's camera, field of view narrowed to a
        256x256 window around the centre) at 4096 spp on the GPU in both forms; the FP64
        integrator renders a crop x crop centre window of it at 4096 spp with the same random
        streams. relMSE of each form against it, and the time of each form at 4096 spp (equal
        samples take equal time here, so equal time is equal spp)."""
    import luxion_b200 as lx
    from luxion_b200 import _ffi
    from luxion_b200._ffi import default_options
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    sc = lx.random_scene(seed=0, total_tris=4_000_000, num_instances=200, min_tris=5000, max_tris=80000,
                         tex_half=1, env_half=1)
    out = {"workload": "4M tris / 200 instances, 1920x1080, %d spp, depth 12, -dmis -emis, seed 0" % spp}
    forms = (("precision", default_options(direct_light_sampling=1, env_importance_sampling=1,
                                           precision=_ffi.PRECISION_COMPENSATED,
                                           texture_storage=_ffi.TEXSTORE_HALF)),
             ("plain_fp32", default_options(direct_light_sampling=1, env_importance_sampling=1)))
    imgs = {}
    for name, opt in forms:
        r = lx.Renderer(sc, opt)
        r.render(1, 4)      # warm-up: graph capture
        r.reset()
        r.render(1, spp)
        st = r.stats()
        imgs[name] = r.image_sum().astype(np.float64)
        r.close()
        out[name] = {"ms": st["ms_total"], "samples_per_s": st["samples"] / (st["ms_total"] * 1e-3),
                     "mrays_per_s": (st["rays_radiance"] + st["rays_shadow"]) / (st["ms_total"] * 1e-3) / 1e6}
    a, b = imgs["precision"], imgs["plain_fp32"]
    out["relmse_precision_vs_plain"] = float(np.mean((a - b) ** 2) / np.mean(b ** 2))
    # the 256x256 view: same position and direction, field of view of the centre 256 rows of 1080
    W0, H0 = sc.width, sc.height
    fov = 2.0 * np.degrees(np.arctan(np.tan(np.radians(45.0) / 2.0) * 256.0 / H0))
    cam = lx.make_camera(256, 256, (0.0, 7.0, 25.0), (0.0, 1.0, 0.0), float(fov))
    saved = _with_camera(sc, cam)
    try:
        o64 = ol.OracleScene(sc, cdf_f64=1, tex_storage=_ffi.TEXSTORE_HALF)
        x0 = (256 - crop) // 2
        t0 = time.perf_counter()
        ref, _ = o64.render(forms[0][1], 1, fp64_spp, crop=(x0, x0, crop, crop), f64=True)
        t_ref = time.perf_counter() - t0
        o64.close()
        errs = {}
        for name, opt in forms:
            R = lx.ResidentScene(sc, opt)
            r = lx.Renderer(R, opt)
            r.render(1, fp64_spp)
            st = r.stats()
            img = r.image_sum().astype(np.float64)[x0:x0 + crop, x0:x0 + crop]
            r.close()
            R.close()
            ref64 = ref.astype(np.float64)
            errs[name] = {"relmse_vs_fp64": float(np.mean((img - ref64) ** 2) / np.mean(ref64 ** 2)),
                          "ms_256x256_%dspp" % fp64_spp: st["ms_total"]}
    finally:
        sc.desc.camera = saved
    out["vs_fp64"] = dict(errs, sample="%dx%d centre crop of a 256x256 view, %d spp, same random streams; FP64 "
                                        "integrator on %d host threads in %.1f s" % (crop, crop, fp64_spp,
                                                                                      os.cpu_count(), t_ref))
    out["instanced_tris"] = sc.instanced_tris
    sc.close()
    return out


def scene_arrays(scene):
    """(address, bytes) of every host array of a scene description: its inputs."""
    d = scene.desc
    out = []
    for i in range(d.num_meshes):
        m = d.meshes[i]
        for p, nb in ((m.positions, m.num_verts * 12), (m.normals, m.num_verts * 12), (m.uvs, m.num_verts * 8),
                      (m.indices, m.num_tris * 12)):
            a = ctypes.cast(p, ctypes.c_void_p).value
            if a:
                out.append((a, nb))
    for i in range(d.num_textures):
        t = d.textures[i]
        per = {0: 4, 1: 8, 2: 16, 3: 8}[t.format]
        out.append((ctypes.cast(t.data, ctypes.c_void_p).value, t.width * t.height * per))
    if d.env_data:
        out.append((ctypes.cast(d.env_data, ctypes.c_void_p).value, d.env_width * d.env_height * (16 if d.env_format == 2 else 8)))
    return out


def scene_bytes(scene):
    d = scene.desc
    return sum(nb for _, nb in scene_arrays(scene)) + d.num_instances * ctypes.sizeof(d.instances[0]) + \
        d.num_materials * ctypes.sizeof(d.materials[0])


def pin_scene(scene):
    """Page-lock the scene's host arrays (cudaHostRegister), so uploads run at DMA speed."""
    import torch
    done = []
    for a, nb in scene_arrays(scene):
        if torch._C._cudart.cudaHostRegister(a, nb, 0) == 0:
            done.append(a)
    return done


def unpin(addrs):
    import torch
    for a in addrs:
        torch._C._cudart.cudaHostUnregister(a)


def make_scene():
    import luxion_b200 as lx
    return lx.random_scene(seed=0)


class ClockSampler:
    """nvidia-smi sampling during the timed region (every 200 ms)."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        try:
            rows = [ln.split(",") for ln in open(self.path).read().strip().splitlines() if ln.strip()]
            os.unlink(self.path)
        except Exception:
            return out
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(nm)
            except Exception:
                continue
        if sm:
            out["sm_mhz"] = float(np.median(sm))
            out["sm_max_mhz"] = float(max(mx))
            out["samples"] = len(sm)
        out["reasons"] = sorted(reasons)
        return out


class CpuArm:
    """The reference's own render-path sources built for the host (oracle/_ref; the oracle
    port when that build is absent), OpenMP over pixel rows, on a centre crop of the frame."""

    def __init__(self, scene, threads: int = 0):
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_lib as ol
        from luxion_b200._ffi import default_options
        self.opt = default_options(direct_light_sampling=1, env_importance_sampling=1)
        self.kind = "reference" if ol.ref_available() else "port"
        self.sc = ol.RefScene(scene) if self.kind == "reference" else ol.OracleScene(scene)
        self.W, self.H = scene.width, scene.height
        self.threads = threads or os.cpu_count()
        self.side = 16

    def run(self, it: int = 1):
        x0, y0 = (self.W - self.side) // 2, (self.H - self.side) // 2
        t0 = time.perf_counter()
        _, st = self.sc.render(self.opt, it, 1, crop=(x0, y0, self.side, self.side), threads=self.threads)
        return time.perf_counter() - t0, st

    def calibrate(self, budget_s: float):
        """Grow the crop until one run takes about budget_s."""
        while True:
            el, _ = self.run()
            if el > budget_s / 4 or self.side * 2 > min(self.W, self.H):
                break
            self.side *= 2
        return el

    def measure(self, it: int = 1):
        el, st = self.run(it)
        rays = float(st[0] + st[1])
        info = {"kind": self.kind, "cores": self.threads,
                "sample": f"{self.side}x{self.side} centre crop of the 1920x1080 frame, 1 spp: {int(st[0])} radiance + "
                          f"{int(st[1])} shadow rays in {el:.2f} s"}
        return rays / el / 1e6, float(st[3]) / el, info


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    arm = CpuArm(make_scene())
    arm.calibrate(8.0)
    vals = []
    info = None
    for k in range(args.warmup + args.steps):
        mr, sps, info = arm.measure(it=1 + k)
        if k >= args.warmup:
            vals.append(mr)
    v = float(np.mean(vals))
    line = {"metric": METRIC, "value": v, "unit": "Mrays/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "impl": "reference", "config": {"workload": WORKLOAD, "arm": "host build of the reference render path"},
            "cpu_baseline": dict(info, value=v, unit="Mrays/s"),
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-forms", action="store_true")
    ap.add_argument("--forms-only", action="store_true", help="run only the batched and served forms")
    ap.add_argument("--serve-requests", type=int, default=256)
    ap.add_argument("--fp64-crop", type=int, default=32, help="side of the FP64-integrator crop (precision form)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    if args.forms_only:
        print(json.dumps({"precision": run_precision(crop=args.fp64_crop), "batched": run_batched(),
                          "served": run_served(requests=args.serve_requests)}), flush=True)
        return

    import torch
    import torch.distributed as dist
    import luxion_b200 as lx
    from luxion_b200._ffi import default_options

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    stream = torch.cuda.current_stream()
    scene = make_scene()
    opt = default_options(direct_light_sampling=1, env_importance_sampling=1, device=local,
                          stream=stream.cuda_stream)
    r = lx.Renderer(scene, opt)
    W, H = scene.width, scene.height
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    img_dev = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda") if world > 1 else None

    def step(k):
        r.reset()
        r.render(1 + (rank * 1000 + k) * SPP, SPP)

    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    rays = 0.0
    launches = 0
    ms = []
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        for k in range(args.steps):
            flush.fill_(float(k))  # L2 flush between steps, outside the step's events
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step(args.warmup + k)
            if world > 1:
                # combine the ranks' sample sums (the one collective of the sharded path),
                # device to device: copy into a torch tensor on the same stream, all-reduce
                r.copy_image_device(img_dev.data_ptr())
                dist.all_reduce(img_dev)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
            st = r.stats()
            rays += st["rays_radiance"] + st["rays_shadow"]
            launches += int(st["kernel_launches"])
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
    clocks = clk.summary()
    t_local = float(np.sum(ms))
    if world > 1:
        tt = torch.tensor([t_local, rays], dtype=torch.float64, device="cuda")
        tmax = tt.clone()
        dist.all_reduce(tmax[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(tt[1:], op=dist.ReduceOp.SUM)
        t_all, rays_all = float(tmax[0]), float(tt[1])
    else:
        t_all, rays_all = t_local, rays
    value = rays_all / (t_all * 1e-3) / 1e6
    ms_per_step = t_all / args.steps

    # per-kernel device times for the roofline (a separate timed pass: events around kernels)
    r.enable_timing(True)
    r.reset()
    r.render(1, SPP)
    kt = r.stats()
    r.enable_timing(False)
    hbm, peak_kind = peaks()
    trace_bytes = TRACE_BYTES_PER_BOUNCE * kt["path_bounces"]
    trace_ms_per_launch = kt["ms_trace"] / max(1.0, kt["launches_trace"])
    trace_bytes_per_launch = trace_bytes / max(1.0, kt["launches_trace"])
    ach = trace_bytes_per_launch / (trace_ms_per_launch * 1e-3) / 1e9
    shade_bytes = SHADE_BYTES_PER_BOUNCE * kt["path_bounces"]
    shade_ach = shade_bytes / (kt["ms_shade"] * 1e-3) / 1e9
    # measured DRAM bytes per traced ray (ncu, profiles/trace_traffic.json) times this run's
    # rays per traversal launch (a launch covers every wave in flight)
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "trace_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            per_ray = json.load(f).get("bytes_per_ray_measured")
        if per_ray:
            rays_per_launch = (kt["rays_radiance"] + kt["rays_shadow"]) / max(1.0, kt["launches_trace"])
            traffic = per_ray * rays_per_launch
    roof = {"bound": "hbm", "kernel": "k_trace (radiance + shadow)", "achieved": ach, "peak": hbm,
            "unit": "GB/s", "frac": ach / hbm, "traffic": traffic, "peak_source": f"{peak_kind} MEASURED_PEAKS hbm_gbs",
            "launch_ms": trace_ms_per_launch, "algorithmic_bytes_per_launch": trace_bytes_per_launch,
            "note": "traversal is latency/L2 bound; BVH node and triangle reads are not counted as "
                    "algorithmic bytes"}
    roof_shade = {"bound": "hbm", "kernel": "k_shade", "achieved": shade_ach, "peak": hbm, "unit": "GB/s",
                  "frac": shade_ach / hbm}
    breakdown = {k: kt[k] for k in ("ms_total", "ms_trace", "ms_shade", "ms_camera", "ms_accum", "ms_sort")}

    # end to end through the C-ABI from host buffers (cold: upload + build + render + readback),
    # with the scene's host arrays page-locked (registered once, outside the timed region)
    e2e = None
    e2e_resident = None
    if not args.no_e2e:
        r.close()
        pinned = pin_scene(scene)
        e_ms, e_rays = [], 0.0
        img_host = np.empty((H, W, 3), np.float32)
        if torch._C._cudart.cudaHostRegister(img_host.ctypes.data, img_host.nbytes, 0) == 0:
            pinned.append(img_host.ctypes.data)  # the result lands in page-locked memory too
        for k in range(3):  # the fastest of three cold runs: host-side init varies from run to run
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rr = lx.Renderer(scene, opt)
            t_init = time.perf_counter()
            rr.render(1 + rank * SPP, SPP)
            rr.image_sum_into(img_host)
            t_copy = time.perf_counter()
            st = rr.stats()
            stages = rr.scene_stats()
            rr.close()
            torch.cuda.synchronize()
            e_ms.append((time.perf_counter() - t0) * 1e3)
            if e_ms[-1] == min(e_ms):
                split = {"lux_init_ms": (t_init - t0) * 1e3, "render_and_copy_ms": (t_copy - t_init) * 1e3,
                         "lux_free_ms": (time.perf_counter() - t_copy) * 1e3,
                         "scene_build_stages_ms": {k: round(v, 2) for k, v in stages.items() if k.startswith("ms_")}}
            e_rays = st["rays_radiance"] + st["rays_shadow"]
        h2d = scene_bytes(scene)
        e2e = {"value": e_rays / (min(e_ms) * 1e-3) / 1e6, "unit": "Mrays/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(W * H * 12), "ms_per_step": min(e_ms), "ms_runs": e_ms,
               "host_memory": "page-locked" if pinned else "pageable", "split": split,
               "includes": "lux_init (scene upload, device BVH8 build, light tables, textures), "
                           "lux_render 16 spp, lux_copy_image, lux_free"}
        # the drop-in's own cycle on a resident scene: pathtraceInit (lux_init_on_scene),
        # 16 samples, copyImageToHost, pathtraceFree -- the scene built once beforehand
        R = lx.ResidentScene(scene, opt)
        rr = lx.Renderer(R, opt)
        rr.render(1, 1)
        rr.close()
        e_ms = []
        for k in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rr = lx.Renderer(R, opt)
            rr.render(1 + rank * SPP, SPP)
            rr.image_sum_into(img_host)
            st = rr.stats()
            rr.close()
            torch.cuda.synchronize()
            e_ms.append((time.perf_counter() - t0) * 1e3)
        R.close()
        e2e_resident = {"value": (st["rays_radiance"] + st["rays_shadow"]) / (min(e_ms) * 1e-3) / 1e6,
                        "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": int(W * H * 12),
                        "ms_per_step": min(e_ms), "ms_runs": e_ms,
                        "includes": "lux_init_on_scene, lux_render 16 spp, lux_copy_image, lux_free on a resident scene"}
        unpin(pinned)
    else:
        r.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        arm = CpuArm(scene)
        arm.calibrate(15.0)
        mr, sps, info = arm.measure()
        cpu = dict(info, value=mr, unit="Mrays/s", samples_per_s=sps)
    batched = served = precision = None
    if rank == 0 and world == 1 and not args.no_forms:
        batched = run_batched()
        served = run_served(requests=args.serve_requests)
        precision = run_precision(crop=args.fp64_crop)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {"metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene, random-init materials)",
            "config": {"workload": WORKLOAD, "width": W, "height": H, "spp": SPP, "depth": 12,
                       "instanced_tris": scene.instanced_tris, "form": "plain wavefront",
                       "parallelism": f"spp-sharded x{world}" if world > 1 else "single GPU",
                       "l2": "256 MiB buffer written between steps, outside the step events"},
            "samples_per_s": (W * H * SPP * world) / (t_all * 1e-3),
            "roofline": roof, "roofline_shade": roof_shade, "kernel_ms_one_step": breakdown,
            "cpu_baseline": cpu, "e2e": e2e, "e2e_resident_scene": e2e_resident, "clocks": clocks,
            "gpu_launches": launches,
            "batched": batched, "served": served, "precision": precision}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
