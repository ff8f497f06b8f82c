"""Request loop of the serving form, and the plain single-job baseline it is compared with.

serve_engine(): replays a stream of timed requests against a job engine in real time. Requests
that have arrived are submitted between waves; the engine admits them against its HBM budget
and batches them into the shared wavefront with the work already on the device; each finished
job's image is read back and its device memory released. A request's latency runs from its
arrival to the end of the wave that completed it, on the engine clock.

serve_plain(): the same stream through the reference-shaped single-job path, first come first
served: for each request a context is created for its scene and camera (lux_init), the samples
are rendered (lux_render), the image read back and the context freed.
"""
from __future__ import annotations

import time
from typing import List

import numpy as np

from . import Engine, Renderer, default_options


def percentiles(lat_ms) -> dict:
    a = np.asarray(lat_ms, np.float64)
    return {"p50_ms": float(np.percentile(a, 50)), "p95_ms": float(np.percentile(a, 95)),
            "p99_ms": float(np.percentile(a, 99)), "mean_ms": float(a.mean()), "max_ms": float(a.max())}


def serve_engine(engine: Engine, requests: List[dict], keep_images: bool = False) -> dict:
    reqs = sorted(requests, key=lambda r: r["arrival_ms"])
    t0 = engine.clock_ms()
    nxt, live, lat, images = 0, {}, [None] * len(reqs), {}
    samples = 0.0
    st0 = engine.stats()
    while nxt < len(reqs) or live:
        now = engine.clock_ms() - t0
        while nxt < len(reqs) and reqs[nxt]["arrival_ms"] <= now:
            r = reqs[nxt]
            jid = engine.submit(r["scene"], r["spp"], trace_depth=r["depth"], camera=r["camera"])
            live[jid] = nxt
            nxt += 1
        done, idle = engine.step()
        if idle and nxt < len(reqs):
            wait = reqs[nxt]["arrival_ms"] - (engine.clock_ms() - t0)
            if wait > 0:
                time.sleep(wait / 1000.0)
            continue
        if done:
            found = 0  # the step finished `done` jobs: stop looking once they are all collected
            for jid in list(live):
                s = engine.status(jid)
                if s["state"] == 2:  # LUX_JOB_DONE
                    i = live.pop(jid)
                    lat[i] = s["t_done_ms"] - t0 - reqs[i]["arrival_ms"]
                    img = engine.image(jid)
                    if keep_images:
                        images[i] = img
                    samples += reqs[i]["camera"].width * reqs[i]["camera"].height * reqs[i]["spp"]
                    engine.release(jid)
                    found += 1
                    if found == done:
                        break
    wall = engine.clock_ms() - t0
    st = engine.stats()
    out = percentiles(lat)
    out.update(requests=len(reqs), wall_ms=wall, samples=samples, samples_per_s=samples / (wall * 1e-3),
               rays=st["rays"] - st0["rays"], mrays_per_s=(st["rays"] - st0["rays"]) / (wall * 1e-3) / 1e6,
               device_ms=st["ms_device"] - st0["ms_device"], waves=st["waves"] - st0["waves"],
               max_paths=st["max_paths"], trace_blocks=st["trace_blocks"])
    if keep_images:
        out["images"] = images
    return out


def serve_plain(scenes, requests: List[dict], options=None, keep_images: bool = False) -> dict:
    reqs = sorted(requests, key=lambda r: r["arrival_ms"])
    opt = options if options is not None else default_options()
    t0 = time.perf_counter()
    lat, images, samples, rays = [], {}, 0.0, 0.0
    for i, r in enumerate(reqs):
        now = (time.perf_counter() - t0) * 1e3
        if r["arrival_ms"] > now:
            time.sleep((r["arrival_ms"] - now) / 1000.0)
        sc = scenes[r["scene"]]
        d = sc.desc
        saved = type(d.camera).from_buffer_copy(d.camera)
        d.camera = r["camera"]
        try:
            opt.trace_depth = r["depth"]
            rr = Renderer(sc, opt)
        finally:
            d.camera = saved
        rr.render(1, r["spp"])
        img = rr.image_sum()
        rays += rr.stats()["rays_radiance"] + rr.stats()["rays_shadow"]
        rr.close()
        if keep_images:
            images[i] = img
        lat.append((time.perf_counter() - t0) * 1e3 - r["arrival_ms"])
        samples += r["camera"].width * r["camera"].height * r["spp"]
    wall = (time.perf_counter() - t0) * 1e3
    out = percentiles(lat)
    out.update(requests=len(reqs), wall_ms=wall, samples=samples, samples_per_s=samples / (wall * 1e-3), rays=rays,
               mrays_per_s=rays / (wall * 1e-3) / 1e6)
    if keep_images:
        out["images"] = images
    return out
