#!/usr/bin/env python
"""Throughput of the path-tracing hot path on B200: Mpaths/s.

Workload (one "step" = one whole render job): the seeded terrain scene --
1024x1024 fBm heightfield (2,093,058 triangles) + 200 spheres (60% Cook-
Torrance, 20% Glass, 20% Lambert) lit by a 1024x512 procedural sky envmap with
a Gaussian sun -- rendered at 1920x1080, 64 spp, max path length 16, Mitchell
filter.  Paths counted = width x height x spp (132,710,400 per step), as the
reference's own rate (paths rendered in the filter margin are extra work not
counted).  Synthetic data: the scene is generated from fixed seeds.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--batch-jobs 1024] [--serve-requests 200] [--serve-rates 100]

`value` is device time (CUDA events on the engine's stream, inputs resident
in HBM) of the streaming engine (snog_engine_render, configuration picked by
snog_engine_autotune); `e2e` is the same metric through the public C ABI with
the image copied back into pinned host memory every step, wall clock;
`plain` is the drop-in renderer (snog_render_device: one job, its own launch
sequence) on the same job.  The path state and queues (several GB) exceed the
126 MB L2, so no flush is needed between steps.

After the headline (rank 0, N=1): `cornell` -- the Cornell box at 256x256,
16 spp, depth 8, one job on the plain renderer and on the engine, beside the
reference on the host cores; `isec` -- 1M random triangles and 16M rays (half
closest-hit, half any-hit) through snog_trace_device, with its roofline on
the reference's own traversal counts for a sample of the rays.  Then two
workloads, each against the plain renderer doing one job per launch sequence
on the same input:
`batched` -- 1024 independent random-triangle soups of 1k-50k triangles
(log-uniform), resolution {64,128,256}^2, spp {4,16,64}, one engine run; and
`serve` -- 8 resident scenes of 10k-8M triangles, requests at Poisson arrivals
(random scene, camera, resolution {128..1024}^2, spp {4,16,64}), p50/p95/p99
latency from arrival to the image in host memory.  The default runs the
whole stream of 2000 requests at 50 and at 2000 requests/s (the ends of the
50-2000 sweep; --serve-rates 50,200,1000,2000 adds the middle), reported in
total and per scene-size class.

Multi-GPU: the path shards trivially (independent paths); each rank renders
its own job replica (weak scaling), no collective on the data path.  Rank 0
prints one JSON line; timings are the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

WIDTH, HEIGHT, SPP, MAX_LEN = 1920, 1080, 64, 16
REF_SPP = 2          # samples per pixel of each reference step (a bounded sample of the job)
METRIC = "Mpaths/s at matched RMSE (terrain 1920x1080, 64 spp, depth 16)"


def scenes_module():
    """snogray_b200/scenes.py (numpy only), loaded from its file: the
    reference arm must not import the package, whose __init__ maps the CUDA
    library into the process."""
    import importlib.util
    if "snogray_b200.scenes" in sys.modules:
        return sys.modules["snogray_b200.scenes"]
    if "_snog_scenes_file" not in sys.modules:
        spec_ = importlib.util.spec_from_file_location("_snog_scenes_file",
                                                       os.path.join(HERE, "snogray_b200", "scenes.py"))
        mod = importlib.util.module_from_spec(spec_)
        sys.modules["_snog_scenes_file"] = mod
        spec_.loader.exec_module(mod)
    return sys.modules["_snog_scenes_file"]


def workload():
    scenes = scenes_module()
    sd = scenes.terrain_scene()
    cam = scenes.terrain_camera(WIDTH, HEIGHT)
    return sd, cam


def workload_config():
    """The `config` both arms print (the workload, nothing arm-specific)."""
    return {"workload": "terrain-2M-tris+200-spheres+sky-envmap", "width": WIDTH, "height": HEIGHT,
            "spp": SPP, "max_path_len": MAX_LEN}


def max_over_ranks(x, dist=None):
    """Max of X over the ranks of the default process group (X itself when
    DIST is None): the job's time is its slowest rank's."""
    if dist is None:
        return x
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seed(rank):
    """Each rank renders its own replica of the job with its own sample
    streams (weak scaling: the whole job's paths = ranks x paths per rank)."""
    return 1 + rank


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ---------------------------------------------------------------------------
# clocks during the timed region

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for ln in f:
                p = [x.strip() for x in ln.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# reference (CPU) runs: the snogray renderer compiled from its own sources

def ref_available():
    sys.path.insert(0, os.path.join(HERE, "oracle"))
    import spec
    return spec.have_ref("base"), spec


def run_reference(sd, cam, params, spp, repeat, threads, rows=0, row0=0):
    """Render with the reference (baseline flavour: the reference's own
    optimisation flags) REPEAT times in one process; returns the per-render
    JSON records."""
    _, spec = ref_available()
    with tempfile.TemporaryDirectory() as d:
        sp, op = os.path.join(d, "s.spec"), os.path.join(d, "o.pfm")
        spec.write_spec(sp, sd, cam, params)
        out = subprocess.run([spec.ref_binary("base"), "render", sp, op, str(threads), "0",
                              str(spp), str(row0), str(rows), str(repeat)],
                             capture_output=True, text=True, timeout=3600)
        if out.returncode != 0:
            raise RuntimeError(out.stderr[-2000:])
    return [json.loads(ln) for ln in out.stdout.splitlines() if ln.startswith("{")]


def algorithmic_bytes_per_ray(rec):
    """Bytes one query must touch by the reference's own traversal counts
    (node visits, surface tests, list entries incl. negative-cache hits):
    28 B ray in + 8 B hit out + 36 B per node (8 child ids + list head)
    + 4 B per list entry + 36 B per primitive test (three float3)."""
    nc = max(rec["scene_intersect_calls"], 1)
    ns = max(rec["scene_shadow_tests"], 1)
    closest = 36 + (36 * rec["node_calls"] + 4 * (rec["surface_tests"] + rec["neg_cache_hits"])
                    + 36 * rec["surface_tests"]) / nc
    shadow = 36 + (36 * rec["shadow_node_calls"]
                   + 4 * (rec["shadow_surface_tests"] + rec["shadow_neg_cache_hits"])
                   + 36 * rec["shadow_surface_tests"]) / ns
    return closest, shadow


# ---------------------------------------------------------------------------

def bench_reference(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return 0
    ok, _ = ref_available()
    if not ok:
        print(json.dumps({"impl": "reference", "unavailable":
                          "compiled reference (oracle/_ref/snog_ref_base) not present"}))
        return 0
    scenes = scenes_module()
    sd, cam = workload()
    params = scenes.terrain_params(WIDTH, HEIGHT, SPP)
    threads = os.cpu_count() or 1
    # Each step renders the whole image at REF_SPP samples per pixel: a
    # bounded sample of the 64-spp job (the rate per path does not depend on
    # the spp, which only repeats the same per-pixel work).
    recs = run_reference(sd, cam, params, REF_SPP, args.warmup + args.steps, threads)
    timed = recs[args.warmup:]
    secs = sum(r["seconds"] for r in timed)
    paths = sum(r["paths"] for r in timed)
    value = paths / secs * 1e-6
    ms_per_step = secs / len(timed) * 1e3
    sample = (f"{WIDTH}x{HEIGHT} (all rows) at {REF_SPP} spp per step of the {SPP}-spp job, "
              f"reference compiled with its own flags, {threads} threads")
    line = {"metric": METRIC, "value": round(value, 4), "unit": "Mpaths/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms_per_step, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(),
            "sample": {"spp_per_step": REF_SPP, "paths_per_step": int(paths / len(timed)),
                       "threads": threads},
            "cpu_baseline": {"value": round(value, 4), "unit": "Mpaths/s", "cores": threads,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": round(value, 4), "unit": "Mpaths/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def bench_isec(args, n_tri=1 << 20, n_rays=1 << 24):
    """Intersection-only batch: 1M random triangles (centroids U[0,1]^3, edges
    U(0.002, 0.02), random orientation), 16M rays (origins U[-0.1,1.1]^3,
    directions uniform on the sphere, t_max = inf), half closest-hit, half
    any-hit.  Returns a dict (Mrays/s, per-launch ms, roofline)."""
    import torch
    import snogray_b200 as sb
    from snogray_b200 import scenes
    n_rays = args.isec_rays or n_rays
    sd = scenes.random_triangles(n_tri, seed=2)
    sc = sb.Scene(sd)
    rays = torch.from_numpy(scenes.random_rays(n_rays, seed=3)).cuda()
    prim = torch.empty(n_rays, dtype=torch.int32, device="cuda")
    tt = torch.empty(n_rays, dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    nc = n_rays // 2
    for _ in range(3):
        sc.trace_device(rays.data_ptr(), n_rays, nc, prim.data_ptr(), tt.data_ptr(), None,
                        stream.cuda_stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 5
    e0.record(stream)
    for _ in range(reps):
        sc.trace_device(rays.data_ptr(), n_rays, nc, prim.data_ptr(), tt.data_ptr(), None,
                        stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    half = 65536
    sample = torch.cat([rays[:, :half], rays[:, nc:nc + half]], 1).cpu().numpy()
    _, _, _, cnt = sc.trace(sample, half)
    out = {"workload": f"{n_tri} random triangles, {n_rays} rays (half closest, half any)",
           "mrays_per_s": round(n_rays / ms * 1e-3, 2), "ms_per_launch": round(ms, 3),
           "hit_rate_closest": round(float((prim[:nc] >= 0).float().mean()), 4),
           "nodes_per_ray": round((cnt["closest_nodes"] + cnt["any_nodes"]) / (2 * half), 2),
           "tests_per_ray": round((cnt["closest_tests"] + cnt["any_tests"]) / (2 * half), 2)}
    sc.close()
    # Roofline on the reference's own traversal counts for the same rays
    # (a sample of each half): bytes per query as for the path tracer.
    ok, spec = ref_available()
    if ok:
        _, _, _, st, _ = spec.ref_trace(sd, sample, half, threads=os.cpu_count() or 8, flavour="base")
        b = []
        for kind in ("closest", "any"):
            c = st[kind]
            b.append(36 + (36 * c["node_calls"] + 4 * (c["surface_tests"] + c["neg_cache_hits"])
                           + 36 * c["surface_tests"]) / half)
        alg = b[0] * nc + b[1] * (n_rays - nc)
        achieved = alg / (ms * 1e-3) / 1e9
        peak, src = hbm_peak()
        out["roofline"] = {"bound": "hbm", "kernel": "k_trace_batch", "achieved": round(achieved, 1),
                           "peak": peak, "peak_source": src, "unit": "GB/s", "frac": round(achieved / peak, 4),
                           "bytes_per_ray": {"closest": round(b[0], 1), "any": round(b[1], 1)},
                           "bytes_source": "reference traversal counts (RenderStats::IsecStats) on "
                                           f"{2 * half} of the rays"}
    return out


def hbm_peak():
    """The measured copy bandwidth (MEASURED_PEAKS.json), else the fallback."""
    pk_path = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(pk_path):
        with open(pk_path) as f:
            peaks = json.load(f)
        if "hbm_gbs" in peaks:
            return float(peaks["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def bench_cornell(args, sb, scenes, torch, stream, reps=5):
    """The Cornell workload at its stated size (256x256, 16 spp, max depth 8):
    one job on the plain renderer and on the streaming engine, device time
    per job, and the reference on the host's cores."""
    w = h = 256
    spp = 16
    sd = scenes.cornell_box()
    cam = scenes.cornell_camera(w, h)
    params = scenes.cornell_params(w, h, spp, seed=1)
    sc = sb.Scene(sd)
    out = torch.empty((h, w, 3), dtype=torch.float32, device="cuda")
    sptr = stream.cuda_stream
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(3):
        sc.render_device(cam, params, out.data_ptr(), sptr)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        sc.render_device(cam, params, out.data_ptr(), sptr)
    e1.record(stream)
    torch.cuda.synchronize()
    plain_ms = e0.elapsed_time(e1) / reps
    job = [(sc, cam, params)]
    with sb.Engine(sb.engine_config(max_lights=1, slots=1 << 20), stream=sptr) as eng:
        for _ in range(3):
            eng.render(job, device_outs=[out.data_ptr()])
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            eng.render(job, device_outs=[out.data_ptr()])
        e1.record(stream)
        torch.cuda.synchronize()
    eng_ms = e0.elapsed_time(e1) / reps
    sc.close()
    paths = w * h * spp
    res = {"workload": "Cornell box (10 tris, Lambert + Glass spheres, 0.25x0.25 area light), 256x256, "
                       "16 spp, depth 8", "paths": paths,
           "plain_mpaths_per_s": round(paths / plain_ms * 1e-3, 2), "plain_ms": round(plain_ms, 3),
           "engine_mpaths_per_s": round(paths / eng_ms * 1e-3, 2), "engine_ms": round(eng_ms, 3)}
    ok, _ = ref_available()
    if ok and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        r = run_reference(sd, cam, params, spp, 2, threads)[-1]
        res["reference_cpu"] = {"mpaths_per_s": round(r["mpaths_per_s"], 3), "cores": threads,
                                "seconds": round(r["seconds"], 3)}
    return res


def _cfg_dict(cfg):
    return {f: getattr(cfg, f) for f, _ in cfg._fields_ if f != "reserved"}


def _pct(xs, q):
    return round(float(np.percentile(np.asarray(xs), q)), 2) if len(xs) else None


def read_traffic_per_ray():
    """DRAM bytes per closest-hit ray of the engine's traversal kernel, from
    the committed ncu summary (one capture of the same kernel on a smaller
    terrain render; traffic scales with rays)."""
    path = os.path.join(HERE, "profiles", "k_e_closest_terrain.md")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        for ln in f:
            if ln.startswith("dram_bytes_per_ray:"):
                return float(ln.split(":", 1)[1])
    return None


def bench_batch(args, sb, scenes, torch, stream):
    """Batched workload: 1024 independent soups of 1k-50k triangles
    (log-uniform), resolution from {64,128,256}^2, spp from {4,16,64}, all in
    one engine run, beside the plain renderer doing one job after another."""
    t0 = time.perf_counter()
    work = scenes.batch_workload(args.batch_jobs)
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    handles = [sb.Scene(sd) for sd, _, _ in work]
    build_s = time.perf_counter() - t0
    jobs = [(h, cam, p) for h, (_, cam, p) in zip(handles, work)]
    paths = sum(p.width * p.height * p.spp for _, _, p in jobs)
    outs = [torch.empty((p.height, p.width, 3), dtype=torch.float32, device="cuda") for _, _, p in jobs]
    ptrs = [o.data_ptr() for o in outs]
    t0 = time.perf_counter()
    cfg, _ = sb.autotune(jobs, sample_jobs=64)
    tune_s = time.perf_counter() - t0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with sb.Engine(cfg, stream=stream.cuda_stream) as eng:
        eng.render(jobs, device_outs=ptrs)        # warm: graph, job-buffer cache
        torch.cuda.synchronize()
        e0.record(stream)
        _, st = eng.render(jobs, device_outs=ptrs)
        e1.record(stream)
        torch.cuda.synchronize()
    eng_ms = e0.elapsed_time(e1)
    # plain: one render call per job, in order, same stream
    plain_outs = [torch.empty_like(o) for o in outs]
    for k in range(min(3, len(jobs))):       # pool and kernels warm
        jobs[k][0].render_device(jobs[k][1], jobs[k][2], plain_outs[k].data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    e0.record(stream)
    for (h, cam, p), o in zip(jobs, plain_outs):
        h.render_device(cam, p, o.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    plain_ms = e0.elapsed_time(e1)
    n_off = sum(not torch.allclose(a, b, rtol=1e-4, atol=1e-5) for a, b in zip(outs, plain_outs))
    worst = max(float(((a - b).abs() / (b.abs() + 1e-3)).max()) for a, b in zip(outs, plain_outs))
    for h in handles:
        h.close()
    return {"workload": f"{len(jobs)} random-triangle soups (1k-50k tris, log-uniform), "
                        "res {64,128,256}^2, spp {4,16,64}, one area light each",
            "paths": paths, "triangles": int(sum(len(sd.triangles) for sd, _, _ in work)),
            "engine_mpaths_per_s": round(paths / eng_ms * 1e-3, 2),
            "plain_mpaths_per_s": round(paths / plain_ms * 1e-3, 2),
            "speedup_vs_plain": round(plain_ms / eng_ms, 3),
            "engine_ms": round(eng_ms, 1), "plain_ms": round(plain_ms, 1),
            "engine_mrays_per_s": round((st["closest_rays"] + st["shadow_rays"]) / eng_ms * 1e-3, 2),
            "images_vs_plain": {"jobs_outside_rtol_1e-4": int(n_off),
                                "max_rel_diff": round(worst, 6)},
            "autotuned": _cfg_dict(cfg),
            "setup_s": {"generate": round(gen_s, 1), "octree_build_upload": round(build_s, 1),
                        "autotune": round(tune_s, 1)}}


def bench_serve(args, sb, scenes):
    """Serving workload: 8 resident soups (10k-8M triangles), requests at
    Poisson arrivals, each a random scene / camera / resolution / spp.  The
    server (continuous batching) and the plain renderer (one job per launch,
    first come first served) get the same request stream; latency is arrival
    to result in host memory."""
    import threading
    t0 = time.perf_counter()
    sds = scenes.serve_scenes()
    handles = [sb.Scene(sd) for sd in sds]
    setup_s = time.perf_counter() - t0
    out = {"workload": "8 resident random-triangle scenes (10k,50k,200k,1M,2M,4M,6M,8M tris; "
                       "area light or sky envmap), Poisson arrivals, res {128,256,512,1024}^2, "
                       "spp {4,16,64}, 120 GB admission budget",
           "requests": args.serve_requests, "setup_s": round(setup_s, 1), "rates": []}
    # warm the plain path and the kernels once per scene
    for h in handles:
        h.render(scenes.orbit_camera(32, 32, np.random.default_rng(0)), sb.RenderParams(32, 32, 1))
    for rate in args.serve_rates:
        reqs = scenes.serve_requests(args.serve_requests, rate)
        paths = sum(r.params.width * r.params.height * r.params.spp for r in reqs)
        # ---- served: continuous batching --------------------------------
        cfg = sb.engine_config(max_lights=4, mem_budget=120 << 30)
        with sb.Server(cfg) as srv:
            slots = [srv.add_scene(h) for h in handles]
            ids = []
            t_start = time.perf_counter()
            for r in reqs:
                dt = r.arrival_s - (time.perf_counter() - t_start)
                if dt > 0:
                    time.sleep(dt)
                ids.append(srv.submit(slots[r.scene], r.camera, r.params))
            res = [srv.wait(j, timeout_ms=600000)[1] for j in ids]
        lat_s = [st["finish_ms"] - st["submit_ms"] for st in res]
        span_s = (max(st["finish_ms"] for st in res) - min(st["submit_ms"] for st in res)) * 1e-3
        # ---- plain: one job per launch, FIFO ------------------------------
        lat_p = []
        lock = threading.Lock()
        t_start = time.perf_counter()
        for r in reqs:
            now = time.perf_counter() - t_start
            if now < r.arrival_s:
                time.sleep(r.arrival_s - now)
            handles[r.scene].render(r.camera, r.params)
            with lock:
                lat_p.append((time.perf_counter() - t_start - r.arrival_s) * 1e3)
        span_p = time.perf_counter() - t_start
        # per scene-size class: where the served path gains or loses
        by_class = {}
        for k, n_tri in enumerate(scenes.SERVE_SIZES):
            idx = [i for i, r in enumerate(reqs) if r.scene == k]
            if not idx:
                continue
            by_class[str(n_tri)] = {
                "requests": len(idx),
                "paths": int(sum(reqs[i].params.width * reqs[i].params.height * reqs[i].params.spp
                                 for i in idx)),
                "served_p50_ms": _pct([lat_s[i] for i in idx], 50),
                "served_p99_ms": _pct([lat_s[i] for i in idx], 99),
                "plain_p50_ms": _pct([lat_p[i] for i in idx], 50),
                "plain_p99_ms": _pct([lat_p[i] for i in idx], 99)}
        out["rates"].append({
            "rate_req_per_s": rate, "paths": paths,
            "served": {"p50_ms": _pct(lat_s, 50), "p95_ms": _pct(lat_s, 95), "p99_ms": _pct(lat_s, 99),
                       "mpaths_per_s": round(paths / span_s * 1e-6, 2), "makespan_s": round(span_s, 2)},
            "plain": {"p50_ms": _pct(lat_p, 50), "p95_ms": _pct(lat_p, 95), "p99_ms": _pct(lat_p, 99),
                      "mpaths_per_s": round(paths / span_p * 1e-6, 2), "makespan_s": round(span_p, 2)},
            "by_scene_triangles": by_class})
    for h in handles:
        h.close()
    return out


def bench_ours(args):
    import ctypes

    import torch
    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    import snogray_b200 as sb
    from snogray_b200 import scenes
    sb.init(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist

    def barrier():
        if pg is not None:
            pg.barrier()

    sd, cam = workload()
    scene = sb.Scene(sd)
    params = scenes.terrain_params(WIDTH, HEIGHT, SPP, seed=replica_seed(rank))
    job = [(scene, cam, params)]
    out = torch.empty((HEIGHT, WIDTH, 3), dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    paths_per_step = WIDTH * HEIGHT * SPP

    # ---- engine configuration picked by the autotuner ----------------------
    if args.no_autotune:
        cfg = sb.engine_config(max_lights=max(1, scene.info()["n_lights"]))
        if args.slots:
            cfg.slots = args.slots
    else:
        cfg, _ = sb.autotune(job, sample_jobs=1)
    eng = sb.Engine(cfg, stream=sptr)

    def step():
        return eng.render(job, device_outs=[out.data_ptr()])[1]

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    # ---- timed region: device time on the engine's stream ------------------
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    launches = 0
    rays = [0, 0]
    for _ in range(args.steps):
        st = step()
        launches += st["kernel_launches"]
        rays[0] += st["closest_rays"]
        rays[1] += st["shadow_rays"]
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, pg)
    value = paths_per_step * ws / ms * 1e-3          # Mpaths/s, whole job

    # ---- the plain renderer (one job per launch sequence) on the same job --
    scene.render_device(cam, params, out.data_ptr(), sptr)
    torch.cuda.synchronize()
    e0.record(stream)
    n_plain = 2
    for _ in range(n_plain):
        scene.render_device(cam, params, out.data_ptr(), sptr)
    e1.record(stream)
    torch.cuda.synchronize()
    plain_ms = max_over_ranks(e0.elapsed_time(e1) / n_plain, pg)

    # ---- per-kernel times for the roofline (live, CUDA events) ------------
    os.environ["SNOG_PROFILE_KERNELS"] = "1"
    prof = step()
    del os.environ["SNOG_PROFILE_KERNELS"]

    # ---- e2e through the public C ABI with host buffers --------------------
    pinned = torch.empty((HEIGHT, WIDTH, 3), dtype=torch.float32, pin_memory=True)
    host = pinned.numpy()
    barrier()
    t0 = time.perf_counter()
    n_e2e = max(1, args.steps)
    for _ in range(n_e2e):
        eng.render(job, host_outs=[host])
    e2e_s = max_over_ranks((time.perf_counter() - t0) / n_e2e, pg)
    e2e_value = paths_per_step * ws / e2e_s * 1e-6
    h2d = ctypes.sizeof(sb.SnogCamera) + ctypes.sizeof(sb.SnogRenderParams)
    d2h = WIDTH * HEIGHT * 3 * 4
    eng.close()

    # ---- CPU baseline (rank 0, N=1) and algorithmic bytes ------------------
    cpu = None
    bytes_ray = None
    if rank == 0:
        ok, _ = ref_available()
        if ok and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            recs = run_reference(sd, cam, params, 2, 1, threads)
            r = recs[-1]
            bytes_ray = algorithmic_bytes_per_ray(r)
            if ws == 1:
                cpu = {"value": round(r["mpaths_per_s"], 4), "unit": "Mpaths/s", "cores": threads,
                       "kind": "reference",
                       "sample": f"{WIDTH}x{HEIGHT} at 2 spp (of {SPP}), all rows, "
                                 f"{r['seconds']:.1f} s"}
    peak, peak_src = hbm_peak()
    roofline = None
    if prof["iterations"] and prof["closest_ms"] > 0:
        per_launch_ms = prof["closest_ms"] / prof["iterations"]
        rays_per_launch = prof["closest_rays"] / prof["iterations"]
        if bytes_ray is not None:
            b_ray, src = bytes_ray[0], "reference traversal counts (RenderStats::IsecStats)"
        else:
            b_ray, src = None, "unavailable"
        traffic_ray = read_traffic_per_ray()
        device_ms = prof["closest_ms"] + prof["shadow_ms"] + prof["shade_ms"] + prof["other_ms"]
        roofline = {"bound": "hbm", "kernel": "k_e_closest", "peak": peak, "unit": "GB/s",
                    "peak_source": peak_src, "bytes_source": src,
                    "rays_per_launch": round(rays_per_launch), "ms_per_launch": round(per_launch_ms, 4),
                    "kernel_share": {k: round(prof[k + "_ms"] / max(device_ms, 1e-9), 4)
                                     for k in ("closest", "shadow", "shade", "other")}}
        if b_ray is not None:
            achieved = b_ray * rays_per_launch / (per_launch_ms * 1e-3) / 1e9
            roofline.update({"achieved": round(achieved, 1), "frac": round(achieved / peak, 4),
                             "bytes_per_ray": round(b_ray, 1)})
        else:
            roofline.update({"achieved": None, "frac": None})
        if bytes_ray is not None and prof["shadow_ms"] > 0:
            # the any-hit kernel on the same step, by the same accounting
            sh_ms = prof["shadow_ms"] / prof["iterations"]
            sh_rays = prof["shadow_rays"] / prof["iterations"]
            sh_ach = bytes_ray[1] * sh_rays / (sh_ms * 1e-3) / 1e9
            roofline["shadow"] = {"kernel": "k_e_shadow", "achieved": round(sh_ach, 1),
                                  "frac": round(sh_ach / peak, 4), "bytes_per_ray": round(bytes_ray[1], 1),
                                  "rays_per_launch": round(sh_rays), "ms_per_launch": round(sh_ms, 4)}
        roofline["traffic"] = round(traffic_ray * rays_per_launch) if traffic_ray else None
        roofline["traffic_per_ray"] = traffic_ray

    batched = serve = isec = cornell = None
    if rank == 0 and ws == 1:
        if not args.no_extra:
            cornell = bench_cornell(args, sb, scenes, torch, stream)
            isec = bench_isec(args)
        if args.batch_jobs:
            batched = bench_batch(args, sb, scenes, torch, stream)
        if args.serve_requests:
            serve = bench_serve(args, sb, scenes)

    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 4), "unit": "Mpaths/s", "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded terrain scene; inputs larger than L2, no flush)",
                "config": workload_config(),
                "parallelism": f"replicas x{ws}", "l2": "working set > L2 (no flush needed)",
                "engine": _cfg_dict(cfg),
                "gpu_launches": launches,
                "e2e": {"value": round(e2e_value, 4), "unit": "Mpaths/s", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h},
                "plain": {"value": round(paths_per_step * ws / plain_ms * 1e-3, 4), "unit": "Mpaths/s",
                          "ms_per_step": round(plain_ms, 3)},
                "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
                "rays": {"closest_per_step": rays[0] // max(args.steps, 1),
                         "shadow_per_step": rays[1] // max(args.steps, 1),
                         "mrays_per_s": round((rays[0] + rays[1]) * ws / (ms * args.steps) * 1e-3, 2)},
                "cornell": cornell, "isec": isec, "batched": batched, "serve": serve}
        print(json.dumps(line))
    scene.close()
    if pg is not None:
        pg.destroy_process_group()
    return 0


def main():
    global WIDTH, HEIGHT, SPP
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--width", type=int, default=WIDTH, help="smaller case for profiling only")
    ap.add_argument("--height", type=int, default=HEIGHT)
    ap.add_argument("--spp", type=int, default=SPP)
    ap.add_argument("--isec-only", action="store_true",
                    help="only the intersection-only batch (1M triangles, 16M rays)")
    ap.add_argument("--isec-rays", type=int, default=0)
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the Cornell and intersection-only workloads after the headline")
    ap.add_argument("--no-autotune", action="store_true",
                    help="default engine configuration (profiling runs)")
    ap.add_argument("--slots", type=int, default=0, help="engine queue slots with --no-autotune")
    ap.add_argument("--batch-jobs", type=int, default=1024,
                    help="jobs of the batched workload (0 = skip it)")
    ap.add_argument("--serve-requests", type=int, default=2000,
                    help="requests of the serving workload per rate (0 = skip it)")
    ap.add_argument("--serve-rates", type=str, default="50,2000",
                    help="comma-separated Poisson arrival rates, requests/s")
    args = ap.parse_args()
    args.serve_rates = [float(x) for x in args.serve_rates.split(",") if x]
    WIDTH, HEIGHT, SPP = args.width, args.height, args.spp
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return bench_reference(args)
    if args.isec_only:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps({"isec": bench_isec(args)}))
        return 0
    return bench_ours(args)


if __name__ == "__main__":
    sys.exit(main())
