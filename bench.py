"""Benchmark: primary rays per second of the treelet ray cast on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]
                    [--shadow] [--no-extra] [--leg NAME]

One step = one frame of the workload cast over its resident octree.  The
device-timed ``value`` has the octree resident in HBM and times the render
kernel with CUDA events (L2 flushed between steps by writing 256 MB).
``e2e`` is the same metric through the C ABI call a user makes
(svo_mm_render_host_async): kernel plus the copy of the RGBA8 image back to
pinned host memory, every step, with the L2 flush inside the wall-clock time.  ``roofline`` relates the kernel's algorithmic bytes
(8 B per parent-node read, 8 B per hit attribute, 4 B per RGBA8 pixel,
counted by the kernel's own per-ray counters) to the measured HBM copy
bandwidth.  ``cpu_baseline`` times the reference's own ray cast compiled for
the host (oracle/_ref; the oracle port when that is absent) on the host cores.

With N > 1 (torchrun), each rank casts the same workload on its own GPU
(replicas: rays are independent, there is no exchange), and the step time is
the maximum over ranks.  At N = 1 the line also carries the extra legs:
flat traversal, batched views, serving, the large shadowed frame, incore
updates and the streaming loop (``--no-extra`` skips them, ``--leg NAME``
runs one alone).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

METRIC = "Mrays/s"
FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="icosphere")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the batched, served, large-shadowed and incore-update measurements")
    ap.add_argument("--leg", choices=["batched", "served", "large_shadowed", "incore_update", "streaming", "flat",
                                      "large_streaming"],
                    help="run only this measurement on one GPU and print its result: the 64 terrain "
                         "views as one batched launch, the request server, the large shadowed "
                         "frame, the incore-update policies, the streaming loop on the icosphere "
                         "scene, or the flat (CpuRaycasterSingleRay3) traversal of the main view "
                         "(--steps sets the timed repetitions of batched and large_shadowed)")
    ap.add_argument("--large-only", action="store_true",
                    help="run only the large shadowed measurement (icosphere built on the GPU, 3840x2160 "
                         "primary + shadow frame) and print its result; the same as --leg large_shadowed")
    ap.add_argument("--large-subdivisions", type=int, default=9)
    ap.add_argument("--large-depth", type=int, default=14)
    ap.add_argument("--legs-json", default=None,
                    help="also write the full records of the extra measurements to this file")
    ap.add_argument("--shadow", action="store_true",
                    help="cast one shadow ray per hit as well (svo_mm_render_shadow, seeded light); "
                         "the metric then counts primary and shadow rays")
    return ap.parse_args()


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.is_file():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def make_workload(name):
    from libsvo_b200 import scenes

    if name == "menger":
        return scenes.menger()
    if hasattr(scenes, name):
        return getattr(scenes, name)()
    raise SystemExit(f"unknown workload {name}")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 20 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.first = 0

    def start(self):
        """Starts sampling and returns once nvidia-smi is reporting (at most
        3 s), so that the samples cover the region timed next; only samples
        taken from then on count."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
            return
        t0 = time.perf_counter()
        while not self.lines and self.proc.poll() is None and time.perf_counter() - t0 < 3.0:
            time.sleep(0.005)
        self.first = len(self.lines)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[self.first:]:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference_frames(wl, nodes, attribs, seconds=10.0, max_frames=200, light=None):
    """Times the reference's renderToBuffer compiled for the host (or the
    oracle port) over whole frames of the workload, all host threads.  With
    `light`, the primary + shadow frame (the shadow shading over the
    reference's own sample()); shadow rays count as rays.  The reference's
    kernel has MAX_STACK_SIZE 13 compiled in, so octrees deeper than 12 levels
    take the oracle port with their own stack size."""
    import oracle

    threads = os.cpu_count() or 1
    ref = oracle.reference_lib() is not None and wl.stack_size == 13
    params = [bytes(c.frame_params()) for c in wl.cameras]
    # shadow rays per frame = primary hits (counted once, outside the timing)
    shadow_rays = [int(oracle.render(nodes, attribs, p, stack_size=wl.stack_size, threads=threads)[1]["hit"].sum())
                   if light is not None else 0 for p in params]
    rays = 0
    frames = 0
    t0 = time.perf_counter()
    while True:
        for p, ns in zip(params, shadow_rays):
            w, h = np.frombuffer(p[:8], dtype=np.uint32)
            rays += int(w) * int(h) + ns
            if light is not None:
                if ref:
                    oracle.reference_render_shadow(nodes, attribs, p, light, threads=threads)
                else:
                    oracle.render_shadow(nodes, attribs, p, light, stack_size=wl.stack_size, threads=threads)
            elif ref:
                oracle.reference_render(nodes, attribs, p, threads=threads)
            else:
                oracle.render(nodes, attribs, p, stack_size=wl.stack_size, threads=threads)
        frames += 1
        el = time.perf_counter() - t0
        if el >= seconds or frames >= max_frames:
            break
    return {"value": rays / el / 1e6, "unit": METRIC, "cores": threads,
            "kind": "reference" if ref else "port",
            "sample": f"{frames} whole frame(s) of the workload ({rays} rays) in {el:.1f} s; "
                      + ("reference treeletRenderer_rgba.cl renderToBuffer compiled for the host"
                         if ref else "oracle restatement of sample()")
                      + ("; primary + shadow rays" if light is not None else "")}


def reference_parity(nodes, attribs, params, gpu_rgba, gpu_hits, light=None, gpu_shadow_hits=None,
                     config="", stack_size=13):
    """Compares one GPU frame with the reference's own renderToBuffer compiled
    for the host (oracle/_ref): every pixel's RGBA8, and per ray the node
    index, depth, hit flag and loop count of the reference's sample() (primary
    rays; with `light`, the shadow rays of the shadow frame).  The oracle
    restatement (pinned to the reference at its stack of 13) stands in when
    the reference build is absent or the octree needs a deeper stack."""
    import oracle

    p = bytes(params)
    w, h = (int(v) for v in np.frombuffer(p[:8], dtype=np.uint32))
    ref = oracle.reference_lib() is not None and stack_size == 13
    fields = ("node", "depth", "hit", "loops")
    out = {"config": config, "pixels": w * h, "against": "reference" if ref else "oracle restatement"}
    if light is None:
        if ref:
            ref_rgba = oracle.to_rgba8(oracle.reference_render(nodes, attribs, p))
            o, d = oracle.pixel_rays(p)
            ref_hits = oracle.reference_sample_rays(nodes, o, d, params.t_scale_ratio)
        else:
            ref_rgba, ref_hits, _, _ = oracle.render(nodes, attribs, p, stack_size=stack_size)
        rays_ref, rays_gpu = ref_hits.reshape(-1), gpu_hits.reshape(-1)
        out["rays"] = w * h
    else:
        if ref:
            rgbaf, ref_shadow = oracle.reference_render_shadow(nodes, attribs, p, light)
            ref_rgba = oracle.to_rgba8(rgbaf)
        else:
            ref_rgba, _, ref_shadow, _, _ = oracle.render_shadow(nodes, attribs, p, light, stack_size=stack_size)
        rays_ref, rays_gpu = ref_shadow.reshape(-1), gpu_shadow_hits.reshape(-1)
        out["rays"] = int(rays_gpu["hit"].size)
        out["rays_compared"] = "shadow rays (one per primary hit; zero records elsewhere)"
    out["mismatched_rgba"] = int((gpu_rgba.reshape(-1) != ref_rgba.reshape(-1)).sum())
    out["mismatched_rays"] = int(np.any(np.stack([rays_gpu[k] != rays_ref[k] for k in fields]), axis=0).sum())
    out["mismatched"] = out["mismatched_rgba"] + out["mismatched_rays"]
    return out


def run_reference(args, wl):
    """The reference arm: the reference's renderToBuffer compiled for the host
    (oracle/_ref; the oracle port if that is absent), all host threads, on
    the same workload.  A step is one frame, or an evenly spread band of its
    rows when whole frames would make the run longer than about two minutes."""
    import libsvo_b200 as L
    import oracle

    info = wl.scene.info
    mm = L.TreeletMemoryManagerCuda(wl.scene, info.treelet_bytes * info.num_treelets)
    mm.insertAll()
    nodes, attribs = mm.getIncoreBuffer()
    threads = os.cpu_count() or 1
    ref = oracle.reference_lib() is not None
    params = [bytes(c.frame_params()) for c in wl.cameras]

    def cast(p, rows):
        if ref:
            oracle.reference_render(nodes, attribs, p, threads=threads, rows=rows)
        else:
            sub = bytearray(p)  # the port renders whole frames: shrink the frame instead
            w = int(np.frombuffer(p[:4], dtype=np.uint32)[0])
            sub[4:8] = np.uint32(rows[1] - rows[0]).tobytes()
            oracle.render(nodes, attribs, bytes(sub), stack_size=wl.stack_size, threads=threads)
            del w

    t0 = time.perf_counter()
    for p in params:
        h = int(np.frombuffer(p[4:8], dtype=np.uint32)[0])
        cast(p, (0, h))
    t_frame = time.perf_counter() - t0
    frac = min(1.0, 120.0 / max(1e-9, (args.steps + args.warmup) * t_frame))
    per = []
    for step in range(args.warmup + args.steps):
        rays = 0
        t0 = time.perf_counter()
        for p in params:
            w, h = (int(v) for v in np.frombuffer(p[:8], dtype=np.uint32))
            nrows = max(1, int(round(h * frac)))
            y0 = (step * nrows) % h
            y1 = min(h, y0 + nrows)
            cast(p, (y0, y1))
            rays += w * (y1 - y0)
        el = time.perf_counter() - t0
        if step >= args.warmup:
            per.append((rays, el))
    rays = sum(r for r, _ in per)
    secs = sum(e for _, e in per)
    value = rays / secs / 1e6
    kind = "reference" if ref else "port"
    sample = (f"{'whole frames' if frac >= 1.0 else f'{frac:.3f} of each frame (row bands)'} per step, "
              f"{rays} rays in {secs:.1f} s; "
              + ("reference treeletRenderer_rgba.cl renderToBuffer compiled for the host"
                 if ref else "oracle restatement of sample()"))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": wl.rays_per_step / value / 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generators)",
        "config": {"workload": wl.name, "description": wl.description, "rays_per_step": wl.rays_per_step},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def max_over_ranks(x: float, world: int, device) -> float:
    """The slowest rank's value (every rank takes part; world 1: x itself)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_mrays_per_s(world: int, rays_per_rank: int, ms_per_step: float) -> float:
    """Whole-job throughput: every rank casts its own replica of the step's
    rays, and the step takes the slowest rank's time."""
    return world * rays_per_rank / (ms_per_step * 1e-3) / 1e6


def _profiled_traffic(workload: str):
    """(DRAM bytes per launch of the workload's frame kernel, the capture
    they come from) from the committed ncu summaries (profiles/); (None,
    why) when no capture of the current kernel covers the workload."""
    tp = ROOT / "profiles" / "render_frame_kernel_dram_traffic.json"
    entry = json.loads(tp.read_text()).get(workload) if tp.is_file() else None
    if not isinstance(entry, dict):
        return None, "no ncu capture of this workload's kernel"
    return entry.get("bytes"), entry.get("capture")


def _kernels_per_render(p, shadow: bool) -> int:
    """Kernels of this library one render launches: the per-frame kernel,
    preceded for primary-ray frames of a million pixels or more by the
    block-cost estimate of longest-first dispatch (csrc/render.cu)."""
    return 1 if shadow or p.width * p.height < (1 << 20) else 2


def _event_ms(torch, fn, reps):
    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def batched_leg(dev, reps=10):
    """64 terrain views of uneven size (depth-12 terrain, 256^2..2048^2): the same views as
    64 per-frame launches on one stream, and as one autotuned, graph-replayed
    persistent launch."""
    import torch

    import libsvo_b200 as L
    from libsvo_b200 import scenes

    t0 = time.perf_counter()
    wl = scenes.terrain()
    info = wl.scene.info
    build_s = time.perf_counter() - t0
    mm = L.TreeletMemoryManagerCuda(wl.scene, info.treelet_bytes * info.num_treelets)
    mm.insertAll()
    mm.initDeviceBuffer()
    ps = [c.frame_params() for c in wl.cameras]
    outs = [torch.empty((p.height, p.width), dtype=torch.int32, device=dev) for p in ps]
    s = torch.cuda.current_stream()

    def per_view():
        for p, o in zip(ps, outs):
            mm.render(p, o, stream=s)

    ms_plain = _event_ms(torch, per_view, reps)
    b = L.Batcher()
    b.set([L.octree_of(mm)], [L.view_desc(p, 0, o) for p, o in zip(ps, outs)], L.batch_cfg(), stream=s)
    best, _ = b.autotune(reps=3, stream=s)
    ms_batch = _event_ms(torch, lambda: b.launch(stream=s), reps)
    rays = wl.rays_per_step
    b.close()
    mm.close()
    return {"workload": wl.name, "description": wl.description, "rays_per_step": rays,
            "scene_build_s": round(build_s, 2), "per_view_launches_mrays_s": rays / ms_plain / 1e3,
            "batched_mrays_s": rays / ms_batch / 1e3, "speedup": ms_plain / ms_batch,
            "batched_ms": ms_batch, "per_view_ms": ms_plain,
            "autotuned": {"tile": [best.tile_w, best.tile_h], "block_threads": best.block_threads,
                          "top_nodes": best.top_nodes, "rays_per_lane": best.rays_per_lane,
                          "graph": True}}


def served_leg(dev, n=400, rates=(4000, 16000, 64000)):
    """8 octrees of depths 9..13 served to a Poisson stream of requests
    from 64x64 to 1920x1080: batched server vs the plain per-frame kernel in the
    same request loop, all octrees resident; then the batched server with a
    budget of half the octrees' footprint, so octrees page in and out."""
    import numpy as np
    import torch

    import libsvo_b200 as L
    from libsvo_b200 import scenes as S

    t0 = time.perf_counter()
    wl = S.serving()
    build_s = time.perf_counter() - t0
    footprint = sum(16 * s.info.treelet_bytes // 8 * s.info.num_treelets for s in wl.scenes)
    reqs = S.serving_requests(n, len(wl.scenes), seed=3)
    outs = [torch.empty((c.height, c.width), dtype=torch.int32, device=dev) for _, c in reqs]
    rays = sum(c.width * c.height for _, c in reqs)

    def run(mode, budget, rate_list, upload=None, streams=4):
        srv = L.Server(L.server_cfg(budget, streams=streams, max_batch_views=256, mode=mode))
        ids = [srv.add_octree(s) for s in wl.scenes]
        if upload is not None:
            for i in ids:
                srv.set_upload_policy(i, upload)
        rq = [L.request(ids[o], c.frame_params(), t) for (o, c), t in zip(reqs, outs)]
        srv.replay(rq[:64], np.zeros(64), timeout_ms=120000)  # first loads
        res = {}
        for rate in rate_list:
            t_run = time.perf_counter()
            arr = S.poisson_arrivals(n, rate, seed=11) if rate else np.zeros(n)
            try:
                r = srv.replay(rq, arr, timeout_ms=60000)
            except L.SvoError:  # some requests failed: their results carry the status
                r = srv.last_replay_results
            ok = [x for x in r if x.status == L.SVO_OK]
            served_rays = sum(q.params.width * q.params.height for q, x in zip(rq, r) if x.status == L.SVO_OK)
            lat = np.array([x.done_s - x.submit_s for x in ok]) * 1e3 if ok else np.zeros(1)
            span = (max(x.done_s for x in ok) - min(x.submit_s for x in r)) if ok else float("inf")
            res[str(rate) if rate else "burst"] = {
                "mrays_s": served_rays / span / 1e6, "p50_ms": float(np.percentile(lat, 50)),
                "p99_ms": float(np.percentile(lat, 99)), "launches": len({x.batch for x in ok}),
                "failed": len(r) - len(ok)}
            print(f"[bench] served mode {mode} budget {budget / 1e9:.2f} GB rate {rate}: "
                  f"{time.perf_counter() - t_run:.1f} s", file=sys.stderr, flush=True)
        st = srv.stats()
        res["paging"] = {"octree_loads": st.octree_loads, "evictions": st.octree_evictions,
                         "treelets_paged_in": st.treelets_paged_in, "gb_uploaded": st.bytes_uploaded / 1e9,
                         "paged_unconverged": st.paged_unconverged}
        srv.close()
        return res

    all_rates = list(rates) + [0]
    # batched and ungated plain on the same 8 streams; the one-stream plain
    # loop keeps 4 slots, the reference's pattern of a blocking enqueue
    batched = run(L.SERVE_BATCHED, 2 * footprint, all_rates, streams=8)
    plain = run(L.SERVE_PLAIN, 2 * footprint, all_rates)
    # the ungated plain baseline: every admitted request's per-frame kernel
    # launched at once, round robin over 8 streams, completion by events
    ungated = run(L.SERVE_PLAIN_STREAMED, 2 * footprint, all_rates, streams=8)
    paging = run(L.SERVE_BATCHED, footprint // 2, [16000], streams=8)
    paging_pinned = run(L.SERVE_BATCHED, footprint // 2, [16000], upload=L.UPLOAD_PINNED, streams=8)
    paging_ungated = run(L.SERVE_PLAIN_STREAMED, footprint // 2, [16000], streams=8)
    paging_ungated_pinned = run(L.SERVE_PLAIN_STREAMED, footprint // 2, [16000], upload=L.UPLOAD_PINNED,
                                streams=8)
    # treelet paging under a budget below the largest octree's footprint.
    # "fits": the largest octree (1.4 GB) alone, served from 0.9x its
    # footprint, the whole budget its region, so every view's treelets fit;
    # "two_regions": the two largest octrees, each paged in half of 0.9x the
    # largest footprint (45 % of its treelets), where some views see more
    # than their region holds and are cast from what is resident.  The
    # octrees' host copies are page-locked (one gather kernel per upload).
    sizes = [16 * s.info.treelet_bytes // 8 * s.info.num_treelets for s in wl.scenes]
    big = sorted(range(len(sizes)), key=lambda i: -sizes[i])[:2]
    tp_budget = int(0.9 * max(sizes))

    def run_paged(octrees, region, rate):
        tp_reqs = [(o, c, t) for (o, c), t in zip(reqs, outs) if o in octrees]
        tp_rays = sum(c.width * c.height for _, c, _ in tp_reqs)
        srv = L.Server(L.server_cfg(tp_budget, streams=4, max_batch_views=256))
        ids = {o: srv.add_octree_paged(wl.scenes[o], region) for o in octrees}
        for i in ids.values():
            srv.set_upload_policy(i, L.UPLOAD_PINNED)
        rq = [L.request(ids[o], c.frame_params(), t) for o, c, t in tp_reqs]
        # untimed warm-up (kernel loading, scratch growth), as the other runs' first loads
        srv.replay(rq[:8], np.zeros(8), timeout_ms=120000)
        st0 = srv.stats()
        t_run = time.perf_counter()
        arr = S.poisson_arrivals(len(rq), rate, seed=13)
        r = srv.replay(rq, arr, timeout_ms=120000)
        ok = [x for x in r if x.status == L.SVO_OK]
        lat = np.array([x.done_s - x.submit_s for x in ok]) * 1e3
        span = max(x.done_s for x in ok) - min(x.submit_s for x in r)
        st1 = srv.stats()
        srv.close()
        st = type("Delta", (), {k: getattr(st1, k) - getattr(st0, k) for k in
                                ("treelets_paged_in", "bytes_uploaded", "paged_unconverged",
                                 "analysis_passes", "paging_us")})
        print(f"[bench] served treelet-paged {len(octrees)} octree(s) rate {rate}: "
              f"{time.perf_counter() - t_run:.1f} s", file=sys.stderr, flush=True)
        return {"requests": len(rq), "rays": tp_rays, "mrays_s": tp_rays / span / 1e6,
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "failed": len(r) - len(ok), "treelets_paged_in": st.treelets_paged_in,
                "gb_uploaded": st.bytes_uploaded / 1e9, "paged_unconverged": st.paged_unconverged,
                "analysis_passes": st.analysis_passes, "paging_s": st.paging_us / 1e6}

    treelet_paged = {"octrees": big, "octree_gb": [sizes[o] / 1e9 for o in big], "budget_gb": tp_budget / 1e9,
                     "fits_rate_100": run_paged(big[:1], tp_budget - 4096, 100),
                     "fits_rate_16000": run_paged(big[:1], tp_budget - 4096, 16000),
                     "two_regions_rate_16000": run_paged(big, tp_budget // 2, 16000)}
    keys = [k for k in batched if k != "paging"]
    return {"workload": wl.name, "description": wl.description, "requests": n, "rays": rays,
            "scene_build_s": round(build_s, 2), "octree_footprint_gb": footprint / 1e9,
            "budget_note": "the stand-in octrees total far less than the configuration's 40 GB cap; "
                           "the paging runs cap the pool at half their footprint",
            "batched": batched, "plain_one_stream": plain, "plain_ungated": ungated,
            "speedup_vs_plain_ungated": {k: batched[k]["mrays_s"] / ungated[k]["mrays_s"] for k in keys},
            "speedup_vs_plain_one_stream": {k: batched[k]["mrays_s"] / plain[k]["mrays_s"] for k in keys},
            "paging_half_budget": {"batched": paging, "batched_pinned_hosts": paging_pinned,
                                   "plain_ungated": paging_ungated,
                                   "plain_ungated_pinned_hosts": paging_ungated_pinned},
            "treelet_paged": treelet_paged}


def incore_update_leg(dev, scene, incore_mb=256, frames=20, seed=5):
    """The reference's incore update measurement (its thesis: 256 MB incore
    buffer, dirty slots uploaded per frame with coalescing ratio 0.6, one copy
    per slot, and ratio 0) on the icosphere scene: each frame evicts 12 MB
    worth of childless resident treelets and inserts as many treelets whose
    parent is resident, then times updateDeviceMemory until the copies
    finish.  Every policy replays the same eviction/insertion sequence."""
    import torch

    import libsvo_b200 as L

    nt = scene.info.num_treelets
    tb = scene.info.treelet_bytes
    parent = [scene.treelet(g)["parent_gid"] if g else -1 for g in range(nt)]
    kids = {}
    for g in range(1, nt):
        kids.setdefault(parent[g], []).append(g)
    policies = [("coalesced_0.6", L.UPLOAD_COALESCED, 0.6), ("one_copy_per_slot", L.UPLOAD_COALESCED, 1.0),
                ("one_range_ratio_0", L.UPLOAD_COALESCED, 0.0), ("packed_scatter", L.UPLOAD_PACKED, 0.6),
                ("pinned_mirror_gather", L.UPLOAD_PINNED, 0.6)]
    out = {"scene": "icosphere_s6_d11 (6-level treelets)", "incore_mb": incore_mb, "treelet_bytes": tb,
           "frames": frames}
    for name, policy, ratio in policies:
        mm = L.TreeletMemoryManagerCuda(scene, incore_mb << 20)
        mm.setUploadPolicy(policy)
        mm.setUploadRatio(ratio)
        mm.initDeviceBuffer()
        mm.insertAll()
        k = max(1, (12 << 20) // tb)
        resident = {g for g in range(nt) if mm.getSlotGid(g) >= 0}
        mm.updateDeviceMemory()
        torch.cuda.synchronize()
        rng = np.random.default_rng(seed)
        ms, calls, dirty, moved = [], [], [], []
        for _ in range(frames):
            leaves = sorted(g for g in resident if g and not any(c in resident for c in kids.get(g, ())))
            for g in rng.permutation(leaves)[:k].tolist():
                mm.removeTreeletFromIncoreBuffer(g)
                resident.discard(g)
            cands = sorted(g for g in range(1, nt) if g not in resident and parent[g] in resident)
            for g in rng.permutation(cands)[:k].tolist():
                if mm.insertTreeletIntoIncoreBuffer(g):
                    resident.add(g)
            ds = mm.getIncoreSlotsToUpload()
            dirty.append(len(ds))
            plan = mm.planUploads()
            moved.append(2 * tb * (len(ds) if policy != L.UPLOAD_COALESCED else sum(c for _, c in plan)))
            t0 = time.perf_counter()
            calls.append(mm.updateDeviceMemory())
            torch.cuda.synchronize()
            ms.append((time.perf_counter() - t0) * 1e3)
        mm.close()
        out[name] = {"ms_mean": statistics.mean(ms), "ms_median": statistics.median(ms),
                     "copy_calls_mean": statistics.mean(calls), "dirty_slots_mean": statistics.mean(dirty),
                     "mb_over_pcie_mean": statistics.mean(moved) / 1e6}
    out["reference_thesis_ms"] = {"coalesced_0.6": 2.48, "one_copy_per_slot": 4.23, "one_range_ratio_0": 52.51,
                                  "hardware": "GTX 580, PCIe 2 (ergebnisse_diskussionen.tex:111)"}
    return out


def streaming_leg(dev, scene, **kw):
    """streaming_run with the reference's upload policy and with the
    page-locked mirror and gather kernel."""
    import libsvo_b200 as L

    return {"coalesced_0.6": streaming_run(dev, scene, L.UPLOAD_COALESCED, **kw),
            "pinned_mirror_gather": streaming_run(dev, scene, L.UPLOAD_PINNED, **kw),
            "pinned_pipelined": streaming_run(dev, scene, L.UPLOAD_PINNED, pipelined=True, **kw),
            "reference_thesis": "mostly above 50 Hz, GTX 580 (ergebnisse_diskussionen.tex:158)"}


def streaming_run(dev, scene, policy, frames=150, incore_mb=256, size=1024, pipelined=False):
    """The loop the reference measured itself (its thesis: "out-of-core cycle
    + ray cast run sequentially, 1024x1024", mostly above 50 Hz on a GTX 580):
    per frame the analysis pass at 1/8 resolution (feedback kernel, records to
    the host, analysis, insertion with eviction, upload of the new treelets),
    then the 1024x1024 frame.  The incore buffer holds 256 MB (the thesis'
    size; 87 % of the icosphere's treelets), only the root treelet is
    resident at the start, and the camera orbits 3 degrees per frame while
    moving in from radius 2.5 to 1.2, so treelets keep paging in and out.
    pipelined: the analysis pass of view k+1 runs on a second stream beside
    the cast of frame k (svo_mm_analysis_begin/_end), and its upload goes
    after that cast; the pool states and frames are the sequential loop's.
    Its frame times are the intervals between frame completions (CUDA
    events), as the loop never waits for a frame."""
    import torch

    import libsvo_b200 as L
    from libsvo_b200 import scenes as S

    mm = L.TreeletMemoryManagerCuda(scene, incore_mb << 20)
    mm.setUploadPolicy(policy)
    mm.initDeviceBuffer()
    out = torch.empty((size, size), dtype=torch.int32, device=dev)
    s = torch.cuda.current_stream()
    ms, new_total = [], 0
    poses = [S.orbit_pose(2.5 - 1.3 * f / max(1, frames - 1), 3.0 * f, 20.0, size, size, 25.0).frame_params()
             for f in range(frames)]
    if pipelined:
        sa = torch.cuda.Stream()
        done = [torch.cuda.Event(enable_timing=True) for _ in range(frames)]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for f, p in enumerate(poses):
            mm.beginAnalysePass(p, divisor=8, stream=sa)  # beside the cast of frame f-1
            new, _ = mm.endAnalysePass(after_stream=s)  # its upload after that cast
            mm.render(p, out, stream=s)
            done[f].record(s)
            new_total += new
        s.synchronize()
        wall = time.perf_counter() - t0
        ms = [wall / frames * 1e3] + [done[f - 1].elapsed_time(done[f]) for f in range(1, frames)]
    for f in range(0 if not pipelined else frames, frames):
        p = poses[f]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        new, _ = mm.performAnalysePass(p, divisor=8, stream=s)
        mm.render(p, out, stream=s)
        s.synchronize()
        ms.append((time.perf_counter() - t0) * 1e3)
        new_total += new
    info = mm.info
    mm.close()
    steady = ms[10:]
    return {"scene": "icosphere_s6_d11 (3175 treelets of 98,848 B)", "incore_mb": incore_mb,
            "frame": f"{size}x{size}", "frames": frames, "analysis_divisor": 8,
            "hz_mean": 1e3 / statistics.mean(steady), "ms_p50": statistics.median(steady),
            "ms_p99": float(np.percentile(steady, 99)), "ms_first_frame": ms[0],
            "treelets_inserted": new_total, "resident_slots_at_end": info.num_slots - info.free_slots}


def host_memory_available() -> int:
    """Bytes this process may still allocate: the host's available memory,
    capped by the container's memory limit when there is one."""
    import psutil

    avail = psutil.virtual_memory().available
    for limit, usage in (("/sys/fs/cgroup/memory.max", "/sys/fs/cgroup/memory.current"),
                         ("/sys/fs/cgroup/memory/memory.limit_in_bytes",
                          "/sys/fs/cgroup/memory/memory.usage_in_bytes")):
        try:
            lim = Path(limit).read_text().strip()
            if lim != "max" and int(lim) < (1 << 60):
                avail = min(avail, int(lim) - int(Path(usage).read_text().strip()))
        except (OSError, ValueError):
            pass
    return avail


def flat_leg(dev, reps=50, workload="icosphere", seconds=10.0, cpu_baseline=True):
    """The CpuRaycasterSingleRay3 traversal (flat breadth-first pool with
    absolute first-child indices, stack = the octree's depth, LOD by tcMax)
    over the same scene and view as the main step: the pool flattened on the
    host and uploaded, the frame timed with CUDA events (L2 flushed between
    frames); the CPU figure is the oracle's restatement of traversSvo (the
    reference's CPU raycaster does not build without its gloost
    dependency)."""
    import torch

    import libsvo_b200 as L
    import oracle

    wl = make_workload(workload)
    depth = int(wl.scene.info.max_depth)
    nodes, attribs = wl.scene.flatten()
    dn = torch.from_numpy(nodes.view(np.int32)).to(dev)
    da = torch.from_numpy(attribs.view(np.int32)).to(dev)
    cfg = L.trace_cfg(L.TRAVERSAL_FLAT, depth)
    params = [c.frame_params() for c in wl.cameras]
    outs = [torch.empty((p.height, p.width), dtype=torch.int32, device=dev) for p in params]
    s = torch.cuda.current_stream()
    fetches = hits = 0
    for p, o in zip(params, outs):
        hb = torch.empty(p.width * p.height * 16, dtype=torch.uint8, device=dev)
        L.render(dn, da, nodes.shape[0], p, o, hb, cfg=cfg, stream=s)
        h = hb.cpu().numpy().view(L.HIT_DTYPE)
        fetches += int(h["fetches"].astype(np.int64).sum())
        hits += int(h["hit"].astype(np.int64).sum())
    rays = wl.rays_per_step
    algo_bytes = 8 * fetches + 8 * hits + 4 * rays
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.int32, device=dev)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(reps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(reps)]
    for _ in range(3):
        for p, o in zip(params, outs):
            L.render(dn, da, nodes.shape[0], p, o, cfg=cfg, stream=s)
    for i in range(reps):
        flush.fill_(i)
        starts[i].record(s)
        for p, o in zip(params, outs):
            L.render(dn, da, nodes.shape[0], p, o, cfg=cfg, stream=s)
        ends[i].record(s)
    torch.cuda.synchronize()
    ms = statistics.mean(a.elapsed_time(b) for a, b in zip(starts, ends))
    peak, _ = load_peaks()
    out = {"workload": wl.name + "_flat", "traversal": f"flat (CpuRaycasterSingleRay3), stack {depth}",
           "pool_nodes": int(nodes.shape[0]), "rays_per_step": rays, "ms_per_step": ms,
           "mrays_s": rays / ms / 1e3,
           "roofline": {"algorithmic_bytes_per_step": algo_bytes, "achieved_gbs": algo_bytes / ms / 1e6,
                        "frac": algo_bytes / ms / 1e6 / peak, "node_reads_per_ray": fetches / rays}}
    del flush
    if cpu_baseline:
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        frames = cast = 0
        while True:
            for p in params:
                oracle.render(nodes, attribs, bytes(p), flat=True, stack_size=depth, threads=threads)
                cast += p.width * p.height
            frames += 1
            el = time.perf_counter() - t0
            if el >= seconds or frames >= 200:
                break
        out["cpu_baseline"] = {"value": cast / el / 1e6, "unit": METRIC, "cores": threads, "kind": "port",
                               "sample": f"{frames} whole frame(s) ({cast} rays) in {el:.1f} s; the oracle's "
                                         "restatement of CpuRaycasterSingleRay3::traversSvo"}
    return out


def large_cpu_baseline(wl, n, seconds=10.0):
    """The reference's shadow frame compiled for the host over the large
    pool: the pool is copied to host memory (16 bytes per node), then whole
    frames are timed on all host threads.  Skipped, with the reason, unless
    the host has twice the pool's size free.  Returns the baseline and the
    host copy of the pool (None when skipped)."""
    import types

    need = 16 * n
    avail = host_memory_available()
    if avail < 2 * need + (16 << 30):
        return {"unavailable": f"the pool copy needs {need / 1e9:.1f} GB of host memory, "
                               f"{avail / 1e9:.1f} GB available"}, None
    t0 = time.perf_counter()
    nodes, attribs = wl.scene.getIncoreBuffer()
    copy_s = time.perf_counter() - t0
    one_view = types.SimpleNamespace(cameras=[wl.camera], stack_size=wl.stack_size)
    out = cpu_reference_frames(one_view, nodes, attribs, seconds=seconds, light=wl.light)
    out["sample"] += f"; the {need / 1e9:.1f} GB pool copied to host memory first ({copy_s:.1f} s, untimed)"
    return out, (nodes, attribs)


def large_shadow_leg(dev, reps=10, cap_gb=60.0, subdivisions=9, depth=14, cpu_baseline=True):
    """The large shadowed workload: the depth-14 icosphere built on the GPU, one
    3840x2160 frame of primary rays plus one shadow ray per hit.  The metric
    counts both kinds of ray."""
    import torch

    import libsvo_b200 as L
    from libsvo_b200 import scenes

    t0 = time.perf_counter()
    wl = scenes.large_shadowed(subdivisions=subdivisions, depth=depth)
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    info = wl.scene.info
    d_nodes, d_attribs, n = wl.scene.buffers()
    pool_gb = 16 * n / 1e9
    octree_nodes, overlaps = wl.scene.counts()
    p = wl.camera.frame_params()
    cfg = L.trace_cfg(L.TRAVERSAL_TREELET, wl.stack_size)
    sc = L.shadow_cfg(wl.light)
    px = p.width * p.height
    rgba = torch.empty((p.height, p.width), dtype=torch.int32, device=dev)
    hb = torch.empty(px * 16, dtype=torch.uint8, device=dev)
    sb = torch.empty(px * 16, dtype=torch.uint8, device=dev)
    stats = torch.zeros(4, dtype=torch.int32, device=dev)
    s = torch.cuda.current_stream()
    L.render_shadow(d_nodes, d_attribs, n, p, rgba, sc, hb, sb, cfg=cfg, d_stats=stats, stream=s)
    torch.cuda.synchronize()
    h = hb.cpu().numpy().view(L.HIT_DTYPE)
    sh = sb.cpu().numpy().view(L.HIT_DTYPE)
    gpu_rgba = rgba.cpu().numpy().view(np.uint32).copy()
    del hb, sb
    primary_hits = int(h["hit"].astype(np.int64).sum())
    shadow_rays = primary_hits  # one per hit (all hits lie in the pool)
    shadowed = int(sh["hit"].astype(np.int64).sum())
    fetches = int(h["fetches"].astype(np.int64).sum()) + int(sh["fetches"].astype(np.int64).sum())
    algo_bytes = 8 * fetches + 8 * primary_hits + 4 * px
    rays = px + shadow_rays
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.int32, device=dev)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(reps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(reps)]
    for i in range(3):
        L.render_shadow(d_nodes, d_attribs, n, p, rgba, sc, cfg=cfg, stream=s)
    for i in range(reps):
        flush.fill_(i)
        starts[i].record(s)
        L.render_shadow(d_nodes, d_attribs, n, p, rgba, sc, cfg=cfg, stream=s)
        ends[i].record(s)
    torch.cuda.synchronize()
    ms = statistics.mean(a.elapsed_time(b) for a, b in zip(starts, ends))
    peak, _ = load_peaks()
    out = {"workload": wl.name, "description": wl.description, "scene_build_s": round(build_s, 2),
           "treelets": int(info.num_treelets), "treelet_bytes": int(info.treelet_bytes),
           "octree_nodes": int(octree_nodes), "leaf_voxels": int(info.leaf_voxels),
           "voxel_triangle_overlaps": int(overlaps), "pool_gb": pool_gb, "residency_cap_gb": cap_gb,
           "resident": "all treelets (the pool fits the cap)" if pool_gb <= cap_gb else "over the cap",
           "primary_rays": px, "shadow_rays": shadow_rays, "shadowed_hits": shadowed,
           "ms_per_frame": ms, "mrays_s": rays / ms / 1e3, "primary_mrays_s": px / ms / 1e3,
           "capped_rays": int(stats[0].item()), "bounds_errors": int(stats[1].item()),
           "roofline": {"algorithmic_bytes_per_frame": algo_bytes, "achieved_gbs": algo_bytes / ms / 1e6,
                        "frac": algo_bytes / ms / 1e6 / peak, "node_reads_per_ray": fetches / rays,
                        "traffic": _profiled_traffic(wl.name)[0],
                        "traffic_source": _profiled_traffic(wl.name)[1]}}
    del flush, rgba
    if cpu_baseline:
        try:
            out["cpu_baseline"], pool = large_cpu_baseline(wl, n)
            if pool is not None:
                out["parity"] = reference_parity(pool[0], pool[1], p, gpu_rgba, h, light=wl.light,
                                                 gpu_shadow_hits=sh, config=wl.name, stack_size=wl.stack_size)
                del pool
        except Exception as e:  # the host copy or the CPU run failed: keep the GPU result
            out["cpu_baseline"] = {"unavailable": f"{type(e).__name__}: {e}"}
    wl.scene.close()
    return out


def _r(x, nd=3):
    """x rounded to `nd` significant digits (None stays None)."""
    if x is None or isinstance(x, (bool, str)):
        return x
    if x == 0:
        return 0
    return float(f"{x:.{nd}g}")


def summarize_legs(legs: dict) -> dict:
    """The extra measurements as short summary numbers (Mrays/s, ms, Hz;
    full records with --legs-json)."""
    out = {}
    for key, v in legs.items():
        if "error" in v:
            out[key] = {"error": v["error"][:120]}
            continue
        if key == "flat":
            out[key] = {"mrays_s": _r(v["mrays_s"]), "frac": _r(v["roofline"]["frac"]),
                        "cpu_mrays_s": _r(v.get("cpu_baseline", {}).get("value"))}
        elif key == "batched":
            out[key] = {"per_view_mrays_s": _r(v["per_view_launches_mrays_s"]),
                        "batched_mrays_s": _r(v["batched_mrays_s"]), "speedup": _r(v["speedup"]),
                        "tile": v["autotuned"]["tile"], "threads": v["autotuned"]["block_threads"],
                        "rays_per_lane": v["autotuned"].get("rays_per_lane", 1)}
        elif key == "served":
            rates = {}
            for k in v["speedup_vs_plain_ungated"]:
                b, u = v["batched"][k], v["plain_ungated"][k]
                rates[k] = {"batched": [_r(b["mrays_s"]), _r(b["p50_ms"]), _r(b["p99_ms"])],
                            "plain_ungated": [_r(u["mrays_s"]), _r(u["p50_ms"]), _r(u["p99_ms"])],
                            "x": _r(v["speedup_vs_plain_ungated"][k])}
            pg = {}
            for k, r in v["paging_half_budget"].items():
                q = r["16000"]
                pg[k] = [_r(q["mrays_s"]), _r(q["p50_ms"]), _r(q["p99_ms"])]
            out[key] = {"cols": "Mrays/s, p50 ms, p99 ms", "rates": rates, "half_budget_16000": pg}
            if "treelet_paged" in v:
                t = v["treelet_paged"]
                out[key]["treelet_paged"] = {
                    "cols": "Mrays/s, p50 ms, p99 ms, requests, unconverged, analysis passes",
                    **{k: [_r(t[k]["mrays_s"]), _r(t[k]["p50_ms"]), _r(t[k]["p99_ms"]), t[k]["requests"],
                           t[k]["paged_unconverged"], t[k]["analysis_passes"]]
                       for k in ("fits_rate_100", "fits_rate_16000", "two_regions_rate_16000")}}
        elif key == "large_shadowed":
            out[key] = {"mrays_s": _r(v["mrays_s"]), "ms": _r(v["ms_per_frame"]),
                        "frac": _r(v["roofline"]["frac"]),
                        "cpu_mrays_s": _r(v.get("cpu_baseline", {}).get("value")),
                        "parity_mismatched": v.get("parity", {}).get("mismatched")}
        elif key == "large_streaming":
            cp = v["converged_parity"]
            out[key] = {"cap_gb": v["residency_cap_gb"], "hz": _r(v["hz_mean"]), "p50_ms": _r(v["ms_p50"]),
                        "p99_ms": _r(v["ms_p99"]), "gb_paged": _r(v["gb_paged_in"]),
                        "parity_mismatched": cp["mismatched"], "converged": cp["converged"],
                        "hz_pipelined": _r(v.get("pipelined", {}).get("hz_mean"))}
        elif key == "incore_update":
            out[key] = {k: _r(r["ms_mean"]) for k, r in v.items() if isinstance(r, dict) and "ms_mean" in r}
        elif key == "streaming":
            out[key] = {k: {"hz": _r(r["hz_mean"]), "p99_ms": _r(r["ms_p99"])}
                        for k, r in v.items() if isinstance(r, dict)}
        else:
            out[key] = {k: _r(x) for k, x in v.items() if isinstance(x, (int, float))}
    return out


def large_streaming_leg(dev, cap_gb=24.0, frames=60, subdivisions=9, depth=14, upload="pinned"):
    """The large shadowed workload under a residency cap: the depth-14
    icosphere built on the GPU, its pool turned back into treelets on the host
    (svo_mm_create_from_device_scene), and 3840x2160 primary + shadow frames
    cast through a manager whose incore buffer (nodes and attributes) holds
    cap_gb -- well below the 40 GB pool.  Each frame runs the analysis pass at
    1/8 resolution with a jittered far plane (the reference's dynamic loading:
    treelets paged in by visibility, evicted when the buffer is full) and
    then the frame; the camera moves in along the orbit from radius 2.5 to
    1.2; a pass places at most 12 MB of treelets, as in the reference.  Then
    the last view is converged by analysis passes (256 MB each) at full
    resolution and its primary-ray frame compared with the same frame over the
    fully resident pool (RGBA8 and, per ray, hit, depth, t and loop count;
    node indices differ between the two pools)."""
    import torch

    import libsvo_b200 as L
    from libsvo_b200 import scenes as S

    t0 = time.perf_counter()
    wl = S.large_shadowed(subdivisions=subdivisions, depth=depth)
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    info = wl.scene.info
    slot_bytes = 2 * info.treelet_bytes
    incore = int(cap_gb * 1e9) // slot_bytes * info.treelet_bytes  # node pool; attributes as much again
    t0 = time.perf_counter()
    s = torch.cuda.current_stream()
    mm = L.TreeletMemoryManagerCuda(wl.scene, incore, stream=s)
    host_s = time.perf_counter() - t0
    if upload == "pinned":
        mm.setUploadPolicy(L.UPLOAD_PINNED)
    # every treelet below the root hangs off the root, whose slot never ages:
    # under the reference's eviction rule none could leave a full buffer
    mm.setEviction(L.EVICT_ANY_UNSEEN)
    mm.initDeviceBuffer()
    cfg = L.trace_cfg(L.TRAVERSAL_TREELET, wl.stack_size)
    sc = L.shadow_cfg(wl.light)
    cam = wl.camera
    out = torch.empty((cam.height, cam.width), dtype=torch.int32, device=dev)
    rng = np.random.default_rng(7)
    ms, placed = [], 0
    for f in range(frames):
        r = 2.5 - 1.3 * f / max(1, frames - 1)
        p = S.orbit_pose(r, 40.0 + 3.0 * f, 15.0, cam.width, cam.height, 25.0).frame_params()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        new, _ = mm.performAnalysePass(p, divisor=8, jitter=tuple(rng.uniform(-1, 1, 2)),
                                       stack_size=wl.stack_size, stream=s)
        mm.render_shadow(p, out, sc, cfg=cfg, stream=s)
        s.synchronize()
        ms.append((time.perf_counter() - t1) * 1e3)
        placed += new
    st = mm.sync(s)
    steady = ms[5:]
    primary = cam.width * cam.height
    res = {"workload": wl.name + "_streamed", "scene_build_s": round(build_s, 2),
           "host_treelets_s": round(host_s, 2), "pool_gb": 16 * info.num_treelets * info.nodes_per_treelet / 1e9,
           "residency_cap_gb": cap_gb, "slots": mm.info.num_slots, "treelets": int(info.num_treelets),
           "upload": upload, "frames": frames, "hz_mean": 1e3 / statistics.mean(steady),
           "ms_p50": statistics.median(steady), "ms_p99": float(np.percentile(steady, 99)),
           "ms_first": ms[0], "treelets_paged_in": placed,
           "gb_paged_in": placed * slot_bytes / 1e9, "primary_mrays_s_mean": primary / statistics.mean(steady) / 1e3,
           "capped_rays": st.capped_rays, "bounds_errors": st.bounds_errors}
    # converged view: full-resolution analysis passes until nothing new is
    # asked for, each placing up to 256 MB (the frames above keep the
    # reference's 12 MB per pass)
    mm.setAnalysisBudget(256 << 20)
    steps, asked = 0, 1
    while asked and steps < 200:
        mm.performAnalysePass(p, divisor=1, stack_size=wl.stack_size, stream=s)
        asked = mm.lastAnalysisRequested()
        steps += 1
    hb = torch.empty(primary * 16, dtype=torch.uint8, device=dev)
    mm.render(p, out, hb, cfg=cfg, stream=s)
    s.synchronize()
    got_rgba = out.cpu().numpy().view(np.uint32).copy()
    got = hb.cpu().numpy().view(L.HIT_DTYPE).copy()
    mm.close()
    d_nodes, d_attribs, n = wl.scene.buffers()
    L.render(d_nodes, d_attribs, n, p, out, hb, cfg=cfg, stream=s)
    s.synchronize()
    want = hb.cpu().numpy().view(L.HIT_DTYPE)
    bad = np.zeros(primary, dtype=bool)
    for k in ("hit", "depth", "loops"):
        bad |= got[k] != want[k]
    bad |= got["t"].view(np.uint32) != want["t"].view(np.uint32)
    res["converged_parity"] = {"view": "the last frame's camera (radius 1.2), primary rays", "analysis_passes": steps,
                               "converged": asked == 0, "pixels": primary,
                               "mismatched_rgba": int((got_rgba.reshape(-1) != out.cpu().numpy().view(np.uint32).reshape(-1)).sum()),
                               "mismatched_rays": int(bad.sum())}
    res["converged_parity"]["mismatched"] = (res["converged_parity"]["mismatched_rgba"]
                                             + res["converged_parity"]["mismatched_rays"])
    # the same frames with the next view's analysis run beside the current
    # frame (svo_mm_analysis_begin/_end: same pool states, same frames), on a
    # fresh manager; frame times from CUDA events at the frames' ends
    mm = L.TreeletMemoryManagerCuda(wl.scene, incore, stream=s)
    if upload == "pinned":
        mm.setUploadPolicy(L.UPLOAD_PINNED)
    mm.setEviction(L.EVICT_ANY_UNSEEN)
    mm.initDeviceBuffer()
    rng = np.random.default_rng(7)
    sa = torch.cuda.Stream()
    done = [torch.cuda.Event(enable_timing=True) for _ in range(frames)]
    torch.cuda.synchronize()
    for f in range(frames):
        r = 2.5 - 1.3 * f / max(1, frames - 1)
        p = S.orbit_pose(r, 40.0 + 3.0 * f, 15.0, cam.width, cam.height, 25.0).frame_params()
        mm.beginAnalysePass(p, divisor=8, jitter=tuple(rng.uniform(-1, 1, 2)), stack_size=wl.stack_size,
                            stream=sa)
        mm.endAnalysePass(after_stream=s)
        mm.render_shadow(p, out, sc, cfg=cfg, stream=s)
        done[f].record(s)
    s.synchronize()
    iv = [done[f - 1].elapsed_time(done[f]) for f in range(6, frames)]
    mm.close()
    res["pipelined"] = {"hz_mean": 1e3 / statistics.mean(iv), "ms_p50": statistics.median(iv),
                        "ms_p99": float(np.percentile(iv, 99))}
    del hb, out
    wl.scene.close()
    return res


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        run_reference(args, make_workload(args.workload))
        return

    import torch
    import torch.distributed as dist

    import libsvo_b200 as L

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if args.large_only:
        args.leg = "large_shadowed"
    if args.leg:
        legs = {"batched": lambda: batched_leg(dev, reps=args.steps),
                "served": lambda: served_leg(dev),
                "large_shadowed": lambda: large_shadow_leg(dev, reps=args.steps,
                                                           subdivisions=args.large_subdivisions,
                                                           depth=args.large_depth,
                                                           cpu_baseline=not args.no_cpu_baseline),
                "incore_update": lambda: incore_update_leg(dev, make_workload("icosphere").scene),
                "streaming": lambda: streaming_leg(dev, make_workload("icosphere").scene),
                "flat": lambda: flat_leg(dev, cpu_baseline=not args.no_cpu_baseline),
                "large_streaming": lambda: large_streaming_leg(dev, subdivisions=args.large_subdivisions,
                                                               depth=args.large_depth)}
        print(json.dumps({"leg": args.leg, **legs[args.leg]()}), flush=True)
        return
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    t_build = time.perf_counter()
    wl = make_workload(args.workload)
    info = wl.scene.info
    build_s = time.perf_counter() - t_build
    incore = info.treelet_bytes * info.num_treelets
    stream = torch.cuda.Stream(device=dev)
    mm = L.TreeletMemoryManagerCuda(wl.scene, incore, stream=stream)
    mm.insertAll()
    mm.initDeviceBuffer()
    cfg = L.trace_cfg(L.TRAVERSAL_TREELET, wl.stack_size)
    params = [c.frame_params() for c in wl.cameras]
    outs = [torch.empty((p.height, p.width), dtype=torch.int32, device=dev) for p in params]
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.int32, device=dev)
    rays = wl.rays_per_step

    # algorithmic bytes of one step, from the kernel's own per-ray counters
    fetches = hits = 0
    shadow = L.shadow_cfg(L.seeded_light(1)) if args.shadow else None
    parity_frame = None  # the first view's GPU image and records, for the parity check
    with torch.cuda.stream(stream):
        for p, o in zip(params, outs):
            hb = torch.empty(p.width * p.height * 16, dtype=torch.uint8, device=dev)
            sb = torch.empty(p.width * p.height * 16, dtype=torch.uint8, device=dev) if shadow else None
            if shadow:
                mm.render_shadow(p, o, shadow, hb, sb, cfg=cfg, stream=stream)
            else:
                mm.render(p, o, hb, cfg=cfg, stream=stream)
            stream.synchronize()
            h = hb.cpu().numpy().view(L.HIT_DTYPE)
            fetches += int(h["fetches"].astype(np.int64).sum())
            hits += int(h["hit"].astype(np.int64).sum())
            sh = sb.cpu().numpy().view(L.HIT_DTYPE) if shadow else None
            if shadow:
                fetches += int(sh["fetches"].astype(np.int64).sum())
            if parity_frame is None:
                parity_frame = (p, o.cpu().numpy().view(np.uint32).copy(), h, sh)
            del hb, sb
    algo_bytes = 8 * fetches + 8 * hits + 4 * rays
    primary_rays = rays
    if shadow:
        rays += hits  # one shadow ray per primary hit

    def step():
        for p, o in zip(params, outs):
            if shadow:
                mm.render_shadow(p, o, shadow, cfg=cfg, stream=stream)
            else:
                mm.render(p, o, None, cfg=cfg, stream=stream)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            flush.fill_(1)
            step()
    stream.synchronize()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(local_rank)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    with torch.cuda.stream(stream):
        for i in range(args.steps):
            flush.fill_(i)
            starts[i].record(stream)
            step()
            ends[i].record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    kernel_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    ms = max_over_ranks(statistics.mean(kernel_ms), world, dev)
    value = job_mrays_per_s(world, rays, ms)

    # end to end through the C ABI: host output buffers, image copied back each step
    host_out = [torch.empty((p.height, p.width), dtype=torch.int32).pin_memory() for p in params]

    # two pinned host images per view, alternating between steps
    host_out2 = [torch.empty_like(h).pin_memory() for h in host_out]

    def e2e_step(i):
        with torch.cuda.stream(stream):
            flush.fill_(i)  # the same L2 flush as the device-timed steps, inside the timed region
        for p, ha, hb in zip(params, host_out, host_out2):
            ho = ha if i % 2 == 0 else hb
            # cast, copy back on a second stream overlapping the next cast
            if shadow:
                mm.render_shadow_host_async(p, ho, shadow, cfg=cfg, stream=stream)
            else:
                mm.render_host_async(p, ho, cfg=cfg, stream=stream)

    for i in range(max(1, args.warmup)):
        e2e_step(i)
    mm.sync(stream)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(args.steps):
        e2e_step(i)
    st = mm.sync(stream)  # every image is in host memory; counters of the e2e frames
    e2e_wall = time.perf_counter() - t0
    # clocks sampled from the start of the device-timed steps to the end of
    # the e2e steps (the e2e warm-up between them keeps the GPU busy too)
    clk = clocks.stop()
    clk["window"] = "device-timed and e2e steps"
    e2e_ms = max_over_ranks(e2e_wall * 1e3 / args.steps, world, dev)
    e2e_value = job_mrays_per_s(world, rays, e2e_ms)

    if rank == 0:
        peak, peak_kind = load_peaks()
        achieved = algo_bytes / (ms * 1e-3) / 1e9
        traffic, traffic_source = _profiled_traffic(wl.name + ("_shadow" if shadow else ""))
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene generators; see libsvo_b200/scenes.py)",
            "config": {"workload": wl.name + ("_shadow" if shadow else ""),
                       "description": wl.description + (" + one shadow ray per hit (seeded light)"
                                                        if shadow else ""),
                       "rays_per_step": rays, "primary_rays_per_step": primary_rays,
                       "octree_nodes": int(info.total_nodes), "treelets": int(info.num_treelets),
                       "treelet_bytes": int(info.treelet_bytes), "stack_size": wl.stack_size,
                       "l2": "flushed between steps (256 MB write)",
                       "parallelism": f"replicas x{world}", "scene_build_s": round(build_s, 2)},
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 4 * primary_rays,
                    "note": ("svo_mm_render_shadow_host_async" if shadow else "svo_mm_render_host_async")
                            + ": cast + RGBA8 image copied to pinned host memory on a second stream "
                            "(overlapping the next cast), all waited for"
                            + "; host wall clock over the steps, the 256 MB L2 flush of every step included; "
                            "frame parameters travel as kernel arguments"},
            "gpu_launches": args.steps * sum(_kernels_per_render(p, shadow) for p in params),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "traffic_source": traffic_source,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                         if peak_kind == "measured" else "fallback 6650 GB/s",
                         "algorithmic_bytes_per_step": algo_bytes,
                         "bytes_per_ray": algo_bytes / rays, "node_reads_per_ray": fetches / rays,
                         "hit_fraction": hits / rays},
            "watchdog": {"capped_rays": st.capped_rays, "bounds_errors": st.bounds_errors,
                         "frames": args.steps * len(params)},
        }
        if not args.no_cpu_baseline and world == 1:
            nodes, attribs = mm.getIncoreBuffer()
            line["cpu_baseline"] = cpu_reference_frames(wl, nodes, attribs,
                                                        light=L.seeded_light(1) if shadow else None)
            pp, p_rgba, p_hits, p_shadow = parity_frame
            line["parity"] = reference_parity(nodes, attribs, pp, p_rgba, p_hits,
                                              light=L.seeded_light(1) if shadow else None,
                                              gpu_shadow_hits=p_shadow, config=line["config"]["workload"],
                                              stack_size=wl.stack_size)
        mm.close()
        legs = {}
        if world == 1 and not args.no_extra and args.workload == "icosphere":
            for key, leg in (("incore_update", incore_update_leg), ("streaming", streaming_leg)):
                t_leg = time.perf_counter()
                try:
                    legs[key] = leg(dev, wl.scene)
                except Exception as e:  # a failing extra leg must not lose the primary line
                    legs[key] = {"error": f"{type(e).__name__}: {e}"}
                print(f"[bench] leg {key}: {time.perf_counter() - t_leg:.1f} s", file=sys.stderr, flush=True)
        if world == 1 and not args.no_extra:
            extra = (("flat", lambda d: flat_leg(d, cpu_baseline=not args.no_cpu_baseline)),
                     ("batched", batched_leg), ("served", served_leg),
                     ("large_shadowed", lambda d: large_shadow_leg(d, cpu_baseline=not args.no_cpu_baseline)),
                     ("large_streaming", large_streaming_leg))
            for key, leg in extra:
                t_leg = time.perf_counter()
                try:
                    legs[key] = leg(dev)
                except Exception as e:  # a failing extra leg must not lose the primary line
                    legs[key] = {"error": f"{type(e).__name__}: {e}"}
                print(f"[bench] leg {key}: {time.perf_counter() - t_leg:.1f} s", file=sys.stderr, flush=True)
        if legs:
            if args.legs_json:
                Path(args.legs_json).write_text(json.dumps(legs, indent=1))
            # the compact summary goes last, so that a reader keeping only the
            # end of the line still sees every leg
            line["legs"] = summarize_legs(legs)
        print(json.dumps(line), flush=True)
    mm.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
