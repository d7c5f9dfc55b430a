#!/usr/bin/env python
"""Benchmark of the TEASAR skeletonizer on one B200 node (one process per GPU).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config NAME]

A step is one skeletonization of the workload volume. At N = 1 the workload is the dense
segmentation: a 512^3 uint64 volume of Voronoi cells (600 seeds, seed 1) cut by random-walk tubes
of radius 3-10, boundaries eroded, anisotropy (8, 8, 40), TEASAR scale 1.5, const 300, PDRF 1e5/4,
dust 100 (synthetic: the reference's connectomics volumes are not available). With N > 1 every
rank skeletonizes its own volume of the same kind (seed 1 + rank): replicas, weak scaling.

`value` is voxels/s with the labels already in HBM (device tensor in, packed host skeletons out);
`e2e` is the same metric through the public API from pinned host memory (host -> device copy of
the labels and device -> host copy of the skeletons inside the timed region). Times are CUDA
events on the device, max over ranks. `--impl reference` times the CPU restatement of the
reference's algorithm (the reference has no CPU implementation of this path) on all host cores.
"""
from __future__ import annotations

import argparse
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

CONFIGS = {
    "dense512": dict(workload="dense segmentation 512x512x512 uint64, 600 Voronoi seeds cut by tubes r=3-10 (seed 1)",
                     shape=(512, 512, 512), seeds=600, seed=1, kind="dense", dtype="uint64", anisotropy=(8, 8, 40)),
    "dense256": dict(workload="dense segmentation 256x256x256 uint64, 80 Voronoi seeds cut by tubes r=3-10 (seed 5); "
                          "the profiling case", shape=(256, 256, 256), seeds=80, seed=5, kind="dense", dtype="uint64",
                     anisotropy=(8, 8, 40)),
    "batch64": dict(workload="64 uneven uint32 volumes (edges log-uniform 64-256), 10-80 tubes r=1-8, ~5% arbors (seed 2)",
                    seed=2, kind="batch", dtype="uint32", anisotropy=(4, 4, 4)),
    "serve": dict(workload="Poisson request stream at 50/200/800 req/s (seed 4), volume edges log-uniform 32-384, "
                       "1 tube per 64^3 voxels, uint32/uint64 50/50, 80 GB admission cap",
                  seed=4, kind="serve", rates=(50, 200, 800), requests=300, anisotropy=(16, 16, 40)),
    "chunks1024": dict(workload="dense segmentation 1024x1024x256 uint32, 3000 Voronoi seeds cut by tubes r=3-10 "
                            "(seed 3): whole in-core, and as 512x512x256 chunks with 64-voxel overlap in one batch",
                       shape=(1024, 1024, 256), seeds=3000, seed=3, kind="chunks", dtype="uint32",
                       anisotropy=(16, 16, 40), chunk=(512, 512, 256), overlap=64),
    "stream1024": dict(workload="dense segmentation 1024x1024x1024 uint32, 4800 Voronoi seeds cut by tubes r=3-10 "
                            "(seed 4), out of core: its in-core state (about 176 GB) does not fit beside the labels",
                       shape=(1024, 1024, 1024), seeds=4800, seed=4, kind="streamed", dtype="uint32",
                       anisotropy=(8, 8, 40)),
    "tubes128": dict(workload="128x128x128 uint32, 20 random-walk tubes r=2-6 (seed 0)", shape=(128, 128, 128),
                     objects=20, seed=0, kind="tubes", dtype="uint32", anisotropy=(16, 16, 40)),
}
PARAMS = dict(scale=1.5, const=300, pdrf_scale=100000, pdrf_exponent=4)
DUST = 100
METRIC = "voxels/s & skeletons/s, batched/graph vs per-volume on 1 B200; p50/p99 latency"


def make_volume(cfg, rank=0):
    from brook_b200 import synthetic

    if cfg["kind"] == "batch":
        return synthetic.uneven_batch(seed=cfg["seed"] + rank)

    if cfg["kind"] in ("dense", "chunks", "streamed"):
        return synthetic.dense_volume(cfg["shape"], seeds=cfg["seeds"], seed=cfg["seed"] + rank, dtype=np.dtype(cfg["dtype"]))
    return synthetic.tube_volume(cfg["shape"], objects=cfg["objects"], seed=cfg["seed"] + rank, dtype=np.dtype(cfg["dtype"]))


def stage_roofline(stage, peak):
    """Per stage: CUDA-event ms, algorithmic bytes (the per-unit figures of the path's measurement
    plan: N voxels, F object voxels, b input label bytes, c component-id bytes), GB/s and the
    fraction of the measured HBM peak."""
    N, F = stage.get("voxels", 0), stage.get("foreground", 0)
    c = stage.get("label_bytes", 2)
    nb = stage.get("input_bytes", 0)
    alg = {
        "ccl": nb + N * c,                               # read labels, write ids
        "edt": N * (3 * c + 20),                         # x: N(c+4), y and z: N(c+8) each
        "mask": N * (4 + 4),                             # ids in, mask out
        "dbf_max": N * (4 + c),                          # argmax
        "prepare": 2 * F * (c + 8) + N * (12 + c),       # two DAF floods and the PDRF
        "order": F * (4 + c) + 4 * F,                    # target-order keys in, order out
        "trace": stage.get("railroad_settled", 0) * (12 + c) + stage.get("invalidated", 0) * (13 + c),
        "assembly": stage.get("path_vertices", 0) * 8 + stage.get("vertices", 0) * 16 + stage.get("edges", 0) * 8,
    }
    out = {}
    for name, b in alg.items():
        ms = stage.get("ms_" + name)
        if not ms:
            continue
        gbs = b / (ms / 1e3) / 1e9
        out[name] = {"ms": round(ms, 3), "algorithmic_bytes": int(b), "gbs": round(gbs, 2), "frac": round(gbs / peak, 5)}
    return out


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while the timed region runs."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        # the raw samples: a temporary file unless BENCH_CLOCKS_DIR names a folder to keep them in
        folder = os.environ.get("BENCH_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(folder, f"clocks_{index}.csv")

    def __enter__(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        query = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap")
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={query}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.out.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            rows = []
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[j] for r in rows for j in range(4) if len(r) > 5 + j and "Active" in r[5 + j]
                          and "Not" not in r[5 + j]})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def result_bytes(packed):
    return int(packed.vertices.nbytes + packed.edges.nbytes + packed.radii.nbytes + packed.labels.nbytes +
               packed.v_off.nbytes + packed.e_off.nbytes)


def oracle_whole(volume, cfg, threads, steps):
    """The oracle (the CPU restatement of the reference's algorithm) over the whole workload volume,
    its work spread over `steps` timed steps: step 0 runs the preamble (components, boxes, EDT,
    border targets, roots, DAF, PDRF, target orders) and each step traces its share of the objects
    in the largest-first order; the last step assembles. Returns (seconds of all steps, skeletons,
    the oracle's per-stage ms)."""
    from oracle import oracle

    t0 = time.perf_counter()
    run = oracle.StagedRun(volume, PARAMS, cfg["anisotropy"], DUST, threads=threads)
    per = -(-run.objects // steps) if run.objects else 0
    for k in range(steps):
        run.trace(k * per, (k + 1) * per)
    result = run.finish()
    return time.perf_counter() - t0, len(result.array("labels")), result.stage_ms()


def cpu_baseline(volume, cfg, threads):
    """The oracle on the whole workload volume, on every host core."""
    dt, skeletons, stages = oracle_whole(volume, cfg, threads, 1)
    return {"value": volume.size / dt, "unit": "voxels/s", "cores": threads, "kind": "port",
            "sample": f"the whole {'x'.join(map(str, volume.shape))} workload volume ({volume.size} voxels, "
                      f"{skeletons} skeletons), {dt:.2f} s on {threads} threads",
            "stages_ms": {k: round(v, 1) for k, v in stages.items()}}


def run_reference(args, cfg):
    """The reference arm: the CPU restatement of the reference's algorithm (the reference has no
    CPU implementation of this path; its GPU code is not built here) on the same whole volume as
    our arm, on all host cores. The W warm-up steps run it on a 64^3 crop; the K timed steps
    together process the whole volume once (oracle_whole), so value = voxels / time of the K
    steps. Only rank 0 works; this process never loads libbrook_b200.so."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle

    volume = make_volume(cfg)
    threads = os.cpu_count() or 1
    crop = np.asfortranarray(volume[:64, :64, :64])
    for _ in range(args.warmup):
        oracle.skeletonize(crop, PARAMS, cfg["anisotropy"], DUST, threads=threads)
    dt, skeletons, stages = oracle_whole(volume, cfg, threads, args.steps)
    value = volume.size / dt
    sample = (f"the whole {'x'.join(map(str, volume.shape))} volume ({volume.size} voxels) once over the "
              f"{args.steps} timed steps: the preamble in the first, the objects' traces split over all, assembly in "
              f"the last; warm-up steps on a 64^3 crop")
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "voxels/s", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "int32/f32", "data": "synthetic",
           "skeletons_per_s": skeletons / dt,
           "config": config_of(cfg, volume),
           "cpu_baseline": {"value": value, "unit": "voxels/s", "cores": threads, "kind": "port", "sample": sample,
                            "stages_ms": {k: round(v, 1) for k, v in stages.items()}},
           "e2e": {"value": value, "unit": "voxels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def config_of(cfg, volume, world=1):
    """The workload description both arms print (same keys and values for the same workload)."""
    return {"workload": cfg["workload"], "voxels_per_gpu": int(volume.size), "anisotropy": list(cfg["anisotropy"]),
            "teasar": PARAMS, "dust_threshold": DUST, "parallelism": f"replicas x{world}",
            "l2": f"labels of {volume.nbytes / 2**20:.0f} MiB per step, "
                  + ("larger than L2 (126 MB)" if volume.nbytes > 126e6 else "smaller than L2: not flushed")}


def run_batch(args, cfg):
    """The uneven batch: one skeletonize_batch call per step (all 64 volumes in one launch of each
    engine kernel) against the same volumes through 64 plain skeletonize calls. With N > 1 ranks
    the same batch is split over the ranks (longest-first by voxels, brook_b200.sharding), each
    rank runs its share as one batch and rank 0 gathers the results: strong scaling."""
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", device_id=torch.device("cuda", local))
    line = batch_measurement(cfg, args.steps, args.warmup, rank, world, local, dist)
    if line is not None:
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


def batch_measurement(cfg, steps, warmup, rank=0, world=1, local=0, dist=None):
    """run_batch's measurement; returns rank 0's line (None on the other ranks)."""
    import torch

    import brook_b200
    from brook_b200 import _native, sharding

    volumes = make_volume(cfg)  # the same batch on every rank
    mine = sharding.partition([v.size for v in volumes], world)[rank]
    devs = {i: torch.from_numpy(np.ascontiguousarray(volumes[i].transpose(2, 1, 0))).cuda(local).permute(2, 1, 0)
            for i in mine}
    opts = dict(teasar_params=PARAMS, anisotropy=cfg["anisotropy"], dust_threshold=DUST, device=local)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(fn, steps):
        barrier()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        out, stage = None, {}
        for _ in range(steps):
            out = fn()
            for k, v in _native.stats(local).items():
                stage[k] = stage.get(k, 0.0) + v
        end.record()
        torch.cuda.synchronize()
        ms = start.elapsed_time(end) / steps
        if dist is not None:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        barrier()
        return ms, out, {k: v / steps for k, v in stage.items()}

    samples = [devs.get(i, v) for i, v in enumerate(volumes)]  # only this rank's share is read
    if world > 1:
        batched = lambda: sharding.skeletonize_batch_sharded(samples, rank, world, **opts)  # noqa: E731
    else:
        batched = lambda: brook_b200.skeletonize_batch([devs[i] for i in mine], output="packed", **opts)  # noqa: E731
    plain = lambda: [brook_b200.skeletonize(devs[i], output="packed", **opts) for i in mine]  # noqa: E731
    for _ in range(warmup):
        batched()
    if world == 1:  # the engine's launch choices measured on the batch (untimed)
        from brook_b200 import tuning

        tuning.autotune([devs[i] for i in mine], PARAMS, cfg["anisotropy"], DUST, device=local, save=False)
    with ClockSampler(local) as clocks:
        ms, out, stage = timed(batched, steps)
    plain()
    plain_ms, plain_out, _ = timed(plain, max(1, steps // 2))
    # identical skeletons both ways (rank 0 holds the whole batch; with one rank `mine` is all)
    if out is not None:
        for j, p in enumerate(plain_out):
            q = out[mine[j]]
            assert list(p.labels) == list(q.labels)
            np.testing.assert_array_equal(p.vertices, q.vertices)
            np.testing.assert_array_equal(p.edges, q.edges)
    # end to end from pinned host memory (this rank's share)
    pinned = {}
    for i in mine:
        t = torch.empty(volumes[i].shape[::-1], dtype=torch.int32, pin_memory=True)
        t.numpy().view(np.uint32)[...] = volumes[i].transpose(2, 1, 0)
        pinned[i] = t.numpy().view(np.uint32).transpose(2, 1, 0)
    host_samples = [pinned.get(i, v) for i, v in enumerate(volumes)]
    if world > 1:
        e2e_fn = lambda: sharding.skeletonize_batch_sharded(host_samples, rank, world, **opts)  # noqa: E731
    else:
        e2e_fn = lambda: brook_b200.skeletonize_batch([pinned[i] for i in mine], output="packed", **opts)  # noqa: E731
    e2e_ms, out_h, _ = timed(e2e_fn, steps)
    if rank != 0:
        return None
    skeletons = len(out.labels)
    voxels = sum(int(v.size) for v in volumes)
    plain_skeletons = sum(len(p) for p in plain_out)
    stage_ms = {k[3:]: v for k, v in stage.items() if k.startswith("ms_") and k != "ms_total"}
    out_line = {
        "metric": METRIC, "value": skeletons / (ms / 1e3), "unit": "skeletons/s", "n_gpus": world, "steps": steps,
        "warmup": warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "int32/f32", "data": "synthetic", "voxels_per_s": voxels / (ms / 1e3),
        "per_volume": {"skeletons_per_s": plain_skeletons / (plain_ms / 1e3), "ms_per_step": plain_ms,
                       "volumes": len(mine), "speedup_batched": (skeletons / ms) / (plain_skeletons / plain_ms),
                       "identical": True, "note": "rank 0's share through per-volume calls on its GPU"},
        "config": {"workload": cfg["workload"], "volumes": len(volumes), "voxels": voxels,
                   "anisotropy": cfg["anisotropy"], "teasar": PARAMS, "dust_threshold": DUST,
                   "parallelism": f"volume shards x{world} (longest first), results gathered to rank 0",
                   "l2": "inputs larger than L2 (0.75 GB of labels per step)"},
        "stages_ms": {k: round(v, 3) for k, v in sorted(stage_ms.items())},
        "stages_roofline": stage_roofline(stage, peaks()[0]),
        "host_ms": {k[8:]: round(v, 3) for k, v in sorted(stage.items()) if k.startswith("host_ms_")},
        "e2e": {"value": skeletons / (e2e_ms / 1e3), "unit": "skeletons/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": int(sum(volumes[i].nbytes for i in mine)),
                "d2h_bytes_per_step": int(out_h.packed.vertices.nbytes + out_h.packed.edges.nbytes +
                                          out_h.packed.radii.nbytes)},
        "gpu_launches": int(stage.get("launches", 0) * steps),
        "clocks": clocks.summary(),
    }
    return out_line


def run_chunks(args, cfg):
    """The large volume: skeletonized whole (in-core) and as overlapping chunks in one batch, each
    with its per-stage HBM figures. The chunks' skeletons are not merged (merging parts is a
    post-processing step)."""
    import torch

    import brook_b200
    from brook_b200 import _native, sharding

    local = int(os.environ.get("LOCAL_RANK", "0"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(local)
    if rank != 0:
        return
    volume = make_volume(cfg)
    dev = torch.from_numpy(np.ascontiguousarray(volume.transpose(2, 1, 0))).cuda(local).permute(2, 1, 0)
    chunks = [dev[c] for c in sharding.iter_chunks(volume.shape, cfg["chunk"], cfg["overlap"])]
    opts = dict(teasar_params=PARAMS, anisotropy=cfg["anisotropy"], dust_threshold=DUST, device=local)
    peak, source = peaks()

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stage = {}
        start.record()
        for _ in range(args.steps):
            out = fn()
            for k, v in _native.stats(local).items():
                stage[k] = stage.get(k, 0.0) + v
        end.record()
        torch.cuda.synchronize()
        return start.elapsed_time(end) / args.steps, out, {k: v / args.steps for k, v in stage.items()}

    with ClockSampler(local) as clocks:
        ms, whole, stage = timed(lambda: brook_b200.skeletonize(dev, output="packed", **opts))
        cms, parts, cstage = timed(lambda: brook_b200.skeletonize_batch(chunks, output="packed", **opts))
    voxels = int(volume.size)
    chunk_voxels = int(sum(c.numel() for c in chunks))
    print(json.dumps({
        "metric": METRIC, "value": voxels / (ms / 1e3), "unit": "voxels/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32/f32", "data": "synthetic", "skeletons_per_s": len(whole) / (ms / 1e3),
        "config": {"workload": cfg["workload"], "voxels": voxels, "anisotropy": cfg["anisotropy"], "teasar": PARAMS,
                   "dust_threshold": DUST, "chunks": len(chunks), "chunk": cfg["chunk"], "overlap": cfg["overlap"],
                   "l2": "labels of 1 GiB per step, larger than L2 (126 MB)"},
        "stages_roofline": stage_roofline(stage, peak), "peak_gbs": peak, "peak_source": source,
        "chunked": {"ms_per_step": cms, "voxels_per_s": chunk_voxels / (cms / 1e3), "voxels": chunk_voxels,
                    "skeletons": int(len(parts.labels)), "stages_roofline": stage_roofline(cstage, peak)},
        "clocks": clocks.summary(),
    }))


def run_serve(args, cfg):
    """The request loop: each rate's stream replayed in real time through the continuous-batching
    server and through the plain per-request path (one worker, one request per call)."""
    import torch

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if rank != 0:  # requests are served by one GPU; other ranks have nothing to do
        return
    print(json.dumps(serve_measurement(cfg, local)))


def serve_measurement(cfg, local=0):
    """run_serve's measurement: the line as a dict."""
    from brook_b200 import serving, synthetic

    base = synthetic.serving_requests(cfg["requests"], 1.0, seed=cfg["seed"])  # arrivals at rate 1, rescaled below
    opts = dict(teasar_params=PARAMS, anisotropy=cfg["anisotropy"], dust_threshold=DUST, device=local,
                memory_cap=80e9, engine_share=int(os.environ.get("BROOK_B200_SERVE_ENGINE_SHARE", "100")))
    warm = [(0.0, v) for _, v in base[:8]]
    serving.replay(warm, lambda: serving.Server(workers=2, **opts))
    rates, total = {}, None
    with ClockSampler(local) as clocks:
        for rate in cfg["rates"]:
            stream = [(t / rate, v) for t, v in base]
            row = {}
            for name, kw in (("batched", dict(workers=2)), ("per_request", dict(workers=1, max_batch=1))):
                servers = []

                def factory():
                    servers.append(serving.Server(**kw, **opts))
                    return servers[-1]

                t0 = time.perf_counter()
                done = serving.replay(stream, factory)
                wall = time.perf_counter() - t0
                skel = sum(len(r.future.result()) for r in done)
                lat = serving.percentiles([r.latency * 1e3 for r in done])
                server = servers[0]
                slow = max(server.records, key=lambda r: r["end"] - r["start"])
                row[name] = {"p50_ms": lat["p50"], "p99_ms": lat["p99"], "skeletons_per_s": skel / wall,
                             "requests_per_s": len(done) / wall, "wall_s": wall, "batches": len(server.records),
                             "hand_backs": server.trims, "state_bytes_per_voxel": server.state_bytes_per_voxel,
                             "slowest_batch": {"wall_ms": (slow["end"] - slow["start"]) * 1e3,
                                               "starts_at_s": slow["start"] - t0,
                                               **{k: slow[k] for k in ("requests", "voxels", "device_ms",
                                                                      "peak_bytes", "handed_back_first")},
                                               "host_ms": {k: round(v, 1) for k, v in slow["host_ms"].items()
                                                           if v >= 1.0}}}
                total = skel
            rates[str(rate)] = row
    head = rates[str(cfg["rates"][1])]["batched"]
    voxels = int(sum(v.size for _, v in base))
    return {
        "metric": METRIC, "value": head["skeletons_per_s"], "unit": "skeletons/s", "n_gpus": 1,
        "steps": len(cfg["rates"]), "warmup": 1, "ms_per_step": head["wall_s"] * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32/f32", "data": "synthetic",
        "latency_ms": rates, "skeletons_per_stream": total,
        "config": {"workload": cfg["workload"], "requests_per_rate": cfg["requests"], "voxels_per_stream": voxels,
                   "value_rate": cfg["rates"][1], "anisotropy": cfg["anisotropy"], "teasar": PARAMS,
                   "dust_threshold": DUST, "workers": 2, "timing": "wall clock per request, arrival to result"},
        "e2e": {"value": head["skeletons_per_s"], "unit": "skeletons/s",
                "h2d_bytes_per_step": int(sum(v.nbytes for _, v in base)), "d2h_bytes_per_step": None},
        "clocks": clocks.summary(),
    }


OPTIONS_CASE = dict(workload="cells with nuclei 256x256x256 uint32, 64 Voronoi cells (seed 6), half with an empty "
                             "cavity; anisotropy (1, 1, 1)", shape=(256, 256, 256), cells=64, seed=6)
OPTIONS_PARAMS = dict(scale=1.5, const=10, pdrf_scale=100000, pdrf_exponent=4, soma_detection_threshold=30,
                      soma_acceptance_threshold=1e6)


def options_measurement(local, steps=3):
    """fill_holes and fix_avocados on a volume that has work for both (enclosed nuclei, empty
    cavities): per option set the device time of one call (CUDA events, mean of `steps` after a
    warm-up), the option's own stage and host time, the skeletons, and the oracle's time for the
    same call on the host cores."""
    import brook_b200
    from brook_b200 import _native, synthetic
    from oracle import oracle

    volume = synthetic.cell_volume(OPTIONS_CASE["shape"], cells=OPTIONS_CASE["cells"], seed=OPTIONS_CASE["seed"])
    out = {"workload": OPTIONS_CASE["workload"], "teasar": OPTIONS_PARAMS}
    for name, opts in (("plain", {}), ("fill_holes", dict(fill_holes=True)), ("fix_avocados", dict(fix_avocados=True)),
                       ("both", dict(fill_holes=True, fix_avocados=True))):
        call = lambda: brook_b200.skeletonize(volume, OPTIONS_PARAMS, (1, 1, 1), dust_threshold=DUST, output="packed",
                                              device=local, **opts)
        call()
        total, stage, host, skeletons = 0.0, 0.0, 0.0, 0
        for _ in range(steps):
            skeletons = len(call())
            st = _native.stats(local)
            total += st.get("ms_total", 0.0)
            for key in ("holes", "avocados"):
                stage += st.get("ms_" + key, 0.0)
                host += st.get("host_ms_" + key, 0.0)
        row = {"ms_per_call": total / steps, "skeletons": skeletons}
        if opts:
            row.update({"option_stage_ms": stage / steps, "option_host_ms": host / steps})
            if "fill_holes" in opts:
                row["hole_filled_voxels"] = st.get("hole_filled_voxels")
            if "fix_avocados" in opts:
                row["avocado_passes"] = st.get("avocado_passes")
        out[name] = row
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    ref = oracle.skeletonize(volume, OPTIONS_PARAMS, (1, 1, 1), DUST, threads=threads, fill_holes=True,
                             fix_avocados=True)
    out["cpu_oracle_both"] = {"ms_per_call": (time.perf_counter() - t0) * 1e3, "threads": threads,
                              "skeletons": len(ref.array("labels"))}
    return out


def post_measurement(local, packed, steps=3, dust=1500.0, ticks=3500.0):
    """The canonical post-processing (the reference's defaults: dust 1500, ticks 3500) of the
    workload's own skeletons on the device: the call's span on the stream (CUDA events, mean of
    `steps` after a warm-up) and its wall time, each step's time, and the oracle's time for the same
    input on one host core, the two outputs compared bit for bit."""
    from brook_b200 import _native, device_post
    from oracle import post as opost

    dev_in = packed.to_device()
    device_post.postprocess(dev_in, dust, ticks)
    span, wall, stages = 0.0, 0.0, {}
    for _ in range(steps):
        t0 = time.perf_counter()
        out = device_post.postprocess(dev_in, dust, ticks)
        wall += time.perf_counter() - t0
        st = _native.stats(local)
        span += st.get("ms_total", 0.0)
        for k, v in st.items():
            if k.startswith("ms_post_"):
                stages[k[8:]] = stages.get(k[8:], 0.0) + v
    got = out.to_host()
    host = dict(labels=packed.labels, vertex_offsets=packed.v_off, edge_offsets=packed.e_off, vertices=packed.vertices,
                edges=packed.edges, radii=packed.radii)
    t0 = time.perf_counter()
    ref = opost.postprocess(host, dust, ticks)
    cpu_ms = (time.perf_counter() - t0) * 1e3
    identical = all(np.array_equal(np.asarray(a), np.asarray(b)) for a, b in (
        (got.labels, ref["labels"]), (got.v_off, ref["vertex_offsets"]), (got.e_off, ref["edge_offsets"]),
        (got.edges, ref["edges"]), (np.asarray(got.vertices).view(np.uint32), ref["vertices"].view(np.uint32)),
        (np.asarray(got.radii).view(np.uint32), ref["radii"].view(np.uint32))))
    return {"workload": f"canonical post-processing (dust {dust:g}, ticks {ticks:g}) of the workload's "
                        f"{len(packed)} skeletons ({int(packed.v_off[-1])} vertices, {int(packed.e_off[-1])} edges)",
            "ms_per_call": span / steps, "wall_ms_per_call": wall / steps * 1e3,
            "stages_ms": {k: round(v / steps, 3) for k, v in sorted(stages.items())},
            "out_vertices": int(got.v_off[-1]), "out_edges": int(got.e_off[-1]),
            "cpu_oracle_ms": cpu_ms, "cpu_oracle_threads": 1, "identical": bool(identical),
            "timing": "CUDA events on the context's stream across the call (host read-backs included), "
                      "mean of 3 calls after a warm-up"}


def extra_measurements(local, packed=None):
    """The metric's two comparisons beside the headline line, on the same GPU: the 64-volume uneven
    batch as one skeletonize_batch call against 64 plain calls (skeletons/s both ways, identical
    skeletons checked), and the request stream's p50/p99 latency at 50/200/800 req/s through the
    continuous-batching server and the per-request path; the fill_holes / fix_avocados options
    on a volume with enclosed nuclei and cavities; and the canonical post-processing of the
    workload's own skeletons (`packed`)."""
    extras = {}
    try:
        b = batch_measurement(CONFIGS["batch64"], steps=3, warmup=2, local=local)
        extras["batch64"] = {
            "workload": CONFIGS["batch64"]["workload"], "batched_skeletons_per_s": b["value"],
            "batched_ms_per_call": b["ms_per_step"], "per_volume_skeletons_per_s": b["per_volume"]["skeletons_per_s"],
            "per_volume_ms_per_64_calls": b["per_volume"]["ms_per_step"],
            "speedup_batched": b["per_volume"]["speedup_batched"], "identical": b["per_volume"]["identical"],
            "e2e_batched_skeletons_per_s": b["e2e"]["value"], "stages_ms": b["stages_ms"],
            "timing": "CUDA events on the device, 3 batched calls and 1 round of 64 plain calls after 2 warm-ups"}
    except Exception as e:  # the headline line still prints
        extras["batch64"] = {"error": f"{type(e).__name__}: {e}"}
    try:
        v = serve_measurement(CONFIGS["serve"], local)
        extras["serve"] = {"workload": CONFIGS["serve"]["workload"], "latency_ms": v["latency_ms"],
                           "timing": "wall clock per request, arrival to result"}
    except Exception as e:
        extras["serve"] = {"error": f"{type(e).__name__}: {e}"}
    try:
        extras["options"] = options_measurement(local)
    except Exception as e:
        extras["options"] = {"error": f"{type(e).__name__}: {e}"}
    if packed is not None:
        try:
            extras["post"] = post_measurement(local, packed)
        except Exception as e:
            extras["post"] = {"error": f"{type(e).__name__}: {e}"}
    return extras


def run_ours(args, cfg):
    import torch

    import brook_b200
    from brook_b200 import _native

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", device_id=torch.device("cuda", local))
    volume = make_volume(cfg, rank)
    # device input: a Fortran-ordered view (x fastest) read in place
    dev = torch.from_numpy(np.ascontiguousarray(volume.transpose(2, 1, 0))).cuda(local).permute(2, 1, 0)
    # host input for the end-to-end leg: pinned memory, Fortran order
    pinned_t = torch.empty(volume.shape[::-1], dtype=dev.dtype, pin_memory=True)
    pinned_t.numpy()[...] = volume.transpose(2, 1, 0)
    pinned = pinned_t.numpy().transpose(2, 1, 0)
    opts = dict(teasar_params=PARAMS, anisotropy=cfg["anisotropy"], dust_threshold=DUST, output="packed", device=local)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(fn, steps):
        barrier()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        out, stage = None, {}
        for _ in range(steps):
            out = fn()
            for k, v in _native.stats(local).items():
                stage[k] = stage.get(k, 0.0) + v
        end.record()
        torch.cuda.synchronize()
        ms = start.elapsed_time(end) / steps
        if dist is not None:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        barrier()
        return ms, out, {k: v / steps for k, v in stage.items()}

    for _ in range(args.warmup):
        brook_b200.skeletonize(dev, **opts)
    # the engine's launch choices measured on this workload (untimed; installed in this context)
    tuned = None
    if not args.no_autotune:
        from brook_b200 import tuning

        tuned = tuning.autotune(dev, PARAMS, cfg["anisotropy"], DUST, device=local, save=False)
        brook_b200.skeletonize(dev, **opts)
    with ClockSampler(local) as clocks:
        ms, packed, stage = timed(lambda: brook_b200.skeletonize(dev, **opts), args.steps)
    for _ in range(max(1, args.warmup // 2)):
        brook_b200.skeletonize(pinned, **opts)
    e2e_ms, packed_h, _ = timed(lambda: brook_b200.skeletonize(pinned, **opts), args.steps)
    np.testing.assert_array_equal(packed.vertices, packed_h.vertices)
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    voxels = volume.size * world
    skeletons = len(packed) * world
    value = voxels / (ms / 1e3)
    # roofline of the dominant kernel (the object engine's trace launch): algorithmic bytes per
    # launch = settled railroad voxels x (12 + c) + invalidated voxels x (13 + c), c = label bytes
    c = stage.get("label_bytes", 2)
    trace_bytes = stage.get("railroad_settled", 0) * (12 + c) + stage.get("invalidated", 0) * (13 + c)
    stage_ms = {k[3:]: v for k, v in stage.items() if k.startswith("ms_") and k != "ms_total"}
    dominant = max(stage_ms, key=stage_ms.get) if stage_ms else "trace"
    peak, source = peaks()
    achieved = trace_bytes / (stage.get("ms_trace", float("nan")) / 1e3) / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic_dense512.txt")
    if os.path.exists(tfile):
        for line in open(tfile):
            if line.startswith("trace_kernel dram_bytes_per_launch"):
                traffic = float(line.split("=")[1])
    out = {
        "metric": METRIC, "value": value, "unit": "voxels/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32/f32", "data": "synthetic",
        "skeletons_per_s": skeletons / (ms / 1e3),
        "config": config_of(cfg, volume, world),
        "objects": int(stage.get("objects", 0)),
        "stages_ms": {k: round(v, 3) for k, v in sorted(stage_ms.items())},
        "stages_roofline": stage_roofline(stage, peaks()[0]),
        "host_ms": {k[8:]: round(v, 3) for k, v in sorted(stage.items()) if k.startswith("host_ms_")},
        "work": {k: stage.get(k) for k in ("paths", "railroad_settled", "railroad_touched", "invalidated", "foreground")},
        "graph": {k: stage.get(k) for k in ("graph_launches", "graph_updates", "graph_instantiations")},
        "autotune": tuned,
        "roofline": {"kernel": "trace_kernel", "stage_dominant": dominant, "bound": "hbm", "achieved": achieved,
                     "peak": peak, "peak_source": source, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "algorithmic_bytes": trace_bytes},
        "e2e": {"value": voxels / (e2e_ms / 1e3), "unit": "voxels/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": int(volume.nbytes), "d2h_bytes_per_step": result_bytes(packed_h)},
        "gpu_launches": int(stage.get("launches", 0) * args.steps),
        "clocks": clocks.summary(),
    }
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(volume, cfg, os.cpu_count() or 1)
    if world == 1 and not args.no_extras:
        out.update(extra_measurements(local, packed))
    print(json.dumps(out))
    if dist is not None:
        dist.destroy_process_group()


def run_streamed(args, cfg):
    """The out-of-core workload: host labels to host skeletons through skeletonize(streaming=True)
    (the device budget: a quarter of the free memory), wall clock per call after one warm-up call
    on a 128^3 crop, with the call's own breakdown (slabs, crop batches, host and device stages)."""
    import torch

    import brook_b200
    from brook_b200 import _native

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    volume = make_volume(cfg)
    torch.cuda.empty_cache()
    opts = dict(teasar_params=PARAMS, anisotropy=cfg["anisotropy"], dust_threshold=DUST, device=local)
    brook_b200.skeletonize(np.asfortranarray(volume[:128, :128, :128]), streaming=True, output="packed", **opts)
    times, stats = [], {}
    for _ in range(max(1, args.steps)):
        t0 = time.perf_counter()
        packed = brook_b200.skeletonize(volume, streaming=True, output="packed", **opts)
        times.append(time.perf_counter() - t0)
        stats = _native.stats(local)
    ms = 1e3 * float(np.mean(times))
    voxels = int(volume.size)
    print(json.dumps({
        "metric": METRIC, "value": voxels / (ms / 1e3), "unit": "voxels/s", "n_gpus": 1, "steps": len(times),
        "warmup": 1, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32/f32", "data": "synthetic", "skeletons_per_s": len(packed) / (ms / 1e3),
        "config": {"workload": cfg["workload"], "voxels": voxels, "anisotropy": cfg["anisotropy"], "teasar": PARAMS,
                   "dust_threshold": DUST, "timing": "wall clock, host labels in, host skeletons out"},
        "skeletons": len(packed), "vertices": int(packed.v_off[-1]),
        "streamed": {k: round(v, 3) for k, v in sorted(stats.items())},
    }))


def run_post(args, cfg):
    """Only the canonical post-processing of the configuration's skeletons (one skeletonize call
    makes them): the post_measurement figures as one JSON line; the profiling entry point of the
    post-processing kernels."""
    import torch

    import brook_b200

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    volume = make_volume(cfg)
    packed = brook_b200.skeletonize(volume, teasar_params=PARAMS, anisotropy=cfg["anisotropy"], dust_threshold=DUST,
                                    output="packed", device=local)
    r = post_measurement(local, packed, steps=args.steps)
    print(json.dumps({"metric": "canonical post-processing ms per call", "value": r["ms_per_call"], "unit": "ms",
                      "higher_is_better": False, "steps": args.steps, "config": {"workload": cfg["workload"]},
                      "post": r}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="dense512", choices=sorted(CONFIGS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the batch and serving comparisons")
    ap.add_argument("--no-autotune", action="store_true", help="keep the engine's built-in launch rule")
    ap.add_argument("--post-only", action="store_true",
                    help="time only the canonical post-processing of the configuration's skeletons")
    args = ap.parse_args()
    cfg = CONFIGS[args.config]
    if args.post_only:
        run_post(args, cfg)
    elif args.impl == "reference":
        run_reference(args, cfg)
    elif cfg["kind"] == "batch":
        run_batch(args, cfg)
    elif cfg["kind"] == "serve":
        run_serve(args, cfg)
    elif cfg["kind"] == "chunks":
        run_chunks(args, cfg)
    elif cfg["kind"] == "streamed":
        run_streamed(args, cfg)
    else:
        run_ours(args, cfg)


if __name__ == "__main__":
    main()
