"""Benchmark: ms per frame of the collision pipeline on the 0.5M-triangle
cloth draped over a 40,500-triangle icosphere (512x512 cloth, damped-wave
fold, heuristic schedule: build every 12 frames, front cycle 6).

One step = one frame (BVH maintain + front maintain + narrow phase) through
the C ABI.  `value` times frames with inputs already resident in HBM;
`e2e` times the same frames with the vertex upload from pinned host memory
and the read-back of the contact pairs inside the timed region.  The L2 is
flushed between timed frames, outside the frame's events: a 256 MB write, then
a 256 MB read that makes the flush write its own dirty lines back
(--l2-flush dirty: the write alone).

The JSON line also carries "batched": 256 independent scenes (about 9.7M
triangles) as one forest with graph-launched frames, against the same scenes
run one by one through their own handles (scene-frames/s, p50/p99 frame
times, and a per-scene pair-set check of the two forms), and "learned": the
learned scheduler against the reference's heuristic on a held-out 1M-triangle
cloth (learn.py).

--impl reference times the CPU restatement of the reference pipeline
(oracle/, OpenMP on all host cores) on the same workload: the reference
ships only a GPU path, so this is its logic on the host cores.

Multi-GPU: one process per GPU (torchrun); each rank runs an independent
replica of the frame sequence (a single scene does not shard), so per-GPU
work is fixed ("scaling": "weak"); value = max device time over ranks / all
frames of all ranks.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "bvh-based-collision-detection-scheme_b200")
sys.path.insert(0, PKG)

WORKLOAD = "cloth512_over_icosphere45"
METRIC = "ms_per_frame_cloth512_over_sphere"
CAPS = dict(int_front_capacity=16_000_000, ext_front_capacity=16_000_000, pair_capacity=4_000_000)


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi's start-up (driver attach, first query) can hold the
            # launch path for milliseconds: the timed region starts after its
            # first sample has arrived
            t_end = time.perf_counter() + 5.0
            while not self.rows and time.perf_counter() < t_end and self.proc.poll() is None:
                time.sleep(0.01)
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


class L2Flush:
    """Between timed frames, outside their events: a 256 MB write (twice the
    126 MB L2), then -- unless `dirty` -- a 256 MB read of another buffer.
    The write alone leaves the L2 full of the flush buffer's dirty lines,
    whose write-back the next frame would pay as its own loads evict them;
    the read makes the flush write them back itself, so a frame starts with
    none of its data in L2 and no foreign dirty lines either."""

    N = 256 * 1024 * 1024 // 4

    def __init__(self, torch, dirty=False):
        self.w = torch.empty(self.N, dtype=torch.float32, device="cuda")
        self.r = None if dirty else torch.zeros(self.N, dtype=torch.float32, device="cuda")
        self.desc = ("flushed between frames (256 MB write" +
                     (")" if dirty else ", then a 256 MB read so the flush's dirty lines leave L2 before the frame)"))

    def __call__(self):
        self.w.zero_()
        if self.r is not None:
            self.r.sum()


FLUSH_DIRTY = False  # --l2-flush dirty: the write alone


def gpu_lead(torch, stream, ms=5.0):
    """A bounded busy-wait kernel (a clock-cycle count) ahead of a timed loop,
    outside its events: the host enqueues the first frames while it runs, so a
    host hiccup early in the loop cannot leave the GPU idle inside a frame's
    interval.  It changes no frame's work."""
    with torch.cuda.stream(stream):
        torch.cuda._sleep(int(ms * 1e-3 * 2.0e9))


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


CLOTH = 512  # cloth side in vertices (--cloth; 512 is the headline workload)


def make_frames(n):
    import scenes
    return scenes.cloth_over_sphere_frames(CLOTH, n)


def run_ours(args):
    import torch
    import torch.distributed as dist

    import bvhcd

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    if not bvhcd.device_check(local):
        raise RuntimeError("libbvhcd.so has no sm_100a code for this GPU")
    W, K = args.warmup, args.steps
    faces, frames = make_frames(W + K)
    # no cyclic garbage collection while frames are timed: a collection between
    # a frame's launches would leave the GPU idle inside the frame's events
    gc.collect()
    gc.disable()
    T, V = faces.shape[0], frames[0].shape[0]
    stream = torch.cuda.current_stream()
    host = torch.from_numpy(np.stack(frames)).pin_memory()          # (W+K, V, 3) pinned
    dev = host.to("cuda", non_blocking=False)                       # resident copy for `value`
    dfaces = torch.from_numpy(faces).cuda()
    flush = L2Flush(torch, FLUSH_DIRTY)
    flush_desc = flush.desc  # (the buffers are released before the JSON line is written)

    def pipeline():
        bvh = bvhcd.LBvh(T, V, enable_restr=True)
        front = bvhcd.BvttFront(bvh, cull_adjacent=True, narrow_phase=True, auto_grow=False, **CAPS)
        return bvh, front

    # Every code path of the schedule runs once before anything is timed, on a
    # pipeline that is then dropped: a kernel's first launch in a process loads
    # its code (CUDA's lazy module loading) and can stall the GPU for
    # milliseconds, and with few warm-up frames the first update or balance
    # would otherwise come inside the timed frames.
    wb, wf = pipeline()
    for f in range(min(W + K, 25)):
        bvhcd.frame(wb, wf, f, 0, dev[f], dfaces, stream=stream, faces_static=f > 0)
    torch.cuda.synchronize()
    wf.close()
    wb.close()

    # ---- value: device-resident inputs
    bvh, front = pipeline()
    for f in range(W):
        bvhcd.frame(bvh, front, f, 0, dev[f], dfaces, stream=stream, faces_static=f > 0)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    l0 = bvhcd.launch_count()
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        gpu_lead(torch, stream)
        for i in range(K):
            f = W + i
            flush()
            starts[i].record(stream)
            bvhcd.frame(bvh, front, f, 0, dev[f], dfaces, stream=stream, faces_static=True)
            ends[i].record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    launches = bvhcd.launch_count() - l0 - 0
    per = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    dev_ms = float(sum(per))
    st = front.stats()
    if st["overflow_any"]:  # sticky: any overflow in any warm-up or timed frame
        raise RuntimeError(f"front/pair capacity overflow during the bench: {st}")
    if world > 1:
        t = torch.tensor([dev_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_ms = float(t.item())
        dist.barrier()
    value = dev_ms / (K * world)

    e2e = roof = batched = fp16 = inter = boxes = prox = grow = None
    if not args.only_value:
        e2e = e2e_pass(bvhcd, torch, pipeline, host, faces, dfaces, flush, stream, W, K, V, world)
        # roofline of the dominant stage, from a stage-timed replay
        roof = roofline_pass(bvhcd, torch, faces, dev, dfaces, stream, W, K, T)
        grow = autogrow_pass(bvhcd, torch, dev, dfaces, stream, W, K, T)
        fp16 = fp16_pass(bvhcd, torch, faces, dev, dfaces, stream, W, K, T)
        inter = inter_pass(bvhcd, torch, faces, dev, dfaces, stream, W, K, st)
        boxes = box_pass(bvhcd, torch, faces, dev, dfaces, stream, W, K, T)
        prox = proximity_pass(bvhcd, torch, front, stream)
    learned = prec = prec_keep = None
    if not args.only_value and not args.no_precision:
        del dev, host, flush
        torch.cuda.empty_cache()
        prec, prec_keep = precision_pass(bvhcd, torch, stream, args)
    if not args.only_value and not args.no_batched:
        dev = host = flush = None
        torch.cuda.empty_cache()
        batched = batched_pass(bvhcd, torch, args, world, rank)
    if not args.only_value and not args.no_learned:
        torch.cuda.empty_cache()
        learned = learned_pass(torch, args)

    out = None
    if rank == 0:
        cpu = cpu_baseline(faces, frames, args) if world == 1 and not args.no_cpu_baseline else None
        if prec is not None and cpu is not None:
            prec["cpu_check"] = precision_check(prec_keep)
        out = {
            "metric": METRIC, "value": round(value, 4), "unit": "ms/frame", "n_gpus": world,
            "steps": K, "warmup": W, "ms_per_step": round(value * world, 4), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD if CLOTH == 512 else f"cloth{CLOTH}_over_icosphere45", "triangles": T, "vertices": V,
                       "frames_timed": K, "schedule": "build/12, front cycle 6 (STATIC_MANDATORY, divergent marks)",
                       "restructure": "quality-triggered (enabled)", "adjacency_culling": True,
                       "narrow_phase": "fp32 17-axis SAT",
                       "l2": flush_desc,
                       "parallelism": "replicas" if world > 1 else "single-gpu",
                       "front_sizes_last_frame": [st["int_front"], st["ext_front"]],
                       "pairs_last_frame": [st["broad_pairs"], st["narrow_hits"]]},
            "wall_s_timed_region": round(wall, 4),
            "per_frame_ms": {"median": round(statistics.median(per), 4), "max": round(max(per), 4),
                             "min": round(min(per), 4),
                             "slowest": [[W + int(k), round(per[k], 4)] for k in np.argsort(per)[::-1][:3]]},
            "e2e": e2e,
            "gpu_launches": int(launches),
            "roofline": roof,
            "clocks": clk.summary(),
            "auto_grow": grow,
            "fp16_node_boxes": fp16,
            "precision": prec,
            "inter_rigid_obstacle": inter,
            "box_scene": boxes,
            "proximity": prox,
            "batched": batched,
            "learned": learned,
        }
        if cpu:
            out["cpu_baseline"] = cpu
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return out


def e2e_pass(bvhcd, torch, pipeline, host, faces, dfaces, flush, stream, W, K, V, world):
    """Same frames through the public API with host buffers: each frame's
    vertex positions go from pinned host memory to HBM and the intersecting
    pairs come back to pinned host memory, both inside the timed frames.  The
    positions of frame f + 1 are staged (bvhcd_bvh_stage_positions) on a copy
    stream while frame f computes; frame f's interval ends only after that
    copy has landed, so every upload is inside a timed interval (the first
    frame's own upload inside the first).  The pairs are written into mapped
    host memory by the library's read-back kernel (bvhcd_front_pairs_async),
    alternating between two buffers, with no host synchronisation between
    frames; the last frame's pairs are checked against a synchronous read."""
    import torch.distributed as dist
    import ctypes
    bvh2, front2 = pipeline()
    copy = torch.cuda.Stream()
    L = bvhcd.lib()
    cap = CAPS["pair_capacity"]
    region = ctypes.c_void_p()
    if L.bvhcd_host_alloc(8 * K + 2 * 8 * cap, ctypes.byref(region)) != 0:
        raise RuntimeError("mapped host allocation failed")
    base = region.value
    bufs = [base + 8 * K, base + 8 * K + 8 * cap]
    for f in range(W):
        staged = bvh2.stage_positions(host[f], copy)
        bvhcd.frame(bvh2, front2, f, 0, staged, dfaces, stream=stream, faces_static=f > 0)
    torch.cuda.synchronize()
    e_starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    e_ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    staged = None
    gpu_lead(torch, stream)
    for i in range(K):
        f = W + i
        flush()
        e_starts[i].record(stream)
        if staged is None:
            copy.wait_event(e_starts[i])
            staged = bvh2.stage_positions(host[f], copy)
        bvhcd.frame(bvh2, front2, f, 0, staged, dfaces, stream=stream, faces_static=True)
        staged = bvh2.stage_positions(host[f + 1], copy) if i + 1 < K else None
        st2 = L.bvhcd_front_pairs_async(front2.handle, 1, ctypes.c_void_p(bufs[i % 2]), cap,
                                        ctypes.c_void_p(base + 8 * i), ctypes.c_void_p(stream.cuda_stream))
        if st2 != 0:
            raise RuntimeError(f"pairs read-back failed: {st2}")
        stream.wait_stream(copy)
        e_ends[i].record(stream)
    torch.cuda.synchronize()
    e2e_ms = float(sum(s.elapsed_time(e) for s, e in zip(e_starts, e_ends)))
    counts = np.frombuffer((ctypes.c_char * (8 * K)).from_address(base), dtype=np.int64).copy()
    last = np.frombuffer((ctypes.c_char * (8 * cap)).from_address(bufs[(K - 1) % 2]), dtype=np.int32)
    last = last[:2 * int(counts[-1])].reshape(-1, 2).copy()
    ref = front2.pairs(narrow=True)
    same = bool(np.array_equal(last, ref))
    L.bvhcd_host_free(region)
    front2.close()
    bvh2.close()
    if not same:
        raise RuntimeError("asynchronously read pairs differ from the synchronous read")
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    return {"value": e2e_ms / (K * world), "unit": "ms/frame", "h2d_bytes_per_step": int(V * 12),
            "d2h_bytes_per_step": int((8 * counts.sum() + 8 * K) // K),
            "upload": "positions of frame f + 1 staged on a copy stream during frame f",
            "download": "intersecting pairs and their count written into mapped pinned host memory by a kernel "
                        "every frame (bvhcd_front_pairs_async); no host synchronisation between frames",
            "pairs_equal_synchronous_read": same}


# Per-stage DRAM traffic (read + write bytes per call) of this workload, from
# the ncu captures summarised in the profiles folder: the file lists, per
# stage, the summed dram__bytes of that stage's kernels per call.
STAGE_TRAFFIC_FILE = os.path.join(ROOT, "profiles", "dram_per_stage_cloth512_sphere.txt")


def _stage_traffic():
    out = {}
    try:
        with open(STAGE_TRAFFIC_FILE) as f:
            for line in f:
                line = line.split("#", 1)[0].split()
                if len(line) == 2:
                    out[line[0]] = float(line[1])
    except OSError:
        pass
    return out


def _uniq_nodes(front):
    """Distinct tree records a front references (internal nodes of the
    internal front, leaves of the external one): the U of the algorithmic-
    bytes formulas, counted on the exported front (a lower bound of the
    records a traversal touches)."""
    fi, fe = front.export(0), front.export(1)
    return len(np.unique(fi[:, 1])) + len(np.unique(fe[:, 1]))


def stage_bytes(stage, T, V, F_in, F_out, U, P, H, pairs=None, faces=None, passes=4):
    """Algorithmic bytes of one call of a stage, per the hot-path scope
    table's measurement formulas (FP32 records):
      refit   12V + 12T + 24T + 24(T-1)*3 + 8(T-1)
      build   refit + 8T + 16T per radix pass + 16T + 8T
      front maintenance (generate / update / keep / balance)
              8 F_in + 12 F_out + 24T + 32U + 8P
      reorder 16F + 4(2T) + 4(2T)*2
      narrow  8P + 12 T_touched + 12 V_touched + 8H"""
    refit = 12 * V + 12 * T + 24 * T + 24 * (T - 1) * 3 + 8 * (T - 1)
    if stage == "bvh_refit":
        return refit
    if stage == "bvh_build":
        return refit + 8 * T + 16 * T * passes + 16 * T + 8 * T
    if stage in ("front_generate", "front_update", "front_keep", "front_balance"):
        return 8 * F_in + 12 * F_out + 24 * T + 32 * U + 8 * P
    if stage == "front_reorder":
        return 16 * F_out + 4 * 2 * T + 4 * 2 * T * 2
    if stage == "narrow":
        tt = len(np.unique(pairs)) if pairs is not None and len(pairs) else 0
        vt = len(np.unique(faces[np.unique(pairs)])) if tt else 0
        return 8 * P + 12 * tt + 12 * vt + 8 * H
    return None


def roofline_pass(bvhcd, torch, faces, dev, dfaces, stream, W, K, T):
    """Replays the frames with stage events on and reads the stage times after
    every frame.  For every stage: calls, average event time per call,
    algorithmic bytes per call (stage_bytes, with this run's front sizes,
    pair counts and distinct records), achieved GB/s and its fraction of the
    measured HBM copy bandwidth, and the DRAM traffic per call from the ncu
    capture of the stage's kernels.  The top-level figures are those of the
    dominant stage (the largest total time over the timed frames)."""
    peak, kind = _peaks()
    V = dev.shape[1]
    traffic = _stage_traffic()
    bvh = bvhcd.LBvh(T, V, enable_restr=True)
    front = bvhcd.BvttFront(bvh, cull_adjacent=True, narrow_phase=True, auto_grow=False, **CAPS)
    bvh.profile(True)
    flush = L2Flush(torch, FLUSH_DIRTY)
    acc = {}   # stage -> [ms, calls, bytes]
    prev = None
    U = 0
    for f in range(W + K):
        flush()
        bvhcd.frame(bvh, front, f, 0, dev[f], dfaces, stream=stream, faces_static=f > 0)
        times = bvh.stage_times(reset=True)
        st = front.stats(stream)
        F = st["int_front"] + st["ext_front"]
        op = st["front_op_run"]
        if op in (bvhcd.FRONT_GENERATE, bvhcd.FRONT_UPDATE, bvhcd.FRONT_REORDER) or prev is None:
            U = _uniq_nodes(front)
        if f < W:
            prev = st
            continue
        F_prev = prev["int_front"] + prev["ext_front"]
        P, H = st["broad_pairs"], st["narrow_hits"]
        hits = None
        for stage, (ms, calls) in times.items():
            if not calls:
                continue
            if stage == "front_generate":
                b = stage_bytes(stage, T, V, 0, F, U, P, H)
            elif stage == "front_update":
                b = stage_bytes(stage, T, V, F_prev, F, U, P, H)
            elif stage == "front_keep":
                b = stage_bytes(stage, T, V, F, 0, U, P, H)
                if not times.get("narrow", (0, 0))[1]:
                    # the keep's last launch ran its narrow phase (one launch with
                    # the traversals below overlapping entries): its bytes count here
                    if hits is None:
                        hits = front.pairs()
                    b += stage_bytes("narrow", T, V, 0, 0, U, P, H, pairs=hits, faces=faces)
            elif stage == "front_balance":
                b = stage_bytes(stage, T, V, F, st["int_front"], U, P, H)
            elif stage == "front_reorder":
                b = stage_bytes(stage, T, V, F, F, U, P, H)
            elif stage == "narrow":
                if hits is None:
                    hits = front.pairs()
                b = stage_bytes(stage, T, V, 0, 0, U, P, H, pairs=hits, faces=faces)
            else:
                b = stage_bytes(stage, T, V, 0, 0, U, P, H)
            a = acc.setdefault(stage, [0.0, 0, 0.0, b is not None])
            a[0] += ms
            a[1] += calls
            a[2] += (b or 0) * calls
        prev = st
    front.close()
    bvh.close()
    stages = {}
    for stage, (ms, calls, byts, has_bytes) in acc.items():
        avg = ms / calls
        e = {"calls": calls, "avg_launch_ms": round(avg, 4), "total_ms": round(ms, 3)}
        if has_bytes:
            algo = byts / calls
            ach = algo / (avg * 1e-3) / 1e9
            e.update({"algorithmic_bytes_per_call": int(algo), "achieved": round(ach, 1),
                      "frac": round(ach / peak, 4)})
        tr = traffic.get(stage)
        e["traffic"] = tr
        stages[stage] = e
    dom = max(stages.items(), key=lambda kv: kv[1]["total_ms"])
    d = dom[1]
    maint = [k for k in ("front_keep", "front_update", "front_balance", "front_reorder") if k in stages]
    m_bytes = sum(stages[k]["algorithmic_bytes_per_call"] * stages[k]["calls"] for k in maint)
    m_ms = sum(stages[k]["total_ms"] for k in maint)
    return {"kernel": f"{dom[0]} stage", "bound": "hbm", "achieved": d.get("achieved"), "peak": peak,
            "unit": "GB/s", "frac": d.get("frac"), "peak_source": kind,
            "traffic": d.get("traffic"),
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the stage's kernels per call "
                              "(profiles/dram_per_stage_cloth512_sphere.txt)",
            "algorithmic_bytes_per_launch": d.get("algorithmic_bytes_per_call"),
            "avg_launch_ms": d["avg_launch_ms"], "dominant_stage": dom[0],
            "front_maintenance": {"stages": maint, "achieved": round(m_bytes / (m_ms * 1e-3) / 1e9, 1) if m_ms else None,
                                  "frac": round(m_bytes / (m_ms * 1e-3) / 1e9 / peak, 4) if m_ms else None},
            "U": "distinct records the front references (exported front; a lower bound)",
            "stages": stages}


def _pct(xs, q):
    xs = sorted(xs)
    return xs[min(len(xs) - 1, int(round(q * (len(xs) - 1))))]


def batched_pass(bvhcd, torch, args, world, rank):
    """256 independent cloth-over-sphere scenes (triangle counts log-uniform in
    [1k, 200k]).  Batched form: one forest (bvhcd_bvh_set_scenes), every frame
    one graph-launched sequence of per-stage launches over all scenes
    (bvhcd_frame_graph).  Plain form: the same scenes one after another, each
    through its own BVH/front handles.  Inputs are resident in HBM; the
    working set (fronts of ~10M triangles) is far larger than L2, so L2 is not
    flushed.  Multi-GPU: scenes are dealt to ranks by a greedy triangle-count
    balance; each rank runs its share."""
    import scenes
    import torch.distributed as dist
    F = args.batched_frames
    B = scenes.BatchedScenes()
    sizes = np.diff(B.tri_offsets)
    mine = scenes.shard_scenes(sizes, world, rank)
    faces, off, vidx = B.subset(mine)
    T, V, S = int(off[-1]), int(vidx.size), len(mine)
    stream = torch.cuda.Stream()      # graphs are captured on a stream of their own
    with torch.cuda.stream(stream):
        return _batched_on(bvhcd, torch, args, world, B, sizes, off, faces, vidx, T, V, S, stream)


def _batched_on(bvhcd, torch, args, world, B, sizes, off, faces, vidx, T, V, S, stream):
    import torch.distributed as dist
    F = args.batched_frames
    frames_dev = torch.empty((F, V, 3), dtype=torch.float32, device="cuda")
    for f in range(F):
        frames_dev[f].copy_(torch.from_numpy(B.positions(f)[vidx]))
    dfaces = torch.from_numpy(faces).cuda()
    pos = torch.empty((V, 3), dtype=torch.float32, device="cuda")
    sched = [bvhcd.schedule(f) for f in range(F)]

    # ---- batched form: captured graphs; two untimed passes capture every key
    bvh = bvhcd.LBvh(T, V, enable_restr=False)
    bvh.set_scenes(off)
    front = bvhcd.BvttFront(bvh, int_front_capacity=24 * T, ext_front_capacity=16 * T, pair_capacity=4 * T,
                            cull_adjacent=True, narrow_phase=True, auto_grow=False)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(F)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(F)]
    l0 = bvhcd.launch_count()
    shapes = tuned_ms = None
    for rep in range(3):
        if rep == 2:
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            l0 = bvhcd.launch_count()
        for f in range(F):
            pos.copy_(frames_dev[f])
            if rep == 2:
                starts[f].record(stream)
            bvhcd.frame_graph(bvh, front, pos, dfaces, sched[f][0], sched[f][1], stream=stream)
            if rep == 2:
                ends[f].record(stream)
            if rep == 0 and f == 0:
                # the project's autotuner picks the launch shapes on this batch
                shapes, tuned_ms = front.autotune(3, stream=stream)
    torch.cuda.synchronize()
    launches = bvhcd.launch_count() - l0
    per = [a.elapsed_time(b) for a, b in zip(starts, ends)]
    st = front.stats()
    if st["overflow_any"]:
        raise RuntimeError(f"batched front/pair capacity overflow: {st}")
    batched_pairs = (front.pairs(), front.pairs(narrow=True))
    total_ms = float(sum(per))

    # ---- plain form: one handle pair per scene, scenes one after another
    hs = []
    for k in range(S):
        a0, a1 = int(off[k]), int(off[k + 1])
        fl = faces[a0:a1]
        v0, v1 = int(fl.min()), int(fl.max()) + 1
        b1 = bvhcd.LBvh(a1 - a0, v1 - v0, enable_restr=False)
        f1 = bvhcd.BvttFront(b1, int_front_capacity=24 * (a1 - a0), ext_front_capacity=16 * (a1 - a0),
                             pair_capacity=4 * (a1 - a0) + 1024, cull_adjacent=True, narrow_phase=True,
                             auto_grow=True)
        hs.append((b1, f1, torch.from_numpy(fl - v0).cuda(), v0, v1))
    p_starts = [[torch.cuda.Event(enable_timing=True) for _ in range(S)] for _ in range(F)]
    p_ends = [[torch.cuda.Event(enable_timing=True) for _ in range(S)] for _ in range(F)]
    for rep in range(2):
        if rep == 1:
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
        for f in range(F):
            pos.copy_(frames_dev[f])
            for k, (b1, f1, fl, v0, v1) in enumerate(hs):
                if rep == 1:
                    p_starts[f][k].record(stream)
                b1.maintain(sched[f][0], pos[v0:v1], fl, stream=stream)
                f1.maintain(sched[f][1], stream=stream)
                if rep == 1:
                    p_ends[f][k].record(stream)
    torch.cuda.synchronize()
    plain_frame = [sum(p_starts[f][k].elapsed_time(p_ends[f][k]) for k in range(S)) for f in range(F)]
    plain_scene = [p_starts[f][k].elapsed_time(p_ends[f][k]) for f in range(F) for k in range(S)]
    plain_ms = float(sum(p_starts[f][0].elapsed_time(p_ends[f][S - 1]) for f in range(F)))

    # the last frame's per-scene pair sets must be the plain form's
    equal = True
    for which in (0, 1):
        p = np.sort(batched_pairs[which].astype(np.int64), axis=1)
        sc = np.searchsorted(off, p[:, 0], side="right") - 1
        equal &= bool(np.array_equal(sc, np.searchsorted(off, p[:, 1], side="right") - 1))
        for k, (b1, f1, fl, v0, v1) in enumerate(hs):
            q = p[sc == k] - off[k]
            r = np.sort(f1.pairs(narrow=bool(which)).astype(np.int64), axis=1)
            equal &= q.shape == r.shape and bool(np.array_equal(q[np.lexsort((q[:, 1], q[:, 0]))],
                                                                r[np.lexsort((r[:, 1], r[:, 0]))]))
    for b1, f1, *_ in hs:
        f1.close()
        b1.close()
    front.close()
    bvh.close()
    if world > 1:
        t = torch.tensor([total_ms, plain_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms, plain_ms = float(t[0].item()), float(t[1].item())
    n_all = B.num_scenes
    return {
        "workload": f"{n_all} independent cloth-over-sphere scenes, {B.num_faces} triangles "
                    f"({int(sizes.min())}..{int(sizes.max())} per scene, log-uniform), {F} frames",
        "metric": "scenes_per_s", "unit": "scene-frames/s",
        "value": round(n_all * F / (total_ms * 1e-3), 1),
        "frame_ms": {"p50": round(_pct(per, 0.5), 4), "p99": round(_pct(per, 0.99), 4),
                     "mean": round(total_ms / F, 4)},
        "per_scene_frame_ms": {"p50": round(_pct(per, 0.5), 4), "p99": round(_pct(per, 0.99), 4),
                               "note": "every scene's frame completes with the batch's"},
        "graph_launched": True, "gpu_launches": int(launches), "l2": "not flushed (working set >> L2)",
        "autotuned_shapes": {k: {"unroll": v[0], "block": v[1]} for k, v in shapes.items()},
        "autotune_best_ms": {k: round(v, 4) for k, v in tuned_ms.items()},
        "plain": {"value": round(n_all * F / (plain_ms * 1e-3), 1), "unit": "scene-frames/s",
                  "frame_ms": {"p50": round(_pct(plain_frame, 0.5), 4), "p99": round(_pct(plain_frame, 0.99), 4)},
                  "per_scene_frame_ms": {"p50": round(_pct(plain_scene, 0.5), 4),
                                         "p99": round(_pct(plain_scene, 0.99), 4)}},
        "speedup_vs_plain": round(plain_ms / total_ms, 3),
        "pairs_equal_plain_last_frame": bool(equal),
        "shard": {"ranks": world, "scenes_this_rank": int(S), "triangles_this_rank": int(T)},
    }


def inter_pass(bvhcd, torch, faces, dev, dfaces, stream, W, K, single):
    """The same frames with the sphere as a rigid obstacle: the cloth in its own
    BVH with an intra front, the sphere in a rigid BVH (refit every frame) and
    an inter front between them, both fronts on the reference's schedule.
    Device ms per frame, timed as `value`; the last frame's pair counts of the
    two fronts plus the sphere's own (static) pairs must equal the single
    front's over the joined scene."""
    Vc = 512 * 512
    Tc = 2 * 511 * 511
    assert int(faces[:Tc].max()) < Vc and int(faces[Tc:].min()) >= Vc
    cfaces = dfaces[:Tc].contiguous()
    sfaces = (dfaces[Tc:] - Vc).contiguous()
    Ts, Vs = faces.shape[0] - Tc, dev.shape[1] - Vc
    cbvh = bvhcd.LBvh(Tc, Vc, enable_restr=True)
    sbvh = bvhcd.LBvh(Ts, Vs, enable_restr=False)
    intra = bvhcd.BvttFront(cbvh, cull_adjacent=True, narrow_phase=True, auto_grow=False, **CAPS)
    inter = bvhcd.BvttFront(cbvh, rigid=sbvh, narrow_phase=True, auto_grow=False, **CAPS)
    own = bvhcd.BvttFront(sbvh, cull_adjacent=True, narrow_phase=True, auto_grow=False, **CAPS)
    flush = L2Flush(torch, FLUSH_DIRTY)

    def frame(f):
        b, fr = bvhcd.schedule(f)
        cbvh.maintain(b, dev[f][:Vc], cfaces, stream=stream, faces_static=f > 0)
        intra.maintain(fr, stream=stream)
        sbvh.maintain(bvhcd.BVH_BUILD if f == 0 else bvhcd.BVH_REFIT, dev[f][Vc:], sfaces, stream=stream,
                      faces_static=f > 0)
        inter.maintain(fr, stream=stream)

    for f in range(W):
        frame(f)
    own.maintain(bvhcd.FRONT_GENERATE, stream=stream)  # the static sphere's own pairs, once
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    torch.cuda.synchronize()
    for i in range(K):
        flush()
        starts[i].record(stream)
        frame(W + i)
        ends[i].record(stream)
    torch.cuda.synchronize()
    ms = float(sum(a.elapsed_time(b) for a, b in zip(starts, ends))) / K
    si, sx, so = intra.stats(), inter.stats(), own.stats()
    if si["overflow_any"] or sx["overflow_any"] or so["overflow_any"]:
        raise RuntimeError(f"inter leg overflow: {si} {sx} {so}")
    pairs = [si["broad_pairs"] + sx["broad_pairs"] + so["broad_pairs"],
             si["narrow_hits"] + sx["narrow_hits"] + so["narrow_hits"]]
    restr = inter_restructure_timing(bvhcd, torch, cbvh, sbvh, intra, inter, dev[W + K - 1], cfaces, sfaces, Vc,
                                     flush, stream)
    for h in (own, inter, intra):
        h.close()
    sbvh.close()
    cbvh.close()
    return {"workload": f"cloth 512x512 ({Tc} triangles, own BVH, intra front) with the icosphere ({Ts} triangles) "
                        "as a rigid obstacle BVH refit every frame, inter front between them",
            "value": round(ms, 4), "unit": "ms/frame",
            "pairs_last_frame": {"cloth_self": [si["broad_pairs"], si["narrow_hits"]],
                                 "cloth_sphere": [sx["broad_pairs"], sx["narrow_hits"]],
                                 "sphere_self": [so["broad_pairs"], so["narrow_hits"]]},
            "pairs_equal_single_front": pairs == [single["broad_pairs"], single["narrow_hits"]],
            "front_restructure": restr}


def _restructure_roots(inode, frac=0.2, lo=16, hi=512):
    """Disjoint subtrees (DFS ids) of lo..hi leaves covering about `frac` of
    the internal nodes, in DFS order: the marks a front-quality check leaves."""
    size = inode[:, 5] - inode[:, 4] + 1
    covered = np.zeros(inode.shape[0] + 1, bool)
    chosen, total = [], 0
    for d in range(inode.shape[0]):
        if lo <= size[d] <= hi and not covered[d]:
            chosen.append(d)
            covered[d:d + size[d] - 1] = True
            total += size[d] - 1
            if total >= frac * inode.shape[0]:
                break
    return np.array(chosen, np.int32)


def inter_restructure_timing(bvhcd, torch, cbvh, sbvh, intra, inter, pos, cfaces, sfaces, Vc, flush, stream):
    """The inter front after a restructure of the cloth's BVH (subtrees
    covering a fifth of its internal nodes marked, as a quality check would):
    CUDA-event time of the front restructure (valid entries kept, the
    restructured subtrees re-sprouted: BvttFrontLooseInter::restructure)
    against a regeneration of the same front on the same trees, and whether
    the two give the same pairs."""
    cbvh.request_restructure(_restructure_roots(cbvh.export()["inode"]), stream=stream)
    cbvh.maintain(bvhcd.BVH_REFIT, pos[:Vc], cfaces, stream=stream, faces_static=True)
    tag = cbvh.opt_tag()
    intra.maintain(bvhcd.FRONT_KEEP, stream=stream)
    sbvh.maintain(bvhcd.BVH_REFIT, pos[Vc:], sfaces, stream=stream, faces_static=True)
    out = {"bvh_opt_tag": tag}
    for name, op in (("resprout", bvhcd.FRONT_KEEP), ("regenerate", bvhcd.FRONT_GENERATE)):
        flush()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        inter.maintain(op, stream=stream)
        b.record(stream)
        torch.cuda.synchronize()
        st = inter.stats(stream)
        out[name] = {"ms": round(a.elapsed_time(b), 4), "front_op_run": st["front_op_run"],
                     "pairs": st["broad_pairs"], "fronts": [st["int_front"], st["ext_front"]]}
        out[name + "_pairs"] = bvhcd_canon(inter.pairs(stream=stream))
    out["pairs_equal"] = bool(np.array_equal(out.pop("resprout_pairs"), out.pop("regenerate_pairs")))
    out["speedup"] = round(out["regenerate"]["ms"] / out["resprout"]["ms"], 3) if out["resprout"]["ms"] else None
    return out


def bvhcd_canon(p):
    p = np.asarray(p, dtype=np.int64).reshape(-1, 2)
    return p[np.lexsort((p[:, 1], p[:, 0]))]


def autogrow_pass(bvhcd, torch, dev, dfaces, stream, W, K, T):
    """The same device-resident frames through fronts with the two
    auto_grow modes an integrator can pick: 2 (deferred: each maintain copies
    its counters to pinned host memory, a later one acts on an overflow; no
    synchronisation) and 1 (grow and replay inside the call: every maintain
    reads the counters back).  The capacities are the bench's, so nothing
    overflows; both give the main loop's pairs."""
    flush = L2Flush(torch, FLUSH_DIRTY)
    out = {}
    for mode, name in ((2, "deferred"), (1, "sync")):
        bvh = bvhcd.LBvh(T, dev.shape[1], enable_restr=True)
        front = bvhcd.BvttFront(bvh, cull_adjacent=True, narrow_phase=True, auto_grow=mode, **CAPS)
        for f in range(W):
            bvhcd.frame(bvh, front, f, 0, dev[f], dfaces, stream=stream, faces_static=f > 0)
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in range(K):
            flush()
            starts[i].record(stream)
            bvhcd.frame(bvh, front, W + i, 0, dev[W + i], dfaces, stream=stream, faces_static=True)
            ends[i].record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        st = front.stats()
        if st["overflow_any"]:
            raise RuntimeError(f"auto_grow {mode} leg overflow: {st}")
        out[name] = {"auto_grow": mode,
                     "value": round(float(sum(a.elapsed_time(b) for a, b in zip(starts, ends))) / K, 4),
                     "unit": "ms/frame", "host_wall_ms_per_frame": round(wall * 1e3 / K, 4),
                     "pairs_last_frame": [st["broad_pairs"], st["narrow_hits"]]}
        front.close()
        bvh.close()
    return out


def box_pass(bvhcd, torch, faces, dev, dfaces, stream, W, K, T):
    """The same frames given as primitive boxes (ARCSimSceneData input): each
    triangle's box swept over frames f and f + 1, computed on the device
    outside the timed region as a simulator would hand them over, read in
    place (FP32).  Broad phase only (a box scene has no triangles to test)."""
    F = dev.shape[0]
    fl = dfaces.long()
    boxes = torch.empty((F, T, 6), dtype=torch.float32, device="cuda")
    for f in range(F):
        a = dev[f][fl]                      # T x 3 x 3
        b = dev[min(f + 1, F - 1)][fl]
        boxes[f, :, :3] = torch.minimum(a.amin(dim=1), b.amin(dim=1))
        boxes[f, :, 3:] = torch.maximum(a.amax(dim=1), b.amax(dim=1))
    bvh = bvhcd.LBvh(T, 0, enable_restr=True)
    front = bvhcd.BvttFront(bvh, cull_adjacent=True, narrow_phase=False, auto_grow=False, **CAPS)
    flush = L2Flush(torch, FLUSH_DIRTY)

    def frame(f):
        b, fr = bvhcd.schedule(f)
        bvh.maintain_boxes(b, boxes[f], dfaces, stream=stream, faces_static=f > 0)
        front.maintain(fr, stream=stream)

    for f in range(W):
        frame(f)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    torch.cuda.synchronize()
    for i in range(K):
        flush()
        starts[i].record(stream)
        frame(W + i)
        ends[i].record(stream)
    torch.cuda.synchronize()
    ms = float(sum(a.elapsed_time(b) for a, b in zip(starts, ends))) / K
    st = front.stats()
    if st["overflow_any"]:
        raise RuntimeError(f"box leg overflow: {st}")
    front.close()
    bvh.close()
    del boxes
    torch.cuda.empty_cache()
    return {"workload": f"the bench frames as {T} swept triangle boxes (frames f and f + 1), FP32, device-resident",
            "value": round(ms, 4), "unit": "ms/frame", "narrow_phase": False,
            "front_sizes_last_frame": [st["int_front"], st["ext_front"]], "pairs_last_frame": st["broad_pairs"]}


def proximity_pass(bvhcd, torch, front, stream, thickness=1e-3, reps=5):
    """Vertex-face / edge-edge proximities (FP64) of the last frame's broad
    pairs through bvhcd_front_proximity into a device buffer: CUDA-event time
    of the call (a counting pass, a scan, the host reading the total, the
    writing pass), the record count and the pairs evaluated."""
    import ctypes
    L = bvhcd.lib()
    n = ctypes.c_int64()
    st = L.bvhcd_front_proximity(front.handle, None, float(thickness), None, 0, ctypes.byref(n), 1,
                                 ctypes.c_void_p(stream.cuda_stream))
    if st not in (0, 3):
        raise RuntimeError(f"proximity: status {st}")
    cap = max(int(n.value), 1)
    buf = torch.empty(cap * bvhcd.PROX_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    times = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        st = L.bvhcd_front_proximity(front.handle, None, float(thickness), ctypes.c_void_p(buf.data_ptr()), cap,
                                     ctypes.byref(n), 1, ctypes.c_void_p(stream.cuda_stream))
        b.record(stream)
        torch.cuda.synchronize()
        if st != 0:
            raise RuntimeError(f"proximity: status {st}")
        times.append(a.elapsed_time(b))
    pairs = front.stats()["broad_pairs"]
    return {"thickness": thickness, "pairs": int(pairs), "records": int(n.value),
            "ms_per_call": round(statistics.median(times), 4), "unit": "ms", "arithmetic": "f64",
            "pairs_per_s": round(pairs / (statistics.median(times) * 1e-3), 1)}


def fp16_pass(bvhcd, torch, faces, dev, dfaces, stream, W, K, T):
    """The same frames with FP16 node boxes (precision mode): device ms per
    frame, timed as `value`, and the last frame's front sizes."""
    bvh = bvhcd.LBvh(T, dev.shape[1], enable_restr=True, node_box_fp16=True)
    front = bvhcd.BvttFront(bvh, cull_adjacent=True, narrow_phase=True, auto_grow=False, **CAPS)
    flush = L2Flush(torch, FLUSH_DIRTY)
    for f in range(W):
        bvhcd.frame(bvh, front, f, 0, dev[f], dfaces, stream=stream, faces_static=f > 0)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    torch.cuda.synchronize()
    for i in range(K):
        flush()
        starts[i].record(stream)
        bvhcd.frame(bvh, front, W + i, 0, dev[W + i], dfaces, stream=stream, faces_static=True)
        ends[i].record(stream)
    torch.cuda.synchronize()
    st = front.stats()
    if st["overflow_any"]:
        raise RuntimeError(f"fp16 leg overflow: {st}")
    ms = float(sum(a.elapsed_time(b) for a, b in zip(starts, ends))) / K
    front.close()
    bvh.close()
    return {"value": round(ms, 4), "unit": "ms/frame", "node_records": "16 B (FP16, outward-rounded)",
            "front_sizes_last_frame": [st["int_front"], st["ext_front"]],
            "pairs_last_frame": [st["broad_pairs"], st["narrow_hits"]]}


# front / pair capacities of the two stacked-layer runs (the grazing layers hold
# about 63 front entries per triangle)
PREC_CAPS = {0.0: dict(int_front_capacity=60_000_000, ext_front_capacity=40_000_000, pair_capacity=8_000_000),
             0.8: dict(int_front_capacity=130_000_000, ext_front_capacity=90_000_000, pair_capacity=16_000_000)}


def precision_pass(bvhcd, torch, stream, args):
    """The precision configuration: four stacked 512x512 cloths (2,088,968
    triangles) 1e-3 apart with a seeded in-plane shear (scenes.
    stacked_layers_frames), 50 frames, FP16 outward-rounded node records and
    precision = 1 (FP32 narrow phase where it is certain, FP64 on the pairs it
    flags), the reference's schedule.  Device-resident frames, L2 flushed
    between timed frames; ms/frame and the share of broad pairs flagged for
    FP64.  A second, 3-frame run of the same layers with a grazing vertical
    jitter (up to 0.8 gaps: layers cut each other) gives intersecting pairs
    whose contact points the CPU check compares with FP64.  Returns the JSON
    block and the last frames' device results for that check."""
    import scenes
    out, keep = {}, {}
    F = args.precision_frames
    for name, zn, nf in (("as_stated", 0.0, F), ("grazing", 0.8, 3)):
        faces, frames = scenes.stacked_layers_frames(512, 4, nf, z_noise=zn)
        T, V = faces.shape[0], frames[0].shape[0]
        dev = torch.from_numpy(np.stack(frames)).cuda()
        dfaces = torch.from_numpy(faces).cuda()
        bvh = bvhcd.LBvh(T, V, enable_restr=True, node_box_fp16=True)
        # the grazing run's fronts (FP16 boxes rounded outward by up to a quarter of the layer gap) are
        # sized by growing (auto_grow = 1); its time is reported but it only serves the contact check
        front = bvhcd.BvttFront(bvh, cull_adjacent=True, narrow_phase=True, auto_grow=1 if zn else 0, precision=1,
                                **PREC_CAPS[zn])
        flush = L2Flush(torch, FLUSH_DIRTY)
        W = min(3, nf - 1)
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(nf)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(nf)]
        flagged = broad = 0
        for f in range(nf):
            flush()
            starts[f].record(stream)
            bvhcd.frame(bvh, front, f, 0, dev[f], dfaces, stream=stream, faces_static=f > 0)
            ends[f].record(stream)
            if f >= W:
                st = front.stats(stream)  # outside the events: counts for the flagged share
                flagged += st["flagged"]
                broad += st["broad_pairs"]
        torch.cuda.synchronize()
        st = front.stats()
        if st["overflow_any"]:
            raise RuntimeError(f"precision leg overflow: {st}")
        ms = float(sum(a.elapsed_time(b) for a, b in zip(starts[W:], ends[W:]))) / (nf - W)
        out[name] = {"workload": f"4 x 512x512 cloths, {T} triangles, 1e-3 apart, in-plane shear"
                                 + (", vertical jitter up to 0.8 gaps" if zn else "") + f", {nf} frames",
                     "value": round(ms, 4), "unit": "ms/frame", "frames_timed": nf - W,
                     "flagged_fraction": round(flagged / broad, 6) if broad else 0.0,
                     "auto_grow": 1 if zn else 0,
                     "pairs_last_frame": [st["broad_pairs"], st["narrow_hits"]]}
        hits = front.pairs(narrow=True)
        keep[name] = {"faces": faces, "pos": frames[-1], "broad": front.pairs(), "hits": hits,
                      "contacts": front.contacts(0)[0] if zn else None,
                      "contacts64": front.contacts64(0) if zn else None,
                      "dist_pairs": front.pairs() if zn else None, "dists": front.contacts(1)[0] if zn else None,
                      "dists64": front.contacts64(1) if zn else None}
        front.close()
        bvh.close()
        del dev, dfaces, flush
        torch.cuda.empty_cache()
    out["node_records"] = "16 B (FP16, outward-rounded)"
    out["narrow_phase"] = "fp32 17-axis SAT, fp64 on flagged pairs (precision = 1)"
    return out, keep


def precision_check(keep):
    """CPU side of the precision leg (the oracle as checker, on the host
    cores): the last frame's broad set against the sweep-and-prune set of
    overlapping FP32 boxes and its hits against the exact expansion-arithmetic
    predicate; on the grazing frame, contact points (segment midpoints) and
    distances against FP64, relative to each pair's extent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    res = {}
    for name, k in keep.items():
        faces, pos = k["faces"], k["pos"]
        exp = pyoracle.brute_pairs(faces, pos, 1)
        exact = pyoracle.narrow(exp, faces, pos, exact=True).astype(bool)
        r = {"broad_equal_bruteforce": bool(np.array_equal(pyoracle.canon_pairs(k["broad"]), exp)),
             "hits_equal_exact_predicate": bool(np.array_equal(pyoracle.canon_pairs(k["hits"]), exp[exact])),
             "broad_pairs": int(len(exp)), "hits": int(exact.sum())}
        if k["contacts"] is not None:
            def scale(pairs):
                a, b = pos[faces[pairs[:, 0]]], pos[faces[pairs[:, 1]]]
                pts = np.concatenate([a, b], axis=1)
                return (pts.max(axis=1) - pts.min(axis=1)).max(axis=1).astype(np.float64)
            h = k["hits"]
            _, con, _ = pyoracle.precision_pairs(h, faces, pos)
            bp = k["dist_pairs"]
            hit64, _, dist = pyoracle.precision_pairs(bp, faces, pos)
            sep = ~hit64

            def errs(c, d):
                both = ~np.isnan(con[:, 0]) & ~np.isnan(c[:, 0])
                e = np.abs(c[both, :3].astype(np.float64) - con[both, :3]).max(axis=1) / scale(h)[both]
                ed = np.abs(d[sep, 3].astype(np.float64) - dist[sep]) / scale(bp)[sep]
                return ({"max": float(e.max()) if e.size else 0.0, "mean": float(e.mean()) if e.size else 0.0,
                         "points": int(both.sum())},
                        {"max": float(ed.max()) if ed.size else 0.0, "mean": float(ed.mean()) if ed.size else 0.0,
                         "pairs": int(sep.sum())})
            # relative to each pair's extent; FP32 results carry the rounding of coordinates near 1
            r["contact_point_error"], r["distance_error"] = errs(k["contacts64"], k["dists64"])
            r["contact_point_error_fp32_results"], r["distance_error_fp32_results"] = errs(k["contacts"], k["dists"])
            r["zero_distance_equals_fp64_hit"] = bool(np.array_equal(k["dists64"][:, 3] == 0, hit64))
        res[name] = r
    return res


def learned_pass(torch, args):
    """The learned scheduler (weights trained on the GPU by learn.py, shipped
    in learned_scheduler.npz) against the reference's heuristic schedule on a
    held-out 708x708 cloth over the sphere (1,040,198 triangles, 200 frames,
    seed 90001), with the no-network refit cycle as the ablation; broad and
    narrow pair sets compared every 10 frames."""
    import learn
    r = learn.evaluate(torch, learn.WEIGHTS, 708, args.learned_frames, 90001, check_every=10, decide_every=3)
    import numpy as np  # noqa: F401
    w = np.load(learn.WEIGHTS)
    rep = json.loads(str(w["report"]))
    r["training"] = {k: rep[k] for k in ("rows", "sequences", "label_counts", "val_acc", "seconds")}
    return r


def cpu_baseline(faces, frames, args, budget_s=20.0):
    """Oracle pipeline (CPU restatement, OpenMP) on a bounded sample: the
    first frames of the same schedule, stopped after ~budget_s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    cores = os.cpu_count() or 1
    pyoracle.set_threads(cores)
    p = pyoracle.Pipeline(restructure=True, cull_adjacent=True, narrow=True)
    times = []
    t_all = time.perf_counter()
    for f in range(len(frames)):
        b, fr = pyoracle.schedule(f)
        t0 = time.perf_counter()
        p.frame(faces, frames[f], b, fr)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_all > budget_s and f >= 1:
            break
    n = len(times)
    return {"value": round(1e3 * sum(times) / n, 3), "unit": "ms/frame", "cores": cores, "kind": "port",
            "sample": f"frames 0..{n - 1} of the same workload and schedule (includes the frame-0 build)"}


def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    cores = os.cpu_count() or 1
    pyoracle.set_threads(cores)
    W, K = args.warmup, args.steps
    faces, frames = make_frames(W + K)
    p = pyoracle.Pipeline(restructure=True, cull_adjacent=True, narrow=True)
    times = []
    budget = args.reference_budget_s
    t_all = time.perf_counter()
    for f in range(W + K):
        b, fr = pyoracle.schedule(f)
        t0 = time.perf_counter()
        p.frame(faces, frames[f], b, fr)
        dt = time.perf_counter() - t0
        if f >= W:
            times.append(dt)
        if time.perf_counter() - t_all > budget and len(times) >= 1:
            break
    n = len(times)
    value = 1e3 * sum(times) / n
    return {"impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "ms/frame",
            "n_gpus": world, "steps": n, "warmup": W, "ms_per_step": round(value, 3),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": WORKLOAD if CLOTH == 512 else f"cloth{CLOTH}_over_icosphere45", "triangles": int(faces.shape[0]), "vertices": int(frames[0].shape[0])},
            "cpu_baseline": {"value": round(value, 3), "unit": "ms/frame", "cores": cores, "kind": "port",
                             "sample": f"frames {W}..{W + n - 1} timed after {W} warm-up frames"
                                       f"{' (stopped at the time budget)' if n < K else ''}"},
            "e2e": {"value": round(value, 3), "unit": "ms/frame", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--l2-flush", choices=["clean", "dirty"], default="clean",
                    help="between timed frames: 256 MB write then 256 MB read (clean), or the write alone")
    ap.add_argument("--only-value", action="store_true",
                    help="time the device-resident frames only (no e2e / roofline replay); for profiling")
    ap.add_argument("--reference-budget-s", type=float, default=150.0)
    ap.add_argument("--no-batched", action="store_true", help="skip the 256-scene batched leg")
    ap.add_argument("--cloth", type=int, default=512,
                    help="cloth side in vertices; 512 is the headline workload, smaller sides are for profiling")
    ap.add_argument("--batched-frames", type=int, default=30)
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-scheduler leg")
    ap.add_argument("--no-precision", action="store_true", help="skip the stacked-layer precision leg")
    ap.add_argument("--precision-frames", type=int, default=50)
    ap.add_argument("--learned-frames", type=int, default=200)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    global CLOTH, FLUSH_DIRTY
    CLOTH = args.cloth
    FLUSH_DIRTY = args.l2_flush == "dirty"
    out = run_reference(args) if args.impl == "reference" else run_ours(args)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
