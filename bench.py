"""Benchmark of the EVX3 encoder pixel pipeline on B200.

Workload (the plain one-stream configuration): a seeded 1920x1080 RGB24
sequence of 120 frames (sinusoid background, global pan with per-frame
velocity in [-24, 24] px at quarter-pel, moving textured rectangles, noise
sigma 3, scene cut at frame 60 where insert_intra() starts a new GOP),
quality 8, deblocking and SAO on, encoded with the reference encoder's own GOP
structure (I, then hierarchical P / reference-B / B groups of 4).

A step is one frame of engine_encode_frame minus serialization in encode
order: RGB->YUV, the macroblock wavefront (mode decision, transform,
quantisation, trellis, reconstruction), deblocking, SAO.  `value` times the
steps on the device with the RGB frames already resident in HBM and L2
flushed between steps; `e2e` times the same steps through the C ABI with
pinned host RGB in and the serializer's tables (block, previous block, SAO
tables and level planes) out, copies inside the timed region.

Multi-GPU (torchrun): every rank encodes its own stream (own seed), no
collective on the data path (weak scaling); time is the max over ranks.
`--impl reference` times the unmodified reference encoder (oracle/_ref, built
from the reference's sources) through its public API on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "1080p-eq frames/s & p99 frame latency, batched vs plain GPU, bit-exact output"
UNIT = "1080p-eq frames/s"
W, H, FRAMES, QUALITY, VMAX, CUT = 1920, 1080, 120, 8, 24.0, 60
EQ = (W * H) / (1920 * 1080)
HBM_PEAK_FALLBACK = 6650.0
# dram__bytes_read.sum + dram__bytes_write.sum of one k_mb_cluster launch
# (a 1080p B frame of this workload), profiles/mb_cluster_1080p.md
MB_TRAFFIC_BYTES = 25_386_496 + 257_792


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return HBM_PEAK_FALLBACK, "fallback"


def max_over_ranks(ms: float, world: int, device: str = "cuda") -> float:
    """The job's time: the slowest rank's (every rank takes part, in the same order)."""
    if world == 1:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def job_value(world: int, steps: int, ms: float) -> float:
    """Whole-job 1080p-eq frames/s: every rank encodes its own stream of `steps` frames."""
    return world * steps * EQ / (ms / 1e3)


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def plan(seed_offset: int):
    from chicago_b200.gop import plan as gop_plan
    return gop_plan(FRAMES, quality=QUALITY, intra_at=(CUT,))


def rank_seed(rank: int) -> int:
    """Every rank encodes its own stream: the same generator, its own seed."""
    return 1000 + rank


def frames_for(rank: int):
    from chicago_b200.synth import generate
    return generate(W, H, FRAMES, seed=rank_seed(rank), vmax=VMAX, n_rects=4, cut_at=CUT)


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index: int):
        self.p = None
        self.path = f"/tmp/evxg_clocks_{os.getpid()}.csv"
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(index), "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_bytes(ftype: int, aw: int, ah: int) -> int:
    """Compulsory HBM bytes of one macroblock-wavefront launch: the source plane
    set read once, every reference slot read once (the intra block-copy search
    reads the destination slot too), reconstruction and levels written once,
    block table written (28 B per MB)."""
    planeset = (aw * ah + 2 * (aw // 2) * (ah // 2)) * 2
    refs = {0: 1, 1: 2, 2: 3}[ftype]
    return planeset * (1 + refs + 2) + (aw // 16) * (ah // 16) * 28


def run_gpu(args):
    import torch
    import chicago_b200 as cb
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=600))
    sched = plan(rank)
    K = min(args.steps, len(sched) - args.warmup)
    frames = frames_for(rank)
    dev_frames = torch.from_numpy(frames).cuda()                       # 746 MB resident in HBM
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")   # > 126 MB L2
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    st = cb.Stream(W, H)
    st.profile(True)
    from chicago_b200.gop import unpack_frame
    # warm-up steps, then K timed steps; state (DPB, tables) carries across steps
    order = sched[:args.warmup + K]
    for ti, f18 in order[:args.warmup]:
        st.encode_frame(dev_frames[ti].data_ptr(), f18, on_device=True, cuda_stream=sp)
    st.sync(sp)
    clocks = Clocks(local)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    step_ms, mb_ms, mb_bytes = [], [], 0
    kernel_tot = {k: 0.0 for k in cb.Stream.KERNELS}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for ti, f18 in order[args.warmup:]:
        flush.zero_()
        ev0.record(stream)
        st.encode_frame(dev_frames[ti].data_ptr(), f18, on_device=True, cuda_stream=sp)
        ev1.record(stream)
        ev1.synchronize()
        step_ms.append(ev0.elapsed_time(ev1))
        km = st.kernel_ms()
        for k, v in km.items():
            kernel_tot[k] += v
        mb_ms.append(km["mb_wavefront"])
        mb_bytes += algorithmic_bytes(unpack_frame(f18)["type"], st.aw, st.ah)
    st.sync(sp)
    torch.cuda.synchronize()
    clk = clocks.stop()
    total_ms = max_over_ranks(sum(step_ms), world)
    value = job_value(world, K, total_ms)

    # end to end through the C ABI: pinned host RGB in, serializer tables out
    nblk = st.mbw * st.mbh
    host_rgb = torch.from_numpy(frames).pin_memory()
    out_bt = torch.empty(nblk * 28, dtype=torch.uint8).pin_memory()
    out_prev = torch.empty(nblk * 28, dtype=torch.uint8).pin_memory()
    out_sao = torch.empty(nblk * 16, dtype=torch.uint8).pin_memory()
    out_lev = torch.empty(st.plane_elems, dtype=torch.int16).pin_memory()
    st2 = cb.Stream(W, H)
    L = cb.lib()
    import ctypes as C
    e2e_ms = []
    for i, (ti, f18) in enumerate(order):
        ev0.record(stream)
        cb._check(L.evxg_encode_frame(st2.h, C.c_void_p(host_rgb[ti].data_ptr()), 0, f18, C.c_void_p(sp)))
        cb._check(L.evxg_fetch_tables(st2.h, C.c_void_p(out_bt.data_ptr()), C.c_void_p(out_prev.data_ptr()),
                                      C.c_void_p(out_sao.data_ptr()), C.c_void_p(out_lev.data_ptr()), 0, C.c_void_p(sp)))
        ev1.record(stream)
        ev1.synchronize()
        if i >= args.warmup:
            e2e_ms.append(ev0.elapsed_time(ev1))
    e2e_total = max_over_ranks(sum(e2e_ms), world)
    e2e_value = job_value(world, K, e2e_total)
    h2d = W * H * 3
    d2h = nblk * 28 * 2 + nblk * 16 + st.plane_elems * 2

    batched = run_batched(args, stream) if args.batch > 1 and world == 1 else None
    served = run_served(args) if args.serve_streams > 0 and world == 1 else None
    served_light = (run_served(args, n=8, per=12, sizes_from=[(640, 360), (1280, 720)], seed=11)
                    if args.serve_streams > 0 and world == 1 else None)

    peak, peak_kind = peaks()
    achieved = mb_bytes / (sum(mb_ms) / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": round(total_ms / K, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int16", "data": "synthetic (seeded generator)",
        "config": {"workload": "plain GPU path, one stream per GPU: 1920x1080 RGB24, 120 frames, pan +-24 px, "
                               "scene cut at 60, quality 8, reference GOP (I + hierarchical P/B of 4), deblock+SAO",
                   "frames": FRAMES, "quality": QUALITY, "l2": "flushed (256 MB write) between timed steps",
                   "parallelism": f"{world} independent streams, no collective"},
        "p50_frame_ms": round(float(np.percentile(step_ms, 50)), 3),
        "p99_frame_ms": round(float(np.percentile(step_ms, 99)), 3),
        "kernel_ms_per_step": {k: round(v / K, 4) for k, v in kernel_tot.items()},
        "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "roofline": {"kernel": "k_mb_cluster" if st.mb_form == cb.MB_FORM_CLUSTER else "k_mb_wavefront",
                     "bound": "hbm", "achieved": round(achieved, 3), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 6),
                     "traffic": MB_TRAFFIC_BYTES if st.mb_form == cb.MB_FORM_CLUSTER else None,
                     "peak_source": f"{peak_kind} hbm_gbs",
                     "note": "dependency-latency bound: macroblock wavefront whose critical path is "
                             "cols + 3*(rows-1) MB steps (321 at 1080p), each one MB's dependent chain"},
        "gpu_launches": st.launch_count() * K,
        "batched": batched,
        "served": served,
        "served_light": served_light,
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


# The batched configuration: 16 streams -- 4 x 1920x1080, 6 x 1280x720,
# 6 x 640x360 -- each with its own seed, at its own GOP position (stream k
# starts k % 4 ticks late and cuts to a new GOP at its own frame), quality 8.
BATCH_MIX = [(1920, 1080)] * 4 + [(1280, 720)] * 6 + [(640, 360)] * 6


def run_batched(args, stream):
    """All streams advance through batched ticks (one launch per stage for all
    streams, one persistent macroblock pass over one (stream, row) queue, the
    tick replayed as a CUDA graph), shape chosen by the library's autotuner.
    Timed end to end on the device: each tick copies its RGB frames in from
    pinned host buffers and its tables out, ticks pipelined on two buffer
    parities while the host fills the next one."""
    import torch
    import chicago_b200 as cb
    from chicago_b200.gop import plan as gop_plan, unpack_frame
    from chicago_b200.synth import generate
    mix = BATCH_MIX[:args.batch] if args.batch < len(BATCH_MIX) else BATCH_MIX
    warm, K = args.warmup, args.batch_ticks
    nfr = warm + K + 4
    seqs = []
    for k, (w, h) in enumerate(mix):
        frames = generate(w, h, nfr, seed=2000 + k, vmax=max(6.0, 24.0 * w / 1920), n_rects=4)
        seqs.append((frames, gop_plan(nfr, quality=QUALITY, intra_at=(5 + (3 * k) % 7,))))
    streams = [cb.Stream(w, h) for w, h in mix]
    b = cb.Batch(streams)
    sp = stream.cuda_stream
    tuned_ms = b.autotune(sp)
    form, grid, policy = b.shape
    pos = [0] * len(mix)
    ev = []
    eq = []
    for t in range(warm + K):
        par = t & 1
        b.wait(par)
        f18s, teq = [], 0.0
        for k, (w, h) in enumerate(mix):
            frames, sched = seqs[k]
            if t < k % 4 or pos[k] >= len(sched):
                f18s.append(None)
                continue
            ti, f18 = sched[pos[k]]
            pos[k] += 1
            b.input(k, par)[:] = frames[ti]
            f18s.append(f18)
            teq += w * h / (1920 * 1080)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.encode(f18s, par, sp)
        e1.record(stream)
        if t >= warm:
            ev.append((e0, e1))
            eq.append(teq)
    for par in (0, 1):
        b.wait(par)
    torch.cuda.synchronize()
    tick_ms = [a.elapsed_time(c) for a, c in ev]
    span_ms = ev[0][0].elapsed_time(ev[-1][1])
    h2d = sum(w * h * 3 for w, h in mix)
    d2h = sum(s.nblk * 72 + s.plane_elems * 2 for s in streams)
    sizes = {}
    for w, h in mix:
        sizes[f"{w}x{h}"] = sizes.get(f"{w}x{h}", 0) + 1
    res = {"streams": len(mix), "sizes": " + ".join(f"{n}x{k}" for k, n in sizes.items()),
           "value": round(sum(eq) / (span_ms / 1e3), 3), "unit": UNIT, "ticks": K,
           "ms_per_tick": round(span_ms / K, 3),
           "p50_frame_ms": round(float(np.percentile(tick_ms, 50)), 3),
           "p99_frame_ms": round(float(np.percentile(tick_ms, 99)), 3),
           "gpu_launches_per_tick": b.launch_count(),
           "shape": {"form": "cluster" if form == cb.MB_FORM_CLUSTER else "single", "grid": grid,
                     "queue_order": policy, "autotune_ms": round(tuned_ms, 3)},
           "e2e": {"h2d_bytes_per_tick": h2d, "d2h_bytes_per_tick": d2h},
           "note": "batched ticks through the C ABI, pinned host RGB in and tables out inside the timed span, "
                   "each stream's own seed and GOP position; a frame's latency is its tick's device time"}
    b.close()
    for s_ in streams:
        s_.close()
    return res


# The serving configuration: 64 streams at 60 fps, sizes drawn uniformly from
# 640x360 / 1280x720 / 1920x1080 / 3840x2160, arrivals every 1/60 s with
# +-2 ms jitter from a random phase, quality 8.
SERVE_SIZES = [(640, 360), (1280, 720), (1920, 1080), (3840, 2160)]


def run_served(args, n=None, per=None, sizes_from=None, seed=7):
    """The request loop (evxg_server_*): all streams admitted by the device
    memory budget, frames submitted at their arrival times by this thread, the
    server's worker batching whatever is ready.  A frame's latency is its done
    time (results seen by the host) minus its arrival time, so it includes the
    reference GOP's reorder wait (a B frame waits for its anchor) and queueing;
    each stream sends `serve_frames` frames and then closes (flushing)."""
    import chicago_b200 as cb
    from chicago_b200.synth import generate
    rng = np.random.default_rng(seed)
    n = args.serve_streams if n is None else n
    per = args.serve_frames if per is None else per
    choices = SERVE_SIZES if sizes_from is None else sizes_from
    sizes = [choices[i] for i in rng.integers(0, len(choices), n)]
    pool = {sz: generate(sz[0], sz[1], per + 3, seed=3000 + k, vmax=max(4.0, 24.0 * sz[0] / 1920))
            for k, sz in enumerate(SERVE_SIZES) if sz in sizes}
    srv = cb.Server(hbm_budget_bytes=96 << 30, max_streams=n, keep_tables=False)
    ids = [srv.open(w, h, QUALITY) for w, h in sizes]
    srv.drain()   # the batch over every admitted stream exists before the first arrival
    phase = rng.uniform(0, 1 / 60, n)
    events = sorted((phase[k] + t / 60 + rng.uniform(-0.002, 0.002), k, t) for k in range(n) for t in range(per))
    t0 = cb.Server.now_ns()
    sent = [0] * n
    for at, k, t in events:
        due = t0 + int(max(at, 0.0) * 1e9)
        while cb.Server.now_ns() < due:
            time.sleep(min(0.0005, (due - cb.Server.now_ns()) / 1e9))
        off = k % 3   # streams of a size class start at different frames of its pool
        srv.submit(ids[k], pool[sizes[k]][off + t], arrival_ns=cb.Server.now_ns())
        sent[k] += 1
        if sent[k] == per:
            srv.close_stream(ids[k])
    srv.drain()
    lat, work, eq, first, last = [], [], 0.0, None, 0
    for k, sid in enumerate(ids):
        w, h = sizes[k]
        for r in srv.results[sid]:
            a, rd, _, d = r["times"]
            lat.append((d - a) / 1e6)
            work.append((d - rd) / 1e6)
            eq += w * h / (1920 * 1080)
            first = a if first is None else min(first, a)
            last = max(last, d)
    st = srv.stats()
    srv.close()
    offered = sum(w * h for w, h in sizes) / (1920 * 1080) * 60
    counts = {f"{w}x{h}": sizes.count((w, h)) for w, h in SERVE_SIZES if (w, h) in sizes}
    return {"streams": n, "sizes": counts, "frames": len(lat), "frames_per_stream": per,
            "value": round(eq / ((last - first) / 1e9), 3), "unit": UNIT,
            "offered_1080p_eq_fps": round(offered, 1),
            "p50_frame_ms": round(float(np.percentile(lat, 50)), 3),
            "p99_frame_ms": round(float(np.percentile(lat, 99)), 3),
            "p999_frame_ms": round(float(np.percentile(lat, 99.9)), 3),
            "ready_to_done_ms": {q: round(float(np.percentile(work, v)), 3) for q, v in (("p50", 50), ("p99", 99), ("p999", 99.9))},
            "ticks": st["ticks"], "batch_rebuilds": st["rebuilds"],
            "note": "latency = results seen by the host minus arrival: includes the reference GOP's reorder wait "
                    "(a B frame waits for its anchor, 3 frames later) and any queueing; ready_to_done starts when "
                    "the frame's encode order is known"}


def cpu_baseline(n_frames: int = 8):
    """The unmodified reference encoder (built here from its sources) with its
    WPP threads on all host cores, on the first n_frames of the same workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from chicago_b200.synth import generate
    from oracle_py import Ref
    frames = generate(W, H, n_frames, seed=1000, vmax=VMAX)
    ref = Ref()
    t0 = time.perf_counter()
    ref.encode_stream(frames, quality=QUALITY)
    dt = time.perf_counter() - t0
    return {"value": round(n_frames * EQ / dt, 4), "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
            "sample": f"first {n_frames} frames of the workload through create_encoder/encode/flush (WPP threads)"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle_py import REF_SO, Ref
    if not os.path.exists(REF_SO):
        print(json.dumps({"impl": "reference", "unavailable": "reference library oracle/_ref/libevxref.so not built"}))
        return
    import ctypes as C
    ref = Ref()
    K = min(args.steps, FRAMES - args.warmup)
    frames = frames_for(0)[:args.warmup + K]
    L = ref.lib
    cap = W * H * 3 * 8
    h = L.evxref_enc_create(cap)
    buf = np.zeros(cap, np.uint8)
    n = C.c_uint32(0)
    L.evxref_enc_set_quality(h, QUALITY)
    for t in range(args.warmup):
        if t == CUT:
            L.evxref_enc_insert_intra(h)
        L.evxref_enc_encode(h, frames[t].ctypes.data_as(C.c_void_p), W, H, buf.ctypes.data_as(C.c_void_p), cap, C.byref(n))
    t0 = time.perf_counter()
    for t in range(args.warmup, args.warmup + K):
        if t == CUT:
            L.evxref_enc_insert_intra(h)
        L.evxref_enc_encode(h, frames[t].ctypes.data_as(C.c_void_p), W, H, buf.ctypes.data_as(C.c_void_p), cap, C.byref(n))
    L.evxref_enc_flush(h, buf.ctypes.data_as(C.c_void_p), cap, C.byref(n))
    dt = time.perf_counter() - t0
    L.evxref_enc_destroy(h)
    value = K * EQ / dt
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world,
            "steps": K, "warmup": args.warmup, "ms_per_step": round(dt * 1e3 / K, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int16", "data": "synthetic (seeded generator)",
            "config": {"workload": "same sequence as the GPU arm, stream 0", "frames": FRAMES, "quality": QUALITY},
            "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                             "sample": f"{K} frames after {args.warmup} warm-up frames, WPP threads"},
            "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=117)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch", type=int, default=16, help="streams of the batched measurement (1 = skip)")
    ap.add_argument("--batch-ticks", type=int, default=12, help="timed ticks of the batched measurement")
    ap.add_argument("--serve-streams", type=int, default=64, help="streams of the serving measurement (0 = skip)")
    ap.add_argument("--serve-frames", type=int, default=4, help="frames each served stream sends")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
