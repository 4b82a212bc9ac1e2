"""Benchmark of the EVX3 encoder pixel pipeline on B200.

Workload (the plain one-stream configuration): a seeded 1920x1080 RGB24
sequence of 120 frames (sinusoid background, global pan with per-frame
velocity in [-24, 24] px at quarter-pel, moving textured rectangles, noise
sigma 3, scene cut at frame 60), quality 8, deblocking and SAO on, encoded as
an I/P GOP of 60 (insert_intra() at the cut) by the reference's I/P build with
three references (EVX_ENABLE_B_FRAMES 0, EVX_REFERENCE_FRAME_COUNT 4): every P
frame searches the last three reconstructed frames.  An I/P GOP with exactly
two references is not expressible in the reference (a reference count of 3
breaks its bitstream), so three stand in for two.

A step is one frame of engine_encode_frame minus serialization in encode
order: RGB->YUV, the macroblock wavefront (mode decision over three
references, transform, quantisation, trellis, reconstruction), deblocking,
SAO.  `value` times the steps on the device with the RGB frames already
resident in HBM and L2 flushed between steps; `e2e` times the same steps
through the C ABI with pinned host RGB in and the serializer's tables (block,
previous block, SAO tables and level planes) out, copies inside the timed
region.  Extra legs: quality 4 and 16, the reference's default GOP
(hierarchical P/B), the batched 16-stream mix and the served request loop.

Parity: the cpu_baseline leg encodes the same frames with the reference's own
I/P build and checks that the GPU arm's tables of every warm-up and timed
frame, serialized by that build's entropy coder, give its .evx bytes exactly
(`parity` in the line).

Multi-GPU (torchrun): every rank encodes its own stream (own seed), no
collective on the data path (weak scaling); time is the max over ranks.
`--impl reference` times the reference encoder of the same build (oracle/_ref,
built from the reference's sources) through its public API on the host cores.
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
CFG = "ip3"          # reference build: I/P GOP, three references
GOP_DESC = "I/P GOP of 60 (insert_intra at the cut), 3 references standing in for 2"
EQ = (W * H) / (1920 * 1080)
HBM_PEAK_FALLBACK = 6650.0
# dram__bytes_read.sum + dram__bytes_write.sum of one k_mb_cluster launch on a
# 1920x1080 P frame with three references of this workload (ncu capture)
MB_TRAFFIC_BYTES = 31_906_304 + 365_568


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


def plan(quality: int = QUALITY, cfg: str = CFG):
    from chicago_b200.gop import plan as gop_plan
    return gop_plan(FRAMES, quality=quality, intra_at=(CUT,), cfg=cfg)


def rank_seed(rank: int) -> int:
    """Every rank encodes its own stream: the same generator, its own seed."""
    return 1000 + rank


def frames_for(rank: int, n: int = FRAMES):
    from chicago_b200.synth import generate
    return generate(W, H, n, seed=rank_seed(rank), vmax=VMAX, n_rects=4, cut_at=CUT)


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


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


def algorithmic_bytes(ftype: int, aw: int, ah: int, nref: int) -> int:
    """Compulsory HBM bytes of one macroblock-wavefront launch: the source plane
    set read once, every reference slot read once (the intra block-copy search
    reads the destination slot too), reconstruction and levels written once,
    block table written (28 B per MB)."""
    planeset = (aw * ah + 2 * (aw // 2) * (ah // 2)) * 2
    refs = {0: 1, 1: 1 + nref, 2: 3}[ftype]
    return planeset * (1 + refs + 2) + (aw // 16) * (ah // 16) * 28


def device_steps(stream, frames_dev, sched, warmup, cfg, flush, profile=False):
    """Encode sched's frames on a fresh stream from device-resident RGB; time
    the steps after the warm-up ones with CUDA events on the launching stream,
    L2 flushed before each.  Returns (stream, step_ms, per-kernel ms list)."""
    import torch
    import chicago_b200 as cb
    sp = stream.cuda_stream
    st = cb.Stream(W, H, cfg)
    if profile:
        st.profile(True)
    for ti, f18 in sched[:warmup]:
        st.encode_frame(frames_dev[ti].data_ptr(), f18, on_device=True, cuda_stream=sp)
    st.sync(sp)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    step_ms, kms = [], []
    for ti, f18 in sched[warmup:]:
        flush.zero_()
        ev0.record(stream)
        st.encode_frame(frames_dev[ti].data_ptr(), f18, on_device=True, cuda_stream=sp)
        ev1.record(stream)
        ev1.synchronize()
        step_ms.append(ev0.elapsed_time(ev1))
        if profile:
            kms.append(st.kernel_ms())
    st.sync(sp)
    return st, step_ms, kms


def run_gpu(args):
    import torch
    import chicago_b200 as cb
    from chicago_b200.gop import unpack_frame
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=600))
    sched = plan()
    K = min(args.steps, len(sched) - args.warmup)
    order = sched[:args.warmup + K]
    frames = frames_for(rank)
    dev_frames = torch.from_numpy(frames).cuda()                       # 746 MB resident in HBM
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")   # > 126 MB L2
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    nref = cb.CONFIGS[CFG][1] - 1

    # headline: device-resident steps at quality 8, per-kernel times
    clocks = Clocks(local)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    st, step_ms, kms = device_steps(stream, dev_frames, order, args.warmup, CFG, flush, profile=True)
    torch.cuda.synchronize()
    clk = clocks.stop()
    total_ms = max_over_ranks(sum(step_ms), world)
    value = job_value(world, K, total_ms)
    kernel_tot = {k: sum(m[k] for m in kms) for k in cb.Stream.KERNELS}
    mb_ms = [m["mb_wavefront"] for m in kms]
    mb_bytes = sum(algorithmic_bytes(unpack_frame(f18)["type"], st.aw, st.ah, nref) for _, f18 in order[args.warmup:])
    launches = st.launch_count() * K
    form = st.mb_form
    st.close()

    # quality 4 and 16, and the reference's default GOP, on fresh streams
    legs = {}
    for q in (4, 16):
        s_, ms, _ = device_steps(stream, dev_frames, plan(q)[:args.warmup + K], args.warmup, CFG, flush)
        s_.close()
        t = max_over_ranks(sum(ms), world)
        legs[f"q{q}"] = {"value": round(job_value(world, K, t), 3), "ms_per_step": round(t / K, 3),
                         "p99_frame_ms": round(float(np.percentile(ms, 99)), 3)}
    s_, ms, _ = device_steps(stream, dev_frames, plan(QUALITY, "default")[:args.warmup + K], args.warmup, "default", flush)
    s_.close()
    t = max_over_ranks(sum(ms), world)
    default_gop = {"value": round(job_value(world, K, t), 3), "ms_per_step": round(t / K, 3),
                   "p99_frame_ms": round(float(np.percentile(ms, 99)), 3),
                   "workload": "same frames, the reference's default build: I + hierarchical P/B groups of 4"}

    # end to end through the C ABI: pinned host RGB in, the serializer's tables
    # out, and every frame's slice bytes from the library's host entropy coder
    # (evxg_serialize_slice, on a pool of host threads while the GPU encodes
    # the next frames)
    e2e_s, slices, e2e_threads = run_e2e(args, frames, order, stream)
    e2e_total = max_over_ranks(e2e_s * 1e3, world)
    e2e_value = job_value(world, K, e2e_total)
    nblk = (W // 16) * ((H + 15) // 16)
    plane_elems = (W * ((H + 15) & ~15)) * 3 // 2
    h2d = W * H * 3
    d2h = nblk * 28 * 2 + nblk * 16 + plane_elems * 2

    decode, decoded = run_decode(args, slices, stream) if world == 1 else (None, None)
    batched = run_batched(args, stream) if args.batch > 1 and world == 1 else None
    served = run_served(args) if args.serve_streams > 0 and world == 1 else None
    served_light = (run_served(args, n=8, per=args.serve_frames, sizes_from=[(640, 360), (1280, 720)], seed=11)
                    if args.serve_streams > 0 and world == 1 else None)

    peak, peak_kind = peaks()
    achieved = mb_bytes / (sum(mb_ms) / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": round(total_ms / K, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int16", "data": "synthetic (seeded generator)",
        "config": {"workload": "plain GPU path, one stream per GPU: 1920x1080 RGB24, 120 frames, pan +-24 px, "
                               f"scene cut at 60, quality 8, {GOP_DESC}, quarter-pel search over +-32 px, "
                               "deblock+SAO",
                   "reference_build": "EVX_ENABLE_B_FRAMES 0, EVX_REFERENCE_FRAME_COUNT 4",
                   "frames": FRAMES, "quality": QUALITY, "l2": "flushed (256 MB write) between timed steps",
                   "parallelism": f"{world} independent streams, no collective"},
        "p50_frame_ms": round(float(np.percentile(step_ms, 50)), 3),
        "p99_frame_ms": round(float(np.percentile(step_ms, 99)), 3),
        "kernel_ms_per_step": {k: round(v / K, 4) for k, v in kernel_tot.items()},
        "e2e": {"value": round(e2e_value, 3), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": round(e2e_total / K, 3),
                "note": "wall clock over the timed frames: pinned host RGB in, tables out, and each frame's .evx "
                        f"slice from the library's host entropy coder on {e2e_threads} host threads -- the same work "
                        "the reference arm's encode() does"},
        "roofline": {"kernel": "k_mb_cluster" if form == cb.MB_FORM_CLUSTER else "k_mb_wavefront",
                     "bound": "hbm", "achieved": round(achieved, 3), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 6),
                     "traffic": MB_TRAFFIC_BYTES if form == cb.MB_FORM_CLUSTER else None,
                     "peak_source": f"{peak_kind} hbm_gbs",
                     "note": "dependency-latency bound: macroblock wavefront whose critical path is "
                             "cols + 3*(rows-1) MB steps (321 at 1080p), each one MB's dependent chain"},
        "gpu_launches": launches,
        "quality_legs": legs,
        "default_gop": default_gop,
        "decode": decode,
        "batched": batched,
        "served": served,
        "served_light": served_light,
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"], line["parity"] = cpu_baseline(order, slices, frames, decoded)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def run_e2e(args, frames, order, stream):
    """Encode the frames of `order` through the C ABI from pinned host RGB
    (evxg_encode_frame_pipelined: uploads and table downloads on the stream's
    copy stream, off the frames' critical path), each frame's tables into one
    of a ring of pinned host buffers, handed to a pool of host threads that
    wait for the frame (evxg_stream_output_wait) and run the library's entropy
    coder (ctypes releases the interpreter lock during the calls); a buffer is
    reused once its frame's slice is done.  Returns the wall time of the frames after
    the warm-up ones (their slices included), every frame's (frame18, slice)
    and the thread count."""
    import ctypes as C
    import concurrent.futures as cf
    import torch
    import chicago_b200 as cb
    L = cb.lib()
    sp = stream.cuda_stream
    st = cb.Stream(W, H, CFG)
    nblk, ne = st.nblk, st.plane_elems
    host_rgb = torch.from_numpy(frames).pin_memory()
    ring = [tuple(torch.empty(n, dtype=dt).pin_memory() for n, dt in
                  ((nblk * 28, torch.uint8), (nblk * 28, torch.uint8), (nblk * 16, torch.uint8), (ne, torch.int16)))
            for _ in range(12)]
    threads = max(1, min(12, (os.cpu_count() or 2) - 1))
    cfg = cb.config(CFG)
    cap = st.aw * st.ah * 4

    def serialize(f18, bufs, ticket):
        cb._check(L.evxg_stream_output_wait(st.h, ticket))   # the frame's tables are in bufs
        out = np.empty(cap, np.uint8)
        n = C.c_uint64(0)
        cb._check(L.evxg_serialize_slice(C.byref(cfg), st.aw, st.ah, f18, *[C.c_void_p(b.data_ptr()) for b in bufs],
                                         out.ctypes.data_as(C.c_void_p), cap, C.byref(n)))
        return out[:n.value].tobytes()

    slices, pending = [], {}
    t0 = None
    with cf.ThreadPoolExecutor(threads) as pool:
        for i, (ti, f18) in enumerate(order):
            if i == args.warmup:   # the timed frames start with every warm-up slice done
                for j in list(pending):
                    slices[j] = (slices[j][0], pending.pop(j).result())
                torch.cuda.synchronize()
                t0 = time.perf_counter()
            k = i % len(ring)
            for j in [j for j in pending if j % len(ring) == k]:   # this buffer's previous frame must be coded
                slices[j] = (slices[j][0], pending.pop(j).result())
            bufs = ring[k]
            ticket = C.c_uint64()
            cb._check(L.evxg_encode_frame_pipelined(st.h, C.c_void_p(host_rgb[ti].data_ptr()), f18,
                                                    *[C.c_void_p(b.data_ptr()) for b in bufs], C.c_void_p(sp),
                                                    C.byref(ticket)))
            slices.append((f18, None))
            pending[i] = pool.submit(serialize, f18, bufs, ticket.value)
        for j in list(pending):
            slices[j] = (slices[j][0], pending.pop(j).result())
        t1 = time.perf_counter()
    st.close()
    return t1 - t0, slices, threads


def decode_bytes_per_frame(aw: int, ah: int) -> int:
    """Algorithmic HBM bytes of one decoded frame: the macroblock reconstruction
    reads a reference plane set and the level planes and writes the
    destination; deblocking reads and writes it; the SAO pass copies it, then
    reads the copy and reads and writes the slot; the conversion reads it and
    writes RGB24 (one plane set = aw*ah*3/2 int16 samples)."""
    ps = aw * ah * 3
    return 3 * ps + 2 * ps + 2 * ps + 3 * ps + ps + aw * ah * 3


def run_decode(args, slices, stream):
    """The decoder on the GPU arm's own stream (its e2e leg's records: I/P,
    three references, 1080p), frames 0..warmup-1 decoded untimed first (the
    DPB needs them):
      device -- the tables entropy-decoded beforehand and resident in HBM, each
                frame's evxg_decode_frame (macroblock reconstruction,
                deblocking, SAO, RGB24 into HBM) timed with CUDA events, L2
                flushed between frames;
      e2e    -- record bytes in host memory to RGB24 in pinned host memory
                through evxg_decoder_decode_record (host entropy decoding,
                copies, the same kernels), wall clock.
    Returns the leg's JSON object and the e2e leg's frames (decode order)."""
    import ctypes as C
    import torch
    import chicago_b200 as cb
    L = cb.lib()
    sp = C.c_void_p(stream.cuda_stream)
    aw, ah = W, (H + 15) & ~15
    nblk, ne = (aw // 16) * (ah // 16), aw * ah * 3 // 2
    blocks, prev = np.zeros(nblk * 28, np.uint8), np.zeros(nblk * 28, np.uint8)
    sao, lev = np.zeros(nblk * 16, np.uint8), np.zeros(ne, np.int16)
    tabs, ent_s = [], 0.0
    for f18, sl in slices:   # I/P build: every frame updates the temporal table
        t0 = time.perf_counter()
        cb.unserialize_slice(CFG, aw, ah, f18, sl, blocks, prev, sao, lev)
        ent_s += time.perf_counter() - t0
        prev[:] = blocks
        tabs.append(tuple(torch.from_numpy(a.copy()).cuda() for a in (blocks, sao, lev)))
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    rgb = torch.empty(H * W * 3, dtype=torch.uint8, device="cuda")
    dec = cb.Decoder(W, H, CFG)
    evs = []
    for i, ((f18, _), (bt, sa, lv)) in enumerate(zip(slices, tabs)):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        cb._check(L.evxg_decode_frame(dec.h, f18, C.c_void_p(bt.data_ptr()), C.c_void_p(sa.data_ptr()),
                                      C.c_void_p(lv.data_ptr()), 1, C.c_void_p(rgb.data_ptr()), 1, sp))
        e1.record()
        if i >= args.warmup:
            evs.append((e0, e1))
    dec.sync(stream.cuda_stream)
    ms = [a.elapsed_time(b) for a, b in evs]
    device_last = rgb.cpu().numpy().reshape(H, W, 3)
    dec.close()
    # e2e: the .evx bytes, record by record
    data = np.frombuffer(cb.stream_header(CFG, W, H) + b"".join(bytes(f18[:10]) + sl for f18, sl in slices), np.uint8)
    out = torch.empty(H * W * 3, dtype=torch.uint8).pin_memory()
    dec = cb.Decoder(W, H, CFG)
    f = (C.c_uint8 * 18)()
    n = C.c_uint64(0)
    pos, frames_out, t0 = 14, [], None
    for i in range(len(slices)):
        if i == args.warmup:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
        cb._check(L.evxg_decoder_decode_record(dec.h, C.c_void_p(data.ctypes.data + pos), len(data) - pos,
                                               C.c_void_p(out.data_ptr()), f, C.byref(n), sp))
        pos += n.value
        frames_out.append(out.numpy().reshape(H, W, 3).copy())
    e2e_s = time.perf_counter() - t0
    dec.close()
    K = len(slices) - args.warmup
    dbytes = decode_bytes_per_frame(aw, ah)
    peak, peak_kind = peaks()
    line = {
        "value": round(K * EQ / (sum(ms) / 1e3), 3), "unit": UNIT, "ms_per_step": round(sum(ms) / K, 3),
        "p99_frame_ms": round(float(np.percentile(ms, 99)), 3),
        "roofline": {"bound": "hbm", "algorithmic_bytes_per_frame": dbytes,
                     "achieved": round(dbytes * K / (sum(ms) / 1e3) / 1e9, 2), "peak": peak, "unit": "GB/s",
                     "frac": round(dbytes * K / (sum(ms) / 1e3) / 1e9 / peak, 4), "peak_source": f"{peak_kind} hbm_gbs"},
        "e2e": {"value": round(K * EQ / e2e_s, 3), "unit": UNIT, "ms_per_step": round(e2e_s * 1e3 / K, 3),
                "entropy_ms_per_frame": round(ent_s * 1e3 / len(slices), 3),
                "h2d_bytes_per_step": int(np.mean([len(sl) + 10 for _, sl in slices])) + nblk * 44 + ne * 2,
                "d2h_bytes_per_step": W * H * 3},
        "device_equals_e2e": bool(np.array_equal(device_last, frames_out[-1])),
        "workload": f"decoding the GPU arm's own {CFG} stream of frames 0..{len(slices) - 1} (1920x1080, quality "
                    f"{QUALITY}); timed frames {args.warmup}..{len(slices) - 1}",
    }
    return line, frames_out


# The batched configuration: 16 streams -- 4 x 1920x1080, 6 x 1280x720,
# 6 x 640x360 -- each with its own seed and GOP phase (I/P GOP of 30, three
# references standing in for two, an intra frame every 30 frames from its own
# start), quality 8.
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
    from chicago_b200.gop import plan as gop_plan
    from chicago_b200.synth import generate
    mix = BATCH_MIX[:args.batch] if args.batch < len(BATCH_MIX) else BATCH_MIX
    warm, K = args.warmup, args.batch_ticks
    nfr = warm + K + 4
    seqs = []
    for k, (w, h) in enumerate(mix):
        frames = generate(w, h, nfr, seed=2000 + k, vmax=max(6.0, 24.0 * w / 1920), n_rects=4)
        phase = (7 * k) % 30   # this stream's GOP position: its next intra frame
        seqs.append((frames, gop_plan(nfr, quality=QUALITY, intra_at=tuple(range(phase, nfr, 30)), cfg=CFG)))
    streams = [cb.Stream(w, h, CFG) for w, h in mix]
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
           "gop": "I/P GOP of 30 per stream (own phase), 3 references standing in for 2, quality 8",
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
# +-2 ms jitter from a random phase, each stream an I/P GOP of 60 with one or
# three references (three standing in for two), quality 8.
SERVE_SIZES = [(640, 360), (1280, 720), (1920, 1080), (3840, 2160)]


def run_served(args, n=None, per=None, sizes_from=None, seed=7):
    """The request loop (evxg_server_*): all streams admitted by the device
    memory budget (spread over the server's lanes by size), frames submitted at
    their arrival times by this thread, each lane's worker batching whatever
    of its streams is ready.  A frame's latency is its done time (results seen
    by the host) minus its arrival time, queueing included; each stream sends
    `serve_frames` frames (a GOP) and then closes."""
    import chicago_b200 as cb
    from chicago_b200.synth import generate
    rng = np.random.default_rng(seed)
    n = args.serve_streams if n is None else n
    per = args.serve_frames if per is None else per
    choices = SERVE_SIZES if sizes_from is None else sizes_from
    sizes = [choices[i] for i in rng.integers(0, len(choices), n)]
    cfgs = ["ip1" if i else "ip3" for i in rng.integers(0, 2, n)]
    pool = {sz: generate(sz[0], sz[1], per + 3, seed=3000 + k, vmax=max(4.0, 24.0 * sz[0] / 1920))
            for k, sz in enumerate(SERVE_SIZES) if sz in sizes}
    srv = cb.Server(hbm_budget_bytes=96 << 30, max_streams=n, keep_tables=False)
    ids = [srv.open(w, h, QUALITY, cfg=c) for (w, h), c in zip(sizes, cfgs)]
    srv.drain()   # the batch over every admitted stream exists before the first arrival
    phase = rng.uniform(0, 1 / 60, n)
    events = sorted((phase[k] + t / 60 + rng.uniform(-0.002, 0.002), k, t) for k in range(n) for t in range(per))
    t0 = cb.Server.now_ns()
    sent = [0] * n
    for at, k, t in events:
        due = t0 + int(max(at, 0.0) * 1e9)
        while (left := due - cb.Server.now_ns()) > 0:
            time.sleep(min(0.0005, left / 1e9))
        off = k % 3   # streams of a size class start at different frames of its pool
        if t > 0 and t % 60 == 0:
            srv.insert_intra(ids[k])   # GOP of 60
        srv.submit(ids[k], pool[sizes[k]][off + t], arrival_ns=cb.Server.now_ns())
        sent[k] += 1
        if sent[k] == per:
            srv.close_stream(ids[k])
    srv.drain()
    lat, work, steady, wait, run, eq, first, last = [], [], [], [], [], 0.0, None, 0
    for k, sid in enumerate(ids):
        w, h = sizes[k]
        for j, r in enumerate(srv.results[sid]):
            a, rd, ln, d = r["times"]
            lat.append((d - a) / 1e6)
            wait.append((ln - a) / 1e6)
            run.append((d - ln) / 1e6)
            if j > 0:   # after the stream's first frame (its I frame, its lane's first tick)
                steady.append((d - a) / 1e6)
            work.append((d - rd) / 1e6)
            eq += w * h / (1920 * 1080)
            first = a if first is None else min(first, a)
            last = max(last, d)
    st = srv.stats()
    srv.close()
    offered = sum(w * h for w, h in sizes) / (1920 * 1080) * 60
    counts = {f"{w}x{h}": sizes.count((w, h)) for w, h in SERVE_SIZES if (w, h) in sizes}
    return {"streams": n, "sizes": counts, "references": {"1": cfgs.count("ip1"), "3": cfgs.count("ip3")},
            "frames": len(lat), "frames_per_stream": per,
            "value": round(eq / ((last - first) / 1e9), 3), "unit": UNIT,
            "offered_1080p_eq_fps": round(offered, 1),
            "p50_frame_ms": round(float(np.percentile(lat, 50)), 3),
            "p99_frame_ms": round(float(np.percentile(lat, 99)), 3),
            "p999_frame_ms": round(float(np.percentile(lat, 99.9)), 3),
            "ready_to_done_ms": {q: round(float(np.percentile(work, v)), 3) for q, v in (("p50", 50), ("p99", 99), ("p999", 99.9))},
            "after_first_frame_ms": {q: round(float(np.percentile(steady, v)), 3) for q, v in (("p50", 50), ("p99", 99), ("p999", 99.9))},
            "arrival_to_launch_ms": {q: round(float(np.percentile(wait, v)), 3) for q, v in (("p50", 50), ("p99", 99))},
            "launch_to_done_ms": {q: round(float(np.percentile(run, v)), 3) for q, v in (("p50", 50), ("p99", 99))},
            "target_ms": round(1000 / 60, 1), "lanes": min(n, 8),
            "ticks": st["ticks"], "batch_rebuilds": st["rebuilds"],
            "note": "latency = results seen by the host minus arrival (I/P GOP: no reorder wait), queueing included"}


def cpu_baseline(order, slices, frames, decoded=None):
    """The reference encoder of the same build (I/P, three references; built
    here from its sources) on the host cores, over the GPU arm's warm-up and
    timed frames: with its WPP threads on all cores, and single-threaded
    (EVX_ENABLE_WPP 0) on the first two frames.  Also the parity check: the
    .evx stream the GPU arm produced for those frames (its e2e leg: GPU pixel
    pipeline and the library's own entropy coder, no reference code) must
    equal the reference's stock stream byte for byte (but the header's
    padding byte, which the reference leaves uninitialised)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import chicago_b200 as cb
    from oracle_py import REF_VARIANTS, Ref
    n = len(order)
    if not os.path.exists(REF_VARIANTS[CFG][0]):
        return None, {"checked": False, "why": "reference I/P build not present"}
    ref = Ref(variant=CFG)
    t0 = time.perf_counter()
    stock = ref.encode_stream(frames[:n], quality=QUALITY, intra_at=tuple(t for t in (CUT,) if t < n))
    dt = time.perf_counter() - t0
    base = {"value": round(n * EQ / dt, 4), "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
            "cpu_model": cpu_model(),
            "sample": f"frames 0..{n - 1} of the workload (the GPU arm's warm-up and timed frames) through "
                      "create_encoder/encode of the reference's I/P build (3 references), its WPP threads on every "
                      "core; host entropy coding included"}
    if os.path.exists(REF_VARIANTS["ip3seq"][0]):
        seq = Ref(variant="ip3seq")
        m = 2
        t0 = time.perf_counter()
        s2 = seq.encode_stream(frames[:m], quality=QUALITY)
        d1 = time.perf_counter() - t0
        base["single_thread"] = {"value": round(m * EQ / d1, 4), "unit": UNIT, "cores": 1,
                                 "sample": f"frames 0..{m - 1}, the same build with EVX_ENABLE_WPP 0",
                                 "same_bytes_as_wpp": s2[:7] == stock[:7] and s2[8:] == stock[8:len(s2)]}
    mine = cb.stream_header(CFG, W, H) + b"".join(bytes(f18[:10]) + sl for f18, sl in slices)
    parity = {"frames": len(slices), "match": len(mine) == len(stock) and mine[:7] == stock[:7] and mine[8:] == stock[8:],
              "bytes": len(stock),
              "how": "the .evx stream of every warm-up and timed frame from the GPU arm's e2e leg (GPU pixel pipeline + "
                     "the library's host entropy coder) vs the reference build's stock stream of the same frames"}
    if decoded is not None:   # the reference decoder on the same records, one per call (its I/P build's framing)
        records = [bytes(f18[:10]) + sl for f18, sl in slices]
        records[0] = cb.stream_header(CFG, W, H) + records[0]
        t0 = time.perf_counter()
        want = ref.decode_records(records, W, H)
        dt = time.perf_counter() - t0
        base["decode"] = {"value": round(len(records) * EQ / dt, 4), "unit": UNIT, "cores": os.cpu_count(),
                          "sample": f"frames 0..{len(records) - 1}: the reference decoder (evx3_decoder, WPP threads) "
                                    "on the GPU arm's records, entropy decoding included"}
        parity["decode_match"] = len(want) == len(decoded) and all(np.array_equal(a, b) for a, b in zip(want, decoded))
    return base, parity


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle_py import REF_VARIANTS, Ref
    if not os.path.exists(REF_VARIANTS[CFG][0]):
        print(json.dumps({"impl": "reference", "unavailable": f"reference build {REF_VARIANTS[CFG][0]} not present"}))
        return
    import ctypes as C
    ref = Ref(variant=CFG)
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
            "config": {"workload": "same sequence as the GPU arm, stream 0: 1920x1080, quality 8, " + GOP_DESC,
                       "reference_build": "EVX_ENABLE_B_FRAMES 0, EVX_REFERENCE_FRAME_COUNT 4",
                       "frames": FRAMES, "quality": QUALITY},
            "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                             "cpu_model": cpu_model(),
                             "sample": f"{K} frames after {args.warmup} warm-up frames, WPP threads, "
                                       "host entropy coding included"},
            "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch", type=int, default=16, help="streams of the batched measurement (1 = skip)")
    ap.add_argument("--batch-ticks", type=int, default=12, help="timed ticks of the batched measurement")
    ap.add_argument("--serve-streams", type=int, default=64, help="streams of the serving measurement (0 = skip)")
    ap.add_argument("--serve-frames", type=int, default=60, help="frames each served stream sends (a GOP)")
    ap.add_argument("--decode-only", action="store_true",
                    help="only the decode leg (its stream from the e2e leg) -- for profiling the decoder")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        run_reference(args)
    elif args.decode_only:
        run_decode_only(args)
    else:
        run_gpu(args)


def run_decode_only(args):
    """The e2e leg to make the stream, then the decode leg alone; prints the
    decode leg's JSON object (not a bench line)."""
    import torch
    torch.cuda.set_device(0)
    sched = plan()
    K = min(args.steps, len(sched) - args.warmup)
    order = sched[:args.warmup + K]
    frames = frames_for(0)
    stream = torch.cuda.current_stream()
    _, slices, _ = run_e2e(args, frames, order, stream)
    line, _ = run_decode(args, slices, stream)
    print(json.dumps({"decode": line}), flush=True)


if __name__ == "__main__":
    main()
