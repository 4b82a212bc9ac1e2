"""ctypes bindings for the test-only CPU checkers (never imported by the product).

* ``Ref``      -- the unmodified reference encoder built from its own sources
                  (oracle/_ref/libevxref.so, see oracle/Makefile and
                  oracle/ref_harness.cpp): stock public API and a staged
                  per-frame driver with stage dumps.
* ``Oracle``   -- this project's plain-C restatement (oracle/_build/liboracle.so).
* ``plan_gop`` -- the frame-type / DPB-slot schedule of the reference encoder's
                  GOP logic (src/video/evx3enc.cpp:105-414), restated in Python,
                  used to drive the staged engines frame by frame.
* ``plan_ip``  -- the same for the I/P builds (EVX_ENABLE_B_FRAMES 0,
                  evx3enc.cpp:137-160): one frame out per frame in.

Build variants of the reference (oracle/variants/, ``REF_VARIANTS``): "ip1"
(I/P GOP, one reference), "ip3" (I/P GOP, three references), "seq" (default
GOP, one thread), "ip3seq" ("ip3", one thread).  ``Ref(variant=...)`` loads one; ``Oracle.context(...,
config=...)`` restates the same switches.
"""
from __future__ import annotations

import ctypes as C
import os
import struct

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libevxref.so")
# variant -> (library, EVX_ENABLE_B_FRAMES, EVX_REFERENCE_FRAME_COUNT)
REF_VARIANTS = {
    "ip1": (os.path.join(HERE, "_ref", "libevxref_ip1.so"), 0, 2),
    "ip3": (os.path.join(HERE, "_ref", "libevxref_ip3.so"), 0, 4),
    "seq": (os.path.join(HERE, "_ref", "libevxref_seq.so"), 1, 4),
    "ip3seq": (os.path.join(HERE, "_ref", "libevxref_ip3seq.so"), 0, 4),
}
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")

BLOCK_DTYPE = np.dtype([
    ("block_type", "<i4"), ("prediction_target", "u1"), ("pad0", "u1"),
    ("motion_x", "<i2"), ("motion_y", "<i2"), ("sp_pred", "u1"), ("sp_amount", "u1"),
    ("sp_index", "u1"), ("q_index", "u1"), ("intra_mode", "u1"), ("pad1", "u1"),
    ("variance", "<i2"), ("prediction_mode", "u1"), ("prediction_target_b", "u1"),
    ("motion_x_b", "<i2"), ("motion_y_b", "<i2"), ("sp_pred_b", "u1"), ("sp_amount_b", "u1"),
    ("sp_index_b", "u1"), ("pad2", "u1")])
assert BLOCK_DTYPE.itemsize == 28
BLOCK_FIELDS = [n for n in BLOCK_DTYPE.names if not n.startswith("pad")]
SAO_DTYPE = np.dtype([("merge_left", "u1"), ("merge_above", "u1"),
                      ("l_type", "u1"), ("l_eo", "u1"), ("l_band", "u1"), ("l_off", "i1", 4),
                      ("c_type", "u1"), ("c_eo", "u1"), ("c_band", "u1"), ("c_off", "i1", 4)])
assert SAO_DTYPE.itemsize == 16

FRAME_INTRA, FRAME_INTER, FRAME_BIDIR = 0, 1, 2


def align16(v: int) -> int:
    return (v + 15) & ~15


def pack_frame(ftype, index, quality, display_order, is_reference, dpb_slot, ref_fwd, ref_bwd) -> bytes:
    """18-byte evx_frame (src/video/common.h:72-87, pack(2))."""
    return struct.pack("<iIHIBBBB", ftype, index, quality, display_order,
                       is_reference, dpb_slot, ref_fwd, ref_bwd)


def unpack_frame(b: bytes) -> dict:
    t, i, q, d, r, s, f, bw = struct.unpack("<iIHIBBBB", bytes(b[:18]))
    return dict(type=t, index=i, quality=q, display_order=d, is_reference=r,
                dpb_slot=s, ref_fwd=f, ref_bwd=bw)


def quality_to_qp(q: int) -> int:
    """evx3_encoder::set_quality (src/video/evx3enc.cpp:64-82)."""
    q = min(max(int(q), 1), 31)
    qp = q if q <= 16 else q + ((q - 16) * (q - 16)) // 10
    return min(qp, 63)


def plan_gop(n_frames: int, quality: int = 8, intra_at=(), b_frames: int = 3):
    """Yield (input_frame_index, frame18) in encode order, mirroring the
    reference's reorder/GOP logic with the default EVX_B_FRAME_COUNT 3.
    ``intra_at`` lists input indices before which insert_intra() is called."""
    qp = quality_to_qp(quality)
    st = dict(type=FRAME_INTRA, index=0, reorder=[], doc=0, ip=0, first=True)
    out = []

    def slot(ip):
        return (ip & 0xFFFFFFFF) % 2

    def gop():
        r = st["reorder"]
        p_in, p_do = r[-1]
        out.append((p_in, pack_frame(FRAME_INTER, st["index"], qp, p_do, 1, slot(st["ip"]), slot(st["ip"] - 1), 0)))
        st["index"] += 1
        bc = len(r) - 1
        if bc > 0:
            ref = bc // 2
            b_in, b_do = r[ref]
            out.append((b_in, pack_frame(FRAME_BIDIR, st["index"], min(qp + 1, 31), b_do, 1, 2,
                                         slot(st["ip"] - 1), slot(st["ip"]))))
            st["index"] += 1
            for bi in range(bc):
                if bi == ref:
                    continue
                b_in, b_do = r[bi]
                fw, bw = (slot(st["ip"] - 1), 2) if bi < ref else (2, slot(st["ip"]))
                out.append((b_in, pack_frame(FRAME_BIDIR, st["index"], min(qp + 2, 31), b_do, 0, 3, fw, bw)))
                st["index"] += 1
        st["ip"] += 1
        st["type"] = FRAME_INTER
        st["reorder"] = []

    for t in range(n_frames):
        if t in intra_at:
            st["type"] = FRAME_INTRA
        if st["doc"] > 0 and st["doc"] % 3600 == 0:
            if st["reorder"]:
                gop()
            st["type"] = FRAME_INTRA
            st["ip"] = 0
        as_intra = st["type"] == FRAME_INTRA
        if as_intra and not st["first"] and st["reorder"]:
            gop()
            st["ip"] = 0
        st["reorder"].append((t, st["doc"]))
        st["doc"] += 1
        if st["first"] or as_intra:
            st["first"] = False
            i_in, i_do = st["reorder"][0]
            out.append((i_in, pack_frame(FRAME_INTRA, st["index"], qp, i_do, 1, slot(st["ip"]), 0, 0)))
            st["ip"] += 1
            st["type"] = FRAME_INTER
            st["index"] += 1
            st["reorder"] = []
        elif len(st["reorder"]) == b_frames + 1:
            gop()
    # flush()
    r = st["reorder"]
    if len(r) == 1:
        p_in, p_do = r[0]
        out.append((p_in, pack_frame(FRAME_INTER, st["index"], qp, p_do, 1, slot(st["ip"]), slot(st["ip"] - 1), 0)))
    elif len(r) > 1:
        gop()
    return out


def plan_ip(n_frames: int, quality: int = 8, intra_at=(), ref_count: int = 2):
    """Yield (input_frame_index, frame18) for the I/P builds
    (EVX_ENABLE_B_FRAMES 0): every frame is encoded as it arrives
    (evx3enc.cpp:137-160), an I frame first and after each insert_intra(),
    else a P frame; the index grows by one per frame and selects the DPB slots
    (query_prediction_index_by_offset, common.cpp:256-259).  Only the first 10
    bytes (type, index, quality) exist in those builds; the rest of the 18-byte
    record carries the slots the index selects: dpb_slot = offset 0,
    ref_fwd = offset 1."""
    qp = quality_to_qp(quality)
    out, ftype = [], FRAME_INTRA
    for t in range(n_frames):
        if t in intra_at:
            ftype = FRAME_INTRA
        out.append((t, pack_frame(ftype, t, qp, t, 1, t % ref_count, (t + ref_count - 1) % ref_count, 0)))
        ftype = FRAME_INTER
        if (t + 1) % 3600 == 0:   # EVX_PERIODIC_INTRA_RATE
            ftype = FRAME_INTRA
    return out


def join_ip_stream(header: bytes, frames) -> bytes:
    """An I/P build's stream: the 14-byte header, then per frame its 10-byte
    evx_frame and the slice bytes, with no size prefix (evx3enc.cpp:141-147)."""
    return header + b"".join(bytes(f18[:10]) + sl for f18, sl in frames)


def split_stream(data: bytes):
    """Split a stock .evx stream into (header, [frame payloads]); each payload
    is frame18 + slice bytes (evx3enc.cpp:249-277)."""
    hdr, pos, frames = bytes(data[:14]), 14, []
    while pos < len(data):
        (n,) = struct.unpack("<I", data[pos:pos + 4])
        frames.append(bytes(data[pos + 4:pos + 4 + n]))
        pos += 4 + n
    return hdr, frames


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class StageDump:
    """Per-frame stage buffers in the plane-set layout."""

    def __init__(self, aw, ah):
        n = aw * ah + 2 * (aw // 2) * (ah // 2)
        nblk = (aw // 16) * (ah // 16)
        self.src = np.zeros(n, np.int16)
        self.blocks = np.zeros(nblk * 28, np.uint8)
        self.levels = np.zeros(n, np.int16)
        self.recon = np.zeros(n, np.int16)
        self.deblock = np.zeros(n, np.int16)
        self.sao = np.zeros(nblk * 16, np.uint8)
        self.final = np.zeros(n, np.int16)

    def block_table(self):
        return self.blocks.view(BLOCK_DTYPE)

    def sao_table(self):
        return self.sao.view(SAO_DTYPE)


class Ref:
    """The unmodified reference library (built here from its own sources)."""

    def __init__(self, path: str = REF_SO, variant: str | None = None):
        if variant is not None:
            path = REF_VARIANTS[variant][0]
        if not os.path.exists(path):
            raise FileNotFoundError(f"reference library not built: {path} (make -C oracle ref variants)")
        L = self.lib = C.CDLL(path)
        L.evxref_config.argtypes = [C.POINTER(C.c_int)] * 5
        v = [C.c_int(0) for _ in range(5)]
        L.evxref_config(*[C.byref(x) for x in v])
        self.b_frames, self.ref_count, self.wpp, self.frame_bytes, self.block_bytes = [x.value for x in v]
        L.evxref_enc_create.restype = C.c_void_p
        L.evxref_enc_create.argtypes = [C.c_uint32]
        L.evxref_enc_destroy.argtypes = [C.c_void_p]
        L.evxref_enc_set_quality.argtypes = [C.c_void_p, C.c_uint8]
        L.evxref_enc_insert_intra.argtypes = [C.c_void_p]
        L.evxref_enc_encode.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                        C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32)]
        L.evxref_enc_flush.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32)]
        L.evxref_enc_peek.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        self.staged = hasattr(L, "evxref_ctx_create")   # builds without encode.cpp have the stock API only
        if self.staged:
            L.evxref_ctx_create.restype = C.c_void_p
            L.evxref_ctx_create.argtypes = [C.c_uint32, C.c_uint32]
            L.evxref_ctx_destroy.argtypes = [C.c_void_p]
            L.evxref_ctx_encode_frame.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                                  C.c_char_p, C.c_int] + [C.c_void_p] * 8 + \
                                                 [C.c_uint32, C.POINTER(C.c_uint32)]
            L.evxref_ctx_serialize.argtypes = [C.c_void_p, C.c_char_p] + [C.c_void_p] * 5 + \
                                              [C.c_uint32, C.POINTER(C.c_uint32)]
            L.evxref_ctx_get_slot.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
        L.evxref_lambda.restype = C.c_float
        L.evxref_lambda.argtypes = [C.c_uint16]
        L.evxref_decode_stream.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p,
                                           C.c_uint32, C.POINTER(C.c_uint32)]
        L.evxref_decode_records.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32,
                                            C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32)]
        L.evxref_mux_file.argtypes = [C.c_char_p, C.c_uint16, C.c_uint16, C.c_float, C.c_int, C.c_uint32, C.c_void_p,
                                      C.c_void_p, C.c_void_p]
        L.evxref_encode_container.argtypes = [C.c_char_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_double,
                                              C.c_uint8]
        L.evxref_demux_file.argtypes = [C.c_char_p, C.POINTER(C.c_uint32), C.c_void_p, C.c_uint64, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32)]
        L.evxref_dctx_create.restype = C.c_void_p
        L.evxref_dctx_create.argtypes = [C.c_uint32, C.c_uint32]
        L.evxref_dctx_destroy.argtypes = [C.c_void_p]
        L.evxref_dctx_decode_frame.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32] + \
            [C.c_void_p] * 6

    # --- stock API ---
    def encode_stream(self, frames: np.ndarray, quality: int = 8, intra_at=(), chunks: bool = False):
        """Encode (T,H,W,3) uint8 frames through create_encoder/encode/flush;
        chunks=True: each encode() call's output and flush()'s, as a list."""
        T, H, W, _ = frames.shape
        cap = max(1 << 22, W * H * 3 * 8)
        h = self.lib.evxref_enc_create(cap)
        buf = np.zeros(cap, np.uint8)
        n = C.c_uint32(0)
        out = []
        try:
            self.lib.evxref_enc_set_quality(h, quality)
            for t in range(T):
                if t in intra_at:
                    self.lib.evxref_enc_insert_intra(h)
                f = np.ascontiguousarray(frames[t])
                rc = self.lib.evxref_enc_encode(h, _p(f), W, H, _p(buf), cap, C.byref(n))
                if rc:
                    raise RuntimeError(f"reference encode failed: {rc}")
                out.append(buf[:n.value].tobytes())
            rc = self.lib.evxref_enc_flush(h, _p(buf), cap, C.byref(n))
            if rc:
                raise RuntimeError(f"reference flush failed: {rc}")
            out.append(buf[:n.value].tobytes())
        finally:
            self.lib.evxref_enc_destroy(h)
        return out if chunks else b"".join(out)

    def peeks(self, frames: np.ndarray, quality: int, states) -> list:
        """Encode (T,H,W,3) frames with the stock encoder and after every
        encode() call take peek(state) for each state: [{state: (H,W,3)}]."""
        T, H, W, _ = frames.shape
        cap = max(1 << 22, W * H * 3 * 8)
        h = self.lib.evxref_enc_create(cap)
        buf = np.zeros(cap, np.uint8)
        n = C.c_uint32(0)
        out = []
        try:
            self.lib.evxref_enc_set_quality(h, quality)
            for t in range(T):
                f = np.ascontiguousarray(frames[t])
                if self.lib.evxref_enc_encode(h, _p(f), W, H, _p(buf), cap, C.byref(n)):
                    raise RuntimeError("reference encode failed")
                views = {}
                for st in states:
                    img = np.zeros((H, W, 3), np.uint8)
                    rc = self.lib.evxref_enc_peek(h, st, _p(img))
                    views[st] = img if rc == 0 else rc
                out.append(views)
        finally:
            self.lib.evxref_enc_destroy(h)
        return out

    def decode_stream(self, data: bytes, width: int, height: int, max_frames: int = 256) -> np.ndarray:
        """Decode a whole .evx stream with the stock decoder; (T,H,W,3) frames in display order."""
        out = np.zeros((max_frames, height, width, 3), np.uint8)
        n = C.c_uint32(0)
        buf = np.frombuffer(data, np.uint8).copy()
        rc = self.lib.evxref_decode_stream(_p(buf), len(data), width, height, _p(out), max_frames, C.byref(n))
        if rc:
            raise RuntimeError(f"reference decode failed: {rc}")
        return out[:min(n.value, max_frames)]

    def decode_records(self, records, width: int, height: int) -> np.ndarray:
        """The stock decoder fed one record per call (records[0] starts with the
        stream header); (T,H,W,3) frames in display order."""
        data = np.frombuffer(b"".join(records), np.uint8).copy()
        offs = np.cumsum([0] + [len(r) for r in records]).astype(np.uint32)
        out = np.zeros((len(records), height, width, 3), np.uint8)
        n = C.c_uint32(0)
        rc = self.lib.evxref_decode_records(_p(data), _p(offs), len(records), width, height, _p(out), len(records),
                                            C.byref(n))
        if rc:
            raise RuntimeError(f"reference decode failed: {rc} after {n.value} frames")
        return out[:n.value]

    # --- container (evx_muxer / evx_demuxer) ---
    def mux_file(self, path: str, width: int, height: int, fps: float, packets, with_audio: bool = False):
        """Write packets [(timestamp_us, payload)] of one video stream with evx_muxer."""
        data = np.frombuffer(b"".join(p for _, p in packets) or b"\0", np.uint8).copy()
        offs = np.cumsum([0] + [len(p) for _, p in packets]).astype(np.uint32)
        ts = np.array([t for t, _ in packets] or [0], np.uint64)
        rc = self.lib.evxref_mux_file(os.fsencode(path), width, height, fps, int(with_audio), len(packets), _p(data),
                                      _p(offs), _p(ts))
        if rc:
            raise RuntimeError(f"reference muxer failed: {rc}")

    def encode_container(self, path: str, frames: np.ndarray, fps: float, quality: int):
        """The reference encoder tool's video path over raw RGB24 frames (T,H,W,3)."""
        T, H, W, _ = frames.shape
        f = np.ascontiguousarray(frames)
        rc = self.lib.evxref_encode_container(os.fsencode(path), _p(f), T, W, H, fps, quality)
        if rc:
            raise RuntimeError(f"reference container encode failed: {rc}")

    def demux_file(self, path: str, max_packets: int = 4096):
        """(stream count, [(stream_id, timestamp_us, payload)]) read with evx_demuxer."""
        cap = os.path.getsize(path)
        data = np.zeros(max(cap, 1), np.uint8)
        sizes = np.zeros(max_packets, np.uint32)
        ids = np.zeros(max_packets, np.uint8)
        ts = np.zeros(max_packets, np.uint64)
        ns, n = C.c_uint32(0), C.c_uint32(0)
        rc = self.lib.evxref_demux_file(os.fsencode(path), C.byref(ns), _p(data), cap, _p(sizes), _p(ids), _p(ts),
                                        max_packets, C.byref(n))
        if rc:
            raise RuntimeError(f"reference demuxer failed: {rc}")
        out, pos = [], 0
        for k in range(min(n.value, max_packets)):
            out.append((int(ids[k]), int(ts[k]), data[pos:pos + sizes[k]].tobytes()))
            pos += int(sizes[k])
        return ns.value, out

    # --- staged engine ---
    def context(self, width: int, height: int):
        return RefContext(self, align16(width), align16(height))

    def decoder(self, width: int, height: int):
        """Staged engine_decode_frame with dumps (see RefDecodeContext)."""
        return RefDecodeContext(self, width, height)

    def lam(self, q: int) -> float:
        return self.lib.evxref_lambda(q)


class RefDecodeContext:
    """The reference's engine_decode_frame step by step (decode.cpp:560-612):
    decode_frame(record) takes one frame record (evx_frame + slice) and returns
    what unserialize_slice produced -- descriptor (18-byte layout), block table
    (28-byte layout), SAO table, level planes -- plus the final reconstruction
    and the RGB24 frame."""

    def __init__(self, ref: Ref, width: int, height: int):
        self.ref, self.w, self.h = ref, width, height
        self.aw, self.ah = align16(width), align16(height)
        self.hd = ref.lib.evxref_dctx_create(self.aw, self.ah)
        if not self.hd:
            raise RuntimeError("reference decoder context creation failed")

    def __del__(self):
        if getattr(self, "hd", None):
            self.ref.lib.evxref_dctx_destroy(self.hd)
            self.hd = None

    def decode_frame(self, record: bytes) -> dict:
        n = self.aw * self.ah + 2 * (self.aw // 2) * (self.ah // 2)
        nblk = (self.aw // 16) * (self.ah // 16)
        out = dict(frame18=np.zeros(18, np.uint8), blocks=np.zeros(nblk * 28, np.uint8),
                   sao=np.zeros(nblk * 16, np.uint8), levels=np.zeros(n, np.int16), final=np.zeros(n, np.int16),
                   rgb=np.zeros((self.h, self.w, 3), np.uint8))
        buf = np.frombuffer(record, np.uint8).copy()
        rc = self.ref.lib.evxref_dctx_decode_frame(self.hd, _p(buf), len(record), self.w, self.h,
                                                   *[_p(out[k]) for k in ("frame18", "blocks", "sao", "levels",
                                                                          "final", "rgb")])
        if rc:
            raise RuntimeError(f"reference staged decode failed: {rc}")
        out["frame18"] = out["frame18"].tobytes()
        return out


class RefContext:
    def __init__(self, ref: Ref, aw: int, ah: int):
        self.ref, self.aw, self.ah = ref, aw, ah
        self.h = ref.lib.evxref_ctx_create(aw, ah)
        self.cap = aw * ah * 8 + (1 << 20)
        self.buf = np.zeros(self.cap, np.uint8)

    def __del__(self):
        if getattr(self, "h", None):
            self.ref.lib.evxref_ctx_destroy(self.h)
            self.h = None

    def encode_frame(self, rgb: np.ndarray, frame18: bytes, wpp: bool = False):
        H, W, _ = rgb.shape
        d = StageDump(self.aw, self.ah)
        n = C.c_uint32(0)
        rgb = np.ascontiguousarray(rgb)
        rc = self.ref.lib.evxref_ctx_encode_frame(
            self.h, _p(rgb), W, H, frame18, int(wpp), _p(d.src), _p(d.blocks), _p(d.levels),
            _p(d.recon), _p(d.deblock), _p(d.sao), _p(d.final), _p(self.buf), self.cap, C.byref(n))
        if rc:
            raise RuntimeError(f"reference staged encode failed: {rc}")
        return d, self.buf[:n.value].tobytes()

    def serialize(self, frame18: bytes, blocks, prev_blocks, sao, levels) -> bytes:
        n = C.c_uint32(0)
        rc = self.ref.lib.evxref_ctx_serialize(self.h, frame18, _p(blocks), _p(prev_blocks), _p(sao),
                                               _p(levels), _p(self.buf), self.cap, C.byref(n))
        if rc:
            raise RuntimeError(f"reference serialize failed: {rc}")
        return self.buf[:n.value].tobytes()

    def slot(self, s: int) -> np.ndarray:
        out = np.zeros(self.aw * self.ah * 3 // 2, np.int16)
        self.ref.lib.evxref_ctx_get_slot(self.h, s, _p(out))
        return out


class Oracle:
    """This project's plain-C restatement (test infrastructure)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle not built: {path} (make -C oracle oracle)")
        L = self.lib = C.CDLL(path)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_uint32, C.c_uint32]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_set_config.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
        L.orc_encode_frame.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_char_p] + \
                                      [C.c_void_p] * 7
        for nm in ("orc_get_slot",):
            getattr(L, nm).argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
        L.orc_get_prev_blocks.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_get_levels.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_lambda.restype = C.c_float
        L.orc_lambda.argtypes = [C.c_uint16]
        L.orc_hadamard_4x4.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
        L.orc_satd_16x16.restype = C.c_int32
        L.orc_satd_16x16.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32]
        L.orc_interpolate.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                      C.c_int16, C.c_int16, C.c_int32, C.c_void_p]
        L.orc_fdct_8x8.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32]
        L.orc_idct_8x8.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32]
        L.orc_intra_predict.argtypes = [C.c_uint8, C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                                        C.c_int32, C.c_void_p]
        L.orc_mv_predictor.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                       C.POINTER(C.c_int16), C.POINTER(C.c_int16)]
        L.orc_deblock_strength.restype = C.c_uint8
        L.orc_deblock_strength.argtypes = [C.c_int32, C.c_void_p, C.c_void_p]
        L.orc_convert.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32]
        L.orc_yuv_to_rgb.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p]

    def yuv_to_rgb(self, planes: np.ndarray, aw: int, ah: int, width: int, height: int) -> np.ndarray:
        """RGB24 (H,W,3) of an int16 plane set (convert.cpp:162-223)."""
        p = np.ascontiguousarray(planes, dtype=np.int16)
        out = np.zeros((height, width, 3), np.uint8)
        self.lib.orc_yuv_to_rgb(_p(p), aw, ah, width, height, _p(out))
        return out

    def context(self, width: int, height: int, b_frames: int = 1, ref_count: int = 4, radius: int = 16):
        """A stream context restating the reference build with these switches
        (EVX_ENABLE_B_FRAMES, EVX_REFERENCE_FRAME_COUNT, EVX_MOTION_SEARCH_RADIUS)."""
        return OracleContext(self, align16(width), align16(height), b_frames, ref_count, radius)


class OracleContext:
    def __init__(self, orc: Oracle, aw: int, ah: int, b_frames: int = 1, ref_count: int = 4, radius: int = 16):
        self.orc, self.aw, self.ah = orc, aw, ah
        self.h = orc.lib.orc_create(aw, ah)
        if orc.lib.orc_set_config(self.h, b_frames, ref_count, radius):
            raise ValueError(f"unsupported oracle configuration b_frames={b_frames} ref_count={ref_count} radius={radius}")

    def __del__(self):
        if getattr(self, "h", None):
            self.orc.lib.orc_destroy(self.h)
            self.h = None

    def encode_frame(self, rgb: np.ndarray, frame18: bytes):
        H, W, _ = rgb.shape
        d = StageDump(self.aw, self.ah)
        rgb = np.ascontiguousarray(rgb)
        rc = self.orc.lib.orc_encode_frame(self.h, _p(rgb), W, H, frame18, _p(d.src), _p(d.blocks),
                                           _p(d.levels), _p(d.recon), _p(d.deblock), _p(d.sao), _p(d.final))
        if rc:
            raise RuntimeError(f"oracle encode failed: {rc}")
        return d

    def prev_blocks(self) -> np.ndarray:
        out = np.zeros((self.aw // 16) * (self.ah // 16) * 28, np.uint8)
        self.orc.lib.orc_get_prev_blocks(self.h, _p(out))
        return out

    def levels(self) -> np.ndarray:
        out = np.zeros(self.aw * self.ah * 3 // 2, np.int16)
        self.orc.lib.orc_get_levels(self.h, _p(out))
        return out


def compare_blocks(a: np.ndarray, b: np.ndarray):
    """Indices and field names where two block tables differ (padding ignored)."""
    ta, tb = a.view(BLOCK_DTYPE), b.view(BLOCK_DTYPE)
    bad = {}
    for f in BLOCK_FIELDS:
        idx = np.nonzero(ta[f] != tb[f])[0]
        if idx.size:
            bad[f] = idx
    return bad
