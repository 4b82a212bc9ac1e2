"""chicago_b200 -- B200 (sm_100a) EVX3 encoder pixel pipeline behind a C ABI.

Python mirror of the C ABI in include/evxg.h over ctypes.  The CUDA library
chicago_b200/libevxg.so is built in-tree (``python -m chicago_b200.build``);
importing this package without it raises: there is no CPU fallback.

* :class:`Stream`  -- one encoding context: ``encode_frame`` is the reference's
  engine_encode_frame minus serialization (src/video/encode.cpp:945-998),
  ``fetch_tables`` returns what the host entropy coder reads.
* :class:`Encoder` -- the reference's evx3_encoder (src/video/evx3.h:67-100:
  set_quality / insert_intra / encode / flush / clear) with its GOP logic,
  emitting one record per encoded frame in bitstream order.
* :class:`Config` -- the reference build a stream reproduces (EVX_ENABLE_B_FRAMES,
  EVX_REFERENCE_FRAME_COUNT, EVX_MOTION_SEARCH_RADIUS); ``CONFIGS`` names the
  supported ones: "default" (hierarchical P/B GOP), "ip1" / "ip3" (I/P GOP with
  one / three references).
"""
from __future__ import annotations

import ctypes as C
import os
import struct

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libevxg.so")

BLOCK_DTYPE = np.dtype([
    ("block_type", "<i4"), ("prediction_target", "u1"), ("pad0", "u1"),
    ("motion_x", "<i2"), ("motion_y", "<i2"), ("sp_pred", "u1"), ("sp_amount", "u1"),
    ("sp_index", "u1"), ("q_index", "u1"), ("intra_mode", "u1"), ("pad1", "u1"),
    ("variance", "<i2"), ("prediction_mode", "u1"), ("prediction_target_b", "u1"),
    ("motion_x_b", "<i2"), ("motion_y_b", "<i2"), ("sp_pred_b", "u1"), ("sp_amount_b", "u1"),
    ("sp_index_b", "u1"), ("pad2", "u1")])
SAO_DTYPE = np.dtype([("merge_left", "u1"), ("merge_above", "u1"),
                      ("l_type", "u1"), ("l_eo", "u1"), ("l_band", "u1"), ("l_off", "i1", 4),
                      ("c_type", "u1"), ("c_eo", "u1"), ("c_band", "u1"), ("c_off", "i1", 4)])

EVXG_SUCCESS = 0
FRAME_INTRA, FRAME_INTER, FRAME_BIDIR = 0, 1, 2

# Exported entry points, as declared in include/evxg.h.
EXPORTS = [
    "evxg_stream_create", "evxg_stream_destroy", "evxg_stream_dims", "evxg_encode_frame",
    "evxg_fetch_tables", "evxg_fetch_planes", "evxg_stream_sync", "evxg_last_launch_count",
    "evxg_lambda", "evxg_last_error", "evxg_stream_profile", "evxg_stream_kernel_ms", "evxg_encoder_create", "evxg_encoder_destroy",
    "evxg_encoder_clear", "evxg_encoder_insert_intra", "evxg_encoder_set_quality",
    "evxg_encoder_encode", "evxg_encoder_flush", "evxg_encoder_stream", "evxg_mb_pass_noalloc",
    "evxg_stream_set_mb_form", "evxg_stream_mb_form",
    "evxg_batch_create", "evxg_batch_destroy", "evxg_batch_input", "evxg_batch_encode", "evxg_batch_wait",
    "evxg_batch_output", "evxg_batch_launch_count", "evxg_batch_set_shape", "evxg_batch_get_shape",
    "evxg_batch_autotune",
    "evxg_server_create", "evxg_server_destroy", "evxg_server_open", "evxg_server_submit", "evxg_server_insert_intra",
    "evxg_server_close", "evxg_server_drain", "evxg_server_stats", "evxg_server_now_ns",
    "evxg_config_default", "evxg_stream_create_config", "evxg_stream_config", "evxg_encoder_create_config",
    "evxg_server_open_config", "evxg_stream_set_timeout_ns", "evxg_stream_reset", "evxg_batch_set_timeout_ns",
    "evxg_mb_pass_noalloc_set_timeout_ns", "evxg_server_cancel", "evxg_inject_alloc_failures",
    "evxg_serialize_slice", "evxg_stream_header", "evxg_encoder_set_output", "evxg_server_create_lanes",
    "evxg_decoder_create", "evxg_decoder_destroy", "evxg_decode_frame", "evxg_decoder_sync",
    "evxg_decoder_fetch_planes", "evxg_decoder_set_timeout_ns", "evxg_decoder_reset",
    "evxg_unserialize_slice", "evxg_decoder_decode_record",
    "evxg_muxer_open", "evxg_muxer_add_video_stream", "evxg_muxer_add_audio_stream", "evxg_muxer_write_header",
    "evxg_muxer_write_packet", "evxg_muxer_close", "evxg_demuxer_open", "evxg_demuxer_stream_count",
    "evxg_demuxer_stream", "evxg_demuxer_read_packet", "evxg_demuxer_close",
    "evxg_stream_decoder_create", "evxg_stream_decoder_destroy", "evxg_stream_decoder_clear",
    "evxg_stream_decoder_dims", "evxg_stream_decoder_decode", "evxg_stream_decoder_flush",
    "evxg_encode_frame_pipelined", "evxg_stream_output_wait", "evxg_encoder_peek",
    "evxg_stream_state_bytes", "evxg_stream_save", "evxg_stream_restore", "evxg_server_evict", "evxg_server_restore",
]
MB_FORM_SINGLE, MB_FORM_CLUSTER = 0, 1


class Config(C.Structure):
    """evxg_config: the compile-time switches of the reference build a stream
    reproduces (include/evxg.h)."""
    _fields_ = [("b_frames", C.c_uint8), ("ref_count", C.c_uint8), ("search_radius", C.c_uint8),
                ("reserved", C.c_uint8)]


CONFIGS = {"default": (1, 4, 16), "ip1": (0, 2, 16), "ip3": (0, 4, 16)}


def config(name_or_tuple="default") -> Config:
    """A Config from a name in CONFIGS or a (b_frames, ref_count, search_radius) tuple."""
    if isinstance(name_or_tuple, Config):
        return name_or_tuple
    v = CONFIGS[name_or_tuple] if isinstance(name_or_tuple, str) else tuple(name_or_tuple)
    return Config(v[0], v[1], v[2], 0)

FRAME_CB = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p)
BYTES_CB = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p, C.c_uint64)


class FrameTimes(C.Structure):
    _fields_ = [("arrival_ns", C.c_uint64), ("ready_ns", C.c_uint64), ("launch_ns", C.c_uint64), ("done_ns", C.c_uint64)]


RESULT_CB = C.CFUNCTYPE(None, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                        C.POINTER(FrameTimes))


class StreamDesc(C.Structure):
    """evxg_stream_desc: one stream of a container (video: size and frame
    rate; audio: sample rate, channels, bit depth, quality)."""
    _fields_ = [("stream_type", C.c_uint8), ("stream_id", C.c_uint8), ("width", C.c_uint16), ("height", C.c_uint16),
                ("frame_rate", C.c_float), ("sample_rate", C.c_uint32), ("channels", C.c_uint8),
                ("bit_depth", C.c_uint8), ("quality", C.c_uint8)]


STREAM_TYPE_VIDEO, STREAM_TYPE_AUDIO = 0, 1
OPERATION_COMPLETED, CAPACITY_LIMIT = 16, 7


class EvxgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"evxg error {code}: {msg}")
        self.code = code


def _load(path: str = LIB_PATH) -> C.CDLL:
    if not os.path.exists(path):
        raise ImportError(f"CUDA library missing: {path}; build it with `python -m chicago_b200.build`")
    L = C.CDLL(path)
    vp, u32, i32 = C.c_void_p, C.c_uint32, C.c_int
    L.evxg_stream_create.argtypes = [u32, u32, C.POINTER(vp)]
    L.evxg_stream_create_config.argtypes = [u32, u32, C.POINTER(Config), C.POINTER(vp)]
    L.evxg_stream_config.argtypes = [vp, C.POINTER(Config)]
    L.evxg_config_default.argtypes = [C.POINTER(Config)]
    L.evxg_config_default.restype = None
    L.evxg_stream_destroy.argtypes = [vp]
    L.evxg_stream_dims.argtypes = [vp] + [C.POINTER(u32)] * 4
    L.evxg_encode_frame.argtypes = [vp, vp, i32, C.c_char_p, vp]
    L.evxg_fetch_tables.argtypes = [vp, vp, vp, vp, vp, i32, vp]
    L.evxg_fetch_planes.argtypes = [vp, u32, vp, i32, vp]
    L.evxg_stream_sync.argtypes = [vp, vp]
    L.evxg_stream_set_timeout_ns.argtypes = [vp, C.c_int64]
    L.evxg_stream_reset.argtypes = [vp, vp]
    L.evxg_batch_set_timeout_ns.argtypes = [vp, C.c_int64]
    L.evxg_mb_pass_noalloc_set_timeout_ns.argtypes = [C.c_int64]
    L.evxg_last_launch_count.argtypes = [vp]
    L.evxg_last_launch_count.restype = u32
    L.evxg_stream_profile.argtypes = [vp, i32]
    L.evxg_stream_kernel_ms.argtypes = [vp, C.POINTER(C.c_float), u32]
    L.evxg_lambda.argtypes = [C.c_uint16]
    L.evxg_lambda.restype = C.c_float
    L.evxg_last_error.restype = C.c_char_p
    L.evxg_encoder_create.argtypes = [FRAME_CB, vp, C.POINTER(vp)]
    L.evxg_encoder_create_config.argtypes = [FRAME_CB, vp, C.POINTER(Config), C.POINTER(vp)]
    for n in ("evxg_encoder_destroy", "evxg_encoder_clear", "evxg_encoder_insert_intra", "evxg_encoder_flush"):
        getattr(L, n).argtypes = [vp]
    L.evxg_encoder_set_quality.argtypes = [vp, C.c_uint8]
    L.evxg_encoder_encode.argtypes = [vp, vp, u32, u32]
    L.evxg_encoder_stream.argtypes = [vp]
    L.evxg_encoder_stream.restype = vp
    L.evxg_encoder_set_output.argtypes = [vp, BYTES_CB, vp]
    L.evxg_mb_pass_noalloc.argtypes = [u32, u32, C.c_char_p, vp, C.POINTER(vp), vp, vp, vp, vp]
    L.evxg_stream_set_mb_form.argtypes = [vp, i32]
    L.evxg_stream_mb_form.argtypes = [vp]
    L.evxg_batch_create.argtypes = [C.POINTER(vp), u32, C.POINTER(vp)]
    L.evxg_batch_destroy.argtypes = [vp]
    L.evxg_batch_input.argtypes = [vp, u32, u32]
    L.evxg_batch_input.restype = C.POINTER(C.c_uint8)
    L.evxg_batch_encode.argtypes = [vp, C.c_char_p, u32, vp]
    L.evxg_batch_wait.argtypes = [vp, u32]
    L.evxg_batch_output.argtypes = [vp, u32, u32] + [C.POINTER(vp)] * 4
    L.evxg_batch_launch_count.argtypes = [vp]
    L.evxg_batch_launch_count.restype = u32
    L.evxg_batch_set_shape.argtypes = [vp, i32, i32, i32]
    L.evxg_batch_get_shape.argtypes = [vp] + [C.POINTER(i32)] * 3
    L.evxg_batch_autotune.argtypes = [vp, vp, C.POINTER(C.c_float)]
    u64 = C.c_uint64
    L.evxg_server_create.argtypes = [u64, u32, RESULT_CB, vp, C.POINTER(vp)]
    L.evxg_server_create_lanes.argtypes = [u64, u32, u32, RESULT_CB, vp, C.POINTER(vp)]
    L.evxg_server_destroy.argtypes = [vp]
    L.evxg_server_open.argtypes = [vp, u32, u32, C.c_uint8, C.POINTER(u32)]
    L.evxg_server_open_config.argtypes = [vp, u32, u32, C.c_uint8, C.POINTER(Config), C.POINTER(u32)]
    L.evxg_server_submit.argtypes = [vp, u32, vp, u64]
    L.evxg_server_insert_intra.argtypes = [vp, u32]
    L.evxg_server_close.argtypes = [vp, u32]
    L.evxg_server_drain.argtypes = [vp]
    L.evxg_server_cancel.argtypes = [vp, u32]
    L.evxg_inject_alloc_failures.argtypes = [u32]
    L.evxg_serialize_slice.argtypes = [C.POINTER(Config), u32, u32, C.c_char_p, vp, vp, vp, vp, vp, u64,
                                       C.POINTER(u64)]
    L.evxg_stream_header.argtypes = [C.POINTER(Config), u32, u32, vp]
    L.evxg_server_stats.argtypes = [vp] + [C.POINTER(u64)] * 4
    L.evxg_server_now_ns.restype = u64
    L.evxg_decoder_create.argtypes = [u32, u32, C.POINTER(Config), C.POINTER(vp)]
    L.evxg_decoder_destroy.argtypes = [vp]
    L.evxg_decode_frame.argtypes = [vp, C.c_char_p, vp, vp, vp, i32, vp, i32, vp]
    L.evxg_decoder_sync.argtypes = [vp, vp]
    L.evxg_decoder_fetch_planes.argtypes = [vp, u32, vp, i32, vp]
    L.evxg_decoder_set_timeout_ns.argtypes = [vp, C.c_int64]
    L.evxg_decoder_reset.argtypes = [vp, vp]
    L.evxg_unserialize_slice.argtypes = [C.POINTER(Config), u32, u32, C.c_char_p, vp, u64, vp, vp, vp, vp,
                                         C.POINTER(u64)]
    L.evxg_decoder_decode_record.argtypes = [vp, vp, u64, vp, vp, C.POINTER(u64), vp]
    L.evxg_muxer_open.argtypes = [C.c_char_p, C.POINTER(vp)]
    L.evxg_muxer_add_video_stream.argtypes = [vp, C.c_uint16, C.c_uint16, C.c_float, C.POINTER(C.c_uint8)]
    L.evxg_muxer_add_audio_stream.argtypes = [vp, u32, C.c_uint8, C.c_uint8, C.c_uint8, C.POINTER(C.c_uint8)]
    L.evxg_muxer_write_header.argtypes = [vp]
    L.evxg_muxer_write_packet.argtypes = [vp, C.c_uint8, C.c_uint8, u64, vp, u32]
    L.evxg_muxer_close.argtypes = [vp]
    L.evxg_demuxer_open.argtypes = [C.c_char_p, C.POINTER(vp)]
    L.evxg_demuxer_stream_count.argtypes = [vp]
    L.evxg_demuxer_stream_count.restype = u32
    L.evxg_demuxer_stream.argtypes = [vp, u32, C.POINTER(StreamDesc)]
    L.evxg_demuxer_read_packet.argtypes = [vp, C.POINTER(C.c_uint8), C.POINTER(C.c_uint8), C.POINTER(u64), vp, u32,
                                           C.POINTER(u32)]
    L.evxg_demuxer_close.argtypes = [vp]
    L.evxg_stream_decoder_create.argtypes = [C.POINTER(Config), C.POINTER(vp)]
    L.evxg_stream_decoder_destroy.argtypes = [vp]
    L.evxg_stream_decoder_clear.argtypes = [vp]
    L.evxg_stream_decoder_dims.argtypes = [vp, C.POINTER(u32), C.POINTER(u32)]
    L.evxg_stream_decoder_decode.argtypes = [vp, vp, u64, C.POINTER(u64), vp, C.POINTER(C.c_int)]
    L.evxg_stream_decoder_flush.argtypes = [vp, vp, C.POINTER(C.c_int)]
    L.evxg_encode_frame_pipelined.argtypes = [vp, vp, C.c_char_p, vp, vp, vp, vp, vp, C.POINTER(u64)]
    L.evxg_stream_output_wait.argtypes = [vp, u64]
    L.evxg_encoder_peek.argtypes = [vp, i32, vp]
    L.evxg_stream_state_bytes.argtypes = [vp]
    L.evxg_stream_state_bytes.restype = u64
    L.evxg_stream_save.argtypes = [vp, vp, u64, vp]
    L.evxg_stream_restore.argtypes = [vp, vp, u64, vp]
    L.evxg_server_evict.argtypes = [vp, u32]
    L.evxg_server_restore.argtypes = [vp, u32]
    return L


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _check(rc: int):
    if rc != EVXG_SUCCESS:
        raise EvxgError(rc, lib().evxg_last_error().decode(errors="replace"))


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, int):
        return C.c_void_p(a)
    if hasattr(a, "data_ptr"):       # torch tensor
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(C.c_void_p)


def lam(quality: int) -> float:
    return lib().evxg_lambda(quality)


def pack_frame(ftype, index, quality, display_order, is_reference, dpb_slot, ref_fwd, ref_bwd) -> bytes:
    """18-byte evx_frame (reference src/video/common.h:72-87)."""
    return struct.pack("<iIHIBBBB", ftype, index, quality, display_order, is_reference, dpb_slot, ref_fwd, ref_bwd)


def serialize_slice(cfg, aligned_w: int, aligned_h: int, frame18: bytes, blocks, prev_blocks, sao, levels) -> bytes:
    """The frame's slice bytes from its tables (host entropy coder, evxg_serialize_slice)."""
    c = config(cfg)
    cap = max(1 << 16, aligned_w * aligned_h * 4)
    out = np.empty(cap, np.uint8)
    n = C.c_uint64(0)
    _check(lib().evxg_serialize_slice(C.byref(c), aligned_w, aligned_h, frame18, _ptr(np.ascontiguousarray(blocks)),
                                      _ptr(np.ascontiguousarray(prev_blocks)), _ptr(np.ascontiguousarray(sao)),
                                      _ptr(np.ascontiguousarray(levels)), _ptr(out), cap, C.byref(n)))
    return out[:n.value].tobytes()


def unserialize_slice(cfg, aligned_w: int, aligned_h: int, frame18: bytes, data: bytes, blocks, prev_blocks, sao,
                      levels) -> int:
    """Entropy-decode one slice into blocks / sao / levels in place (the tables
    persist across frames: only coded fields are written); returns the slice's
    length in bytes (evxg_unserialize_slice)."""
    c = config(cfg)
    for a in (blocks, prev_blocks, sao, levels):
        if not (isinstance(a, np.ndarray) and a.flags.c_contiguous):
            raise ValueError("tables must be C-contiguous arrays")
    buf = np.frombuffer(data, np.uint8)
    n = C.c_uint64(0)
    _check(lib().evxg_unserialize_slice(C.byref(c), aligned_w, aligned_h, frame18, _ptr(buf), len(data), _ptr(blocks),
                                        _ptr(prev_blocks), _ptr(sao), _ptr(levels), C.byref(n)))
    return n.value


def stream_header(cfg, width: int, height: int) -> bytes:
    """The 14-byte stream header (evxg_stream_header)."""
    c = config(cfg)
    out = np.zeros(14, np.uint8)
    _check(lib().evxg_stream_header(C.byref(c), width, height, _ptr(out)))
    return out.tobytes()


class Stream:
    """One device encoding context (evx_context on the GPU) of the reference
    build ``cfg`` names (see :func:`config`)."""

    def __init__(self, width: int, height: int, cfg="default"):
        self.width, self.height = int(width), int(height)
        self.cfg = config(cfg)
        h = C.c_void_p()
        _check(lib().evxg_stream_create_config(self.width, self.height, C.byref(self.cfg), C.byref(h)))
        self.h = h
        d = [C.c_uint32() for _ in range(4)]
        _check(lib().evxg_stream_dims(self.h, *[C.byref(x) for x in d]))
        self.aw, self.ah, self.mbw, self.mbh = (x.value for x in d)
        self.nblk = self.mbw * self.mbh
        self.plane_elems = self.aw * self.ah + 2 * (self.aw // 2) * (self.ah // 2)

    def close(self):
        if getattr(self, "h", None):
            lib().evxg_stream_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def encode_frame(self, rgb, frame18: bytes, on_device: bool = False, cuda_stream=None):
        """Asynchronously encode one RGB24 frame (host ndarray, or device pointer/tensor)."""
        if not on_device:
            rgb = np.ascontiguousarray(rgb, dtype=np.uint8)
            if rgb.size != self.width * self.height * 3:
                raise ValueError("rgb must hold width*height*3 bytes")
        _check(lib().evxg_encode_frame(self.h, _ptr(rgb), int(on_device), frame18, _ptr(cuda_stream)))

    def sync(self, cuda_stream=None):
        _check(lib().evxg_stream_sync(self.h, _ptr(cuda_stream)))

    def encode_pipelined(self, rgb, frame18: bytes, out: dict, cuda_stream=None) -> int:
        """evxg_encode_frame_pipelined: encode a host RGB24 frame without waiting;
        its tables land in out (arrays as fetch_tables returns them, kept alive by
        the caller) once output_wait(ticket) returns.  Returns the ticket."""
        t = C.c_uint64()
        _check(lib().evxg_encode_frame_pipelined(self.h, _ptr(rgb), frame18, _ptr(out["blocks"]),
                                                 _ptr(out["prev_blocks"]), _ptr(out["sao"]), _ptr(out["levels"]),
                                                 _ptr(cuda_stream), C.byref(t)))
        return t.value

    def output_wait(self, ticket: int):
        _check(lib().evxg_stream_output_wait(self.h, ticket))

    def save(self, cuda_stream=None) -> bytes:
        """evxg_stream_save: the stream's device state, to continue it later."""
        buf = np.empty(lib().evxg_stream_state_bytes(self.h), np.uint8)
        _check(lib().evxg_stream_save(self.h, _ptr(buf), len(buf), _ptr(cuda_stream)))
        return buf.tobytes()

    def restore(self, state: bytes, cuda_stream=None):
        buf = np.frombuffer(state, np.uint8)
        _check(lib().evxg_stream_restore(self.h, _ptr(buf), len(buf), _ptr(cuda_stream)))

    def set_timeout_ns(self, ns: int):
        """Bound on every device-side wait of this stream's kernels (5 s by default)."""
        _check(lib().evxg_stream_set_timeout_ns(self.h, int(ns)))

    def reset(self, cuda_stream=None):
        """Back to the state at creation (zero DPB slots and tables)."""
        _check(lib().evxg_stream_reset(self.h, _ptr(cuda_stream)))

    def fetch_tables(self, cuda_stream=None):
        bt = np.zeros(self.nblk * 28, np.uint8)
        prev = np.zeros(self.nblk * 28, np.uint8)
        sao = np.zeros(self.nblk * 16, np.uint8)
        lev = np.zeros(self.plane_elems, np.int16)
        _check(lib().evxg_fetch_tables(self.h, _ptr(bt), _ptr(prev), _ptr(sao), _ptr(lev), 0, _ptr(cuda_stream)))
        return dict(blocks=bt, prev_blocks=prev, sao=sao, levels=lev)

    def fetch_planes(self, slot: int, cuda_stream=None) -> np.ndarray:
        out = np.zeros(self.plane_elems, np.int16)
        _check(lib().evxg_fetch_planes(self.h, slot, _ptr(out), 0, _ptr(cuda_stream)))
        return out

    KERNELS = ("convert", "mb_wavefront", "deblock", "sao_rdo", "sao_merge", "sao_apply")

    def profile(self, enable: bool = True):
        _check(lib().evxg_stream_profile(self.h, int(enable)))

    def kernel_ms(self) -> dict:
        buf = (C.c_float * 6)()
        n = lib().evxg_stream_kernel_ms(self.h, buf, 6)
        if n < 0:
            raise EvxgError(-n, "kernel timing failed")
        return {self.KERNELS[i]: buf[i] for i in range(n)}

    def launch_count(self) -> int:
        return lib().evxg_last_launch_count(self.h)

    @property
    def mb_form(self) -> int:
        """MB_FORM_CLUSTER (three CTAs per macroblock row) or MB_FORM_SINGLE (one)."""
        return lib().evxg_stream_mb_form(self.h)

    @mb_form.setter
    def mb_form(self, form: int):
        _check(lib().evxg_stream_set_mb_form(self.h, int(form)))


class Decoder:
    """The decoder's pixel half on the device (engine_decode_frame after
    unserialize_slice, src/video/decode.cpp:560-612) for one stream of the
    reference build ``cfg`` names: ``decode_frame`` takes a frame's descriptor
    and the tables the entropy decoder produces (the layouts of
    :meth:`Stream.fetch_tables`) and returns the visible RGB24 frame."""

    def __init__(self, width: int, height: int, cfg="default"):
        self.width, self.height = int(width), int(height)
        self.cfg = config(cfg)
        h = C.c_void_p()
        _check(lib().evxg_decoder_create(self.width, self.height, C.byref(self.cfg), C.byref(h)))
        self.h = h
        self.aw, self.ah = (self.width + 15) & ~15, (self.height + 15) & ~15
        self.plane_elems = self.aw * self.ah + 2 * (self.aw // 2) * (self.ah // 2)

    def close(self):
        if getattr(self, "h", None):
            lib().evxg_decoder_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def decode_frame(self, frame18: bytes, blocks, sao, levels, rgb: bool = True, cuda_stream=None):
        """Decode one frame (host tables); returns the (H, W, 3) RGB24 frame, or None with rgb=False."""
        bt = np.ascontiguousarray(blocks)
        sa = np.ascontiguousarray(sao)
        lv = np.ascontiguousarray(levels, dtype=np.int16)
        out = np.empty((self.height, self.width, 3), np.uint8) if rgb else None
        _check(lib().evxg_decode_frame(self.h, frame18, _ptr(bt), _ptr(sa), _ptr(lv), 0, _ptr(out), 0,
                                       _ptr(cuda_stream)))
        self.sync(cuda_stream)
        return out

    def decode_record(self, data, rgb: bool = True, cuda_stream=None):
        """Decode the frame record at the start of data (bitstream order):
        returns (rgb frame or None, 18-byte descriptor, bytes the record used)."""
        buf = np.frombuffer(data, np.uint8)
        out = np.empty((self.height, self.width, 3), np.uint8) if rgb else None
        f = (C.c_uint8 * 18)()
        n = C.c_uint64(0)
        _check(lib().evxg_decoder_decode_record(self.h, _ptr(buf), len(buf), _ptr(out), f, C.byref(n),
                                                _ptr(cuda_stream)))
        return out, bytes(f), n.value

    def sync(self, cuda_stream=None):
        _check(lib().evxg_decoder_sync(self.h, _ptr(cuda_stream)))

    def set_timeout_ns(self, ns: int):
        _check(lib().evxg_decoder_set_timeout_ns(self.h, int(ns)))

    def reset(self, cuda_stream=None):
        _check(lib().evxg_decoder_reset(self.h, _ptr(cuda_stream)))

    def fetch_planes(self, slot: int, cuda_stream=None) -> np.ndarray:
        out = np.zeros(self.plane_elems, np.int16)
        _check(lib().evxg_decoder_fetch_planes(self.h, slot, _ptr(out), 0, _ptr(cuda_stream)))
        return out


class Muxer:
    """The packet container writer (evxg_muxer_*; the reference's evx_muxer)."""

    def __init__(self, path: str):
        h = C.c_void_p()
        _check(lib().evxg_muxer_open(os.fsencode(path), C.byref(h)))
        self.h = h

    def add_video_stream(self, width: int, height: int, frame_rate: float) -> int:
        sid = C.c_uint8()
        _check(lib().evxg_muxer_add_video_stream(self.h, width, height, frame_rate, C.byref(sid)))
        return sid.value

    def add_audio_stream(self, sample_rate: int, channels: int, bit_depth: int, quality: int) -> int:
        sid = C.c_uint8()
        _check(lib().evxg_muxer_add_audio_stream(self.h, sample_rate, channels, bit_depth, quality, C.byref(sid)))
        return sid.value

    def write_header(self):
        _check(lib().evxg_muxer_write_header(self.h))

    def write_packet(self, stream_id: int, stream_type: int, timestamp_us: int, payload: bytes):
        buf = np.frombuffer(bytes(payload), np.uint8)
        _check(lib().evxg_muxer_write_packet(self.h, stream_id, stream_type, timestamp_us, _ptr(buf), len(buf)))

    def close(self):
        if getattr(self, "h", None):
            h, self.h = self.h, None
            _check(lib().evxg_muxer_close(h))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Demuxer:
    """The packet container reader (evxg_demuxer_*; the reference's evx_demuxer):
    ``streams`` lists the descriptors, iterating yields (stream_id, stream_type,
    timestamp_us, payload) per packet."""

    def __init__(self, path: str):
        h = C.c_void_p()
        _check(lib().evxg_demuxer_open(os.fsencode(path), C.byref(h)))
        self.h = h
        self.streams = []
        for i in range(lib().evxg_demuxer_stream_count(self.h)):
            d = StreamDesc()
            _check(lib().evxg_demuxer_stream(self.h, i, C.byref(d)))
            self.streams.append(d)

    def __iter__(self):
        buf = np.empty(1 << 20, np.uint8)
        sid, stype, ts, n = C.c_uint8(), C.c_uint8(), C.c_uint64(), C.c_uint32()
        while True:
            rc = lib().evxg_demuxer_read_packet(self.h, C.byref(sid), C.byref(stype), C.byref(ts), _ptr(buf), len(buf),
                                                C.byref(n))
            if rc == OPERATION_COMPLETED:
                return
            if rc == CAPACITY_LIMIT:
                buf = np.empty(n.value, np.uint8)
                continue
            _check(rc)
            yield sid.value, stype.value, ts.value, buf[:n.value].tobytes()

    def close(self):
        if getattr(self, "h", None):
            lib().evxg_demuxer_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class StreamDecoder:
    """The reference's evx3_decoder (src/video/evx3.h:103-127) for a whole
    .evx stream of the build ``cfg`` names (evxg_stream_decoder_*, C++):
    ``decode(data)`` feeds the header and every frame record and drains the
    display buffer, returning the frames in display order as (H, W, 3) RGB24
    arrays.  Records need no size prefix: the entropy decoder finds each
    slice's end, so the I/P builds' concatenated records decode too."""

    def __init__(self, cfg="default"):
        self.cfg = config(cfg)
        h = C.c_void_p()
        _check(lib().evxg_stream_decoder_create(C.byref(self.cfg), C.byref(h)))
        self.h = h

    def decode(self, data: bytes):
        buf = np.frombuffer(bytes(data), np.uint8)
        if len(buf) < 14 or buf[:4].tobytes() != b"EVX1":
            raise EvxgError(8, "not an .evx stream (header)")
        self.width, self.height = struct.unpack_from("<HH", buf.tobytes()[:14], 10)
        _check(lib().evxg_stream_decoder_clear(self.h))
        frames, pos = [], 0
        out = np.empty((self.height, self.width, 3), np.uint8)
        used, ready = C.c_uint64(0), C.c_int(0)
        while pos < len(buf):
            _check(lib().evxg_stream_decoder_decode(self.h, C.c_void_p(buf.ctypes.data + pos), len(buf) - pos,
                                                    C.byref(used), _ptr(out), C.byref(ready)))
            pos += used.value
            if ready.value:
                frames.append(out.copy())
        while True:
            _check(lib().evxg_stream_decoder_flush(self.h, _ptr(out), C.byref(ready)))
            if not ready.value:
                return frames
            frames.append(out.copy())

    def close(self):
        if getattr(self, "h", None):
            lib().evxg_stream_decoder_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


NO_FRAME = struct.pack("<iIHIBBBB", -1, 0, 0, 0, 0, 0, 0, 0)   # a stream without a frame in a batch tick


class Batch:
    """Batched ticks over several streams (evxg_batch_*): one launch per stage
    for all streams, the tick replayed as a CUDA graph, two buffer parities.

    Per tick: write frames into input(i, p), encode(frames18, p), wait(p),
    read output(i, p).  frames18[i] is None for a stream without a frame."""

    def __init__(self, streams):
        self.streams = list(streams)
        arr = (C.c_void_p * len(self.streams))(*[s.h.value for s in self.streams])
        h = C.c_void_p()
        _check(lib().evxg_batch_create(arr, len(self.streams), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().evxg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def input(self, i: int, parity: int) -> np.ndarray:
        """Pinned (height, width, 3) uint8 buffer of stream i's next frame of this parity."""
        s = self.streams[i]
        p = lib().evxg_batch_input(self.h, i, parity)
        return np.ctypeslib.as_array(p, shape=(s.height, s.width, 3))

    def encode(self, frames18, parity: int, cuda_stream=None):
        buf = b"".join(NO_FRAME if f is None else f for f in frames18)
        _check(lib().evxg_batch_encode(self.h, buf, parity, _ptr(cuda_stream)))

    def wait(self, parity: int):
        _check(lib().evxg_batch_wait(self.h, parity))

    def output(self, i: int, parity: int) -> dict:
        """Copies of stream i's tables from the last tick of this parity (as Stream.fetch_tables)."""
        s = self.streams[i]
        ptrs = [C.c_void_p() for _ in range(4)]
        _check(lib().evxg_batch_output(self.h, i, parity, *[C.byref(x) for x in ptrs]))
        def arr(p, n, dt):
            return np.ctypeslib.as_array(C.cast(p, C.POINTER(dt)), shape=(n,)).copy()
        return dict(blocks=arr(ptrs[0], s.nblk * 28, C.c_uint8), prev_blocks=arr(ptrs[1], s.nblk * 28, C.c_uint8),
                    sao=arr(ptrs[2], s.nblk * 16, C.c_uint8), levels=arr(ptrs[3], s.plane_elems, C.c_int16))

    def launch_count(self) -> int:
        return lib().evxg_batch_launch_count(self.h)

    def set_timeout_ns(self, ns: int):
        _check(lib().evxg_batch_set_timeout_ns(self.h, int(ns)))

    @property
    def shape(self):
        v = [C.c_int() for _ in range(3)]
        _check(lib().evxg_batch_get_shape(self.h, *[C.byref(x) for x in v]))
        return tuple(x.value for x in v)   # (form, grid, policy)

    def set_shape(self, form: int, grid: int, policy: int):
        _check(lib().evxg_batch_set_shape(self.h, form, grid, policy))

    def autotune(self, cuda_stream=None) -> float:
        ms = C.c_float()
        _check(lib().evxg_batch_autotune(self.h, _ptr(cuda_stream), C.byref(ms)))
        return ms.value


class Server:
    """Request loop over live streams (evxg_server_*): admission by device
    memory budget, batched ticks of whatever frames are ready, results through
    a callback on the server's worker thread.

    results[stream_id] is that stream's list of records in bitstream order:
    frame18 and times (arrival, ready, launch, done in ns), plus the
    serializer's tables when keep_tables is set."""

    def __init__(self, hbm_budget_bytes: int, max_streams: int, keep_tables: bool = True, lanes: int | None = None):
        import threading
        self.keep_tables = keep_tables
        self.results = {}
        self.dims = {}
        self._lock = threading.Lock()
        self._cb = RESULT_CB(self._on_result)
        h = C.c_void_p()
        if lanes is None:
            _check(lib().evxg_server_create(int(hbm_budget_bytes), int(max_streams), self._cb, None, C.byref(h)))
        else:
            _check(lib().evxg_server_create_lanes(int(hbm_budget_bytes), int(max_streams), int(lanes), self._cb, None,
                                                  C.byref(h)))
        self.h = h

    def _on_result(self, user, sid, frame, bt, pv, sao, lev, times):
        t = times.contents
        rec = {"frame18": C.string_at(frame, 18),
               "times": (t.arrival_ns, t.ready_ns, t.launch_ns, t.done_ns)}
        if self.keep_tables:
            nblk, pe = self.dims[sid]
            def arr(p, n, dt):
                return np.ctypeslib.as_array(C.cast(p, C.POINTER(dt)), shape=(n,)).copy()
            rec.update(blocks=arr(bt, nblk * 28, C.c_uint8), prev_blocks=arr(pv, nblk * 28, C.c_uint8),
                       sao=arr(sao, nblk * 16, C.c_uint8), levels=arr(lev, pe, C.c_int16))
        with self._lock:
            self.results.setdefault(sid, []).append(rec)

    def open(self, width: int, height: int, quality: int = 8, cfg="default") -> int:
        sid = C.c_uint32()
        aw, ah = (width + 15) & ~15, (height + 15) & ~15
        c = config(cfg)
        _check(lib().evxg_server_open_config(self.h, width, height, quality, C.byref(c), C.byref(sid)))
        self.dims[sid.value] = ((aw // 16) * (ah // 16), aw * ah + 2 * (aw // 2) * (ah // 2))
        self.results.setdefault(sid.value, [])
        return sid.value

    def submit(self, sid: int, rgb, arrival_ns: int = 0):
        rgb = np.ascontiguousarray(rgb, dtype=np.uint8)
        _check(lib().evxg_server_submit(self.h, sid, rgb.ctypes.data_as(C.c_void_p), int(arrival_ns)))

    def insert_intra(self, sid: int):
        _check(lib().evxg_server_insert_intra(self.h, sid))

    def close_stream(self, sid: int):
        _check(lib().evxg_server_close(self.h, sid))

    def drain(self):
        _check(lib().evxg_server_drain(self.h))

    def cancel(self, sid: int):
        """Drop the stream's frames not yet in a tick; those in flight are delivered."""
        _check(lib().evxg_server_cancel(self.h, sid))

    def evict(self, sid: int):
        """Move the stream's device state to host memory, freeing its device memory."""
        _check(lib().evxg_server_evict(self.h, sid))

    def restore(self, sid: int):
        """Bring an evicted stream back onto the device; it continues bit-identically."""
        _check(lib().evxg_server_restore(self.h, sid))

    def stats(self) -> dict:
        v = [C.c_uint64() for _ in range(4)]
        _check(lib().evxg_server_stats(self.h, *[C.byref(x) for x in v]))
        return dict(zip(("frames", "ticks", "rebuilds", "bytes_in_use"), (x.value for x in v)))

    @staticmethod
    def now_ns() -> int:
        return lib().evxg_server_now_ns()

    def close(self):
        if getattr(self, "h", None):
            lib().evxg_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Encoder:
    """evx3_encoder mirror: frames in, per-frame table records out (bitstream order)."""

    def __init__(self, quality: int | None = None, cfg="default", bitstream: bool = False):
        """bitstream=True: the encoder also emits the .evx stream into self.stream."""
        self.records = []
        self.stream = bytearray()
        self.cfg = config(cfg)
        self._cb = FRAME_CB(self._on_frame)
        h = C.c_void_p()
        _check(lib().evxg_encoder_create_config(self._cb, None, C.byref(self.cfg), C.byref(h)))
        self.h = h
        if bitstream:
            self._out = BYTES_CB(lambda user, p, n: self.stream.extend(C.string_at(p, n)))
            _check(lib().evxg_encoder_set_output(self.h, self._out, None))
        if quality is not None:
            self.set_quality(quality)

    def _on_frame(self, user, frame, blocks, prev, sao, levels):
        st = lib().evxg_encoder_stream(self.h)
        d = [C.c_uint32() for _ in range(4)]
        lib().evxg_stream_dims(st, *[C.byref(x) for x in d])
        aw, ah, mbw, mbh = (x.value for x in d)
        nblk, ne = mbw * mbh, aw * ah + 2 * (aw // 2) * (ah // 2)
        self.records.append(dict(
            frame18=C.string_at(frame, 18),
            blocks=np.frombuffer(C.string_at(blocks, nblk * 28), np.uint8).copy(),
            prev_blocks=np.frombuffer(C.string_at(prev, nblk * 28), np.uint8).copy(),
            sao=np.frombuffer(C.string_at(sao, nblk * 16), np.uint8).copy(),
            levels=np.frombuffer(C.string_at(levels, ne * 2), np.int16).copy()))

    def set_quality(self, q: int):
        _check(lib().evxg_encoder_set_quality(self.h, q))

    def insert_intra(self):
        _check(lib().evxg_encoder_insert_intra(self.h))

    def encode(self, rgb: np.ndarray):
        rgb = np.ascontiguousarray(rgb, dtype=np.uint8)
        H, W = rgb.shape[:2]
        _check(lib().evxg_encoder_encode(self.h, _ptr(rgb), W, H))

    def flush(self):
        _check(lib().evxg_encoder_flush(self.h))

    PEEK = {"source": 0, "prediction": 1, "block_table": 2, "quant_table": 3, "spmp_table": 4,
            "block_variance": 5, "destination": 6}

    def peek(self, which, width: int, height: int) -> np.ndarray:
        """evx3_encoder::peek: the (H, W, 3) RGB24 view ``which`` (a name of PEEK
        or its number) of the encoder's state after the last encode call."""
        out = np.zeros((height, width, 3), np.uint8)
        _check(lib().evxg_encoder_peek(self.h, self.PEEK.get(which, which), _ptr(out)))
        return out

    def clear(self):
        _check(lib().evxg_encoder_clear(self.h))

    def close(self):
        if getattr(self, "h", None):
            lib().evxg_encoder_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
