"""Command-line encoder and decoder for raw RGB24 files, the reference's
evx_encode / evx_decode tools (tools/evx_encode.cpp, tools/evx_decode.cpp)
without FFmpeg: input and output are raw RGB24 frames (width*height*3 bytes
each, back to back), the coded file is the EVX3 packet container.

    python -m chicago_b200.tools encode in.rgb out.evx3 --width 1920 --height 1080 --fps 30 --quality 8 --cfg ip3
    python -m chicago_b200.tools decode in.evx3 out.rgb --cfg ip3

The video stream's packets are cut the way the reference tool cuts its
encoder's output (tools/evx_encode.cpp:185-275): with B frames, the first
non-empty output whole (stream header and first record), then one
size-prefixed record per packet, flush() included; without B frames, one
packet per encode() call; packet k is stamped k * 10^6 / fps microseconds
(bitstream order).  Encoding runs on the GPU (Encoder), decoding through the
host entropy decoder and the GPU pixel half (StreamDecoder).
"""
from __future__ import annotations

import argparse
import struct
import sys

import numpy as np

import chicago_b200 as cb


def split_records(chunk: bytes):
    """The size-prefixed frame records of one encoder output (u32 size + payload each)."""
    pos, out = 0, []
    while pos + 4 <= len(chunk):
        (n,) = struct.unpack_from("<I", chunk, pos)
        if pos + 4 + n > len(chunk):
            break
        out.append(chunk[pos:pos + 4 + n])
        pos += 4 + n
    return out


class Packetizer:
    """Cuts an encoder's per-call outputs into container packets as the
    reference tool does, with its timestamps."""

    def __init__(self, b_frames: bool, fps: float):
        self.b_frames, self.fps = b_frames, fps
        self.count = 0
        self.header_done = False
        self.packets = []   # (timestamp_us, payload)

    def _emit(self, payload: bytes):
        self.packets.append((int(self.count * 1000000.0 / self.fps), payload))
        self.count += 1

    def output(self, chunk: bytes):
        """The bytes one encode() call produced."""
        if not self.b_frames:
            self._emit(chunk)
        elif chunk:
            if not self.header_done:
                self._emit(chunk)
                self.header_done = True
            else:
                for r in split_records(chunk):
                    self._emit(r)

    def flushed(self, chunk: bytes):
        """The bytes flush() produced (builds with B frames)."""
        for r in split_records(chunk):
            self._emit(r)


def read_frames(path: str, width: int, height: int):
    raw = np.fromfile(path, np.uint8)
    fb = width * height * 3
    if raw.size % fb:
        raise ValueError(f"{path}: {raw.size} bytes is not a whole number of {width}x{height} RGB24 frames")
    return raw.reshape(-1, height, width, 3)


def encode_frames(frames: np.ndarray, fps: float, quality: int, cfg: str = "default", intra_only: bool = False):
    """Encode (T,H,W,3) RGB24 frames on the GPU; returns the container packets."""
    T, H, W, _ = frames.shape
    enc = cb.Encoder(quality=quality, cfg=cfg, bitstream=True)
    pk = Packetizer(bool(cb.config(cfg).b_frames), fps)
    for t in range(T):
        if intra_only:
            enc.insert_intra()
        n0 = len(enc.stream)
        enc.encode(frames[t])
        pk.output(bytes(enc.stream[n0:]))
    n0 = len(enc.stream)
    enc.flush()
    if cb.config(cfg).b_frames:
        pk.flushed(bytes(enc.stream[n0:]))
    enc.close()
    return pk.packets


def write_container(path: str, width: int, height: int, fps: float, packets):
    mux = cb.Muxer(path)
    vid = mux.add_video_stream(width, height, fps)
    mux.write_header()
    for ts, payload in packets:
        mux.write_packet(vid, cb.STREAM_TYPE_VIDEO, ts, payload)
    mux.close()


def encode_file(src: str, dst: str, width: int, height: int, fps: float, quality: int, cfg: str = "default",
                intra_only: bool = False) -> dict:
    frames = read_frames(src, width, height)
    packets = encode_frames(frames, fps, quality, cfg, intra_only)
    write_container(dst, width, height, fps, packets)
    return {"frames": len(frames), "packets": len(packets), "bytes": sum(len(p) for _, p in packets)}


def decode_container(path: str, cfg: str = "default"):
    """The video stream of a container decoded to RGB24 frames in display order."""
    dmx = cb.Demuxer(path)
    vids = [s.stream_id for s in dmx.streams if s.stream_type == cb.STREAM_TYPE_VIDEO]
    if not vids:
        raise cb.EvxgError(8, f"{path}: no video stream")
    data = b"".join(p for sid, stype, _, p in dmx if sid == vids[0] and stype == cb.STREAM_TYPE_VIDEO)
    dmx.close()
    return cb.StreamDecoder(cfg).decode(data)


def decode_file(src: str, dst: str, cfg: str = "default") -> dict:
    frames = decode_container(src, cfg)
    with open(dst, "wb") as f:
        for fr in frames:
            f.write(np.ascontiguousarray(fr).tobytes())
    return {"frames": len(frames)}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m chicago_b200.tools", description=__doc__.split("\n\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    e = sub.add_parser("encode", help="raw RGB24 frames -> EVX3 container")
    e.add_argument("src")
    e.add_argument("dst")
    e.add_argument("--width", type=int, required=True)
    e.add_argument("--height", type=int, required=True)
    e.add_argument("--fps", type=float, default=30.0)
    e.add_argument("--quality", type=int, default=8)
    e.add_argument("--cfg", default="default", choices=sorted(cb.CONFIGS))
    e.add_argument("--intra-only", action="store_true")
    d = sub.add_parser("decode", help="EVX3 container -> raw RGB24 frames")
    d.add_argument("src")
    d.add_argument("dst")
    d.add_argument("--cfg", default="default", choices=sorted(cb.CONFIGS))
    a = ap.parse_args(argv)
    if a.cmd == "encode":
        r = encode_file(a.src, a.dst, a.width, a.height, a.fps, a.quality, a.cfg, a.intra_only)
    else:
        r = decode_file(a.src, a.dst, a.cfg)
    print(r)
    return 0


if __name__ == "__main__":
    sys.exit(main())
